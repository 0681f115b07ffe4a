/*
 * snow_io.h -- C ABI of the particle input/output of the drop-in library
 * (libsnow.so, host code; no GPU work except the read-back of a resident
 * vector, which these entry points do not touch).
 *
 * Reference interfaces replaced (reference tree paths):
 *   snow_io_import   import_particles(groups_csv, particles_csv)   include/snow/import.hpp:25, src/import.cpp:131-136
 *   snow_io_export   export_particles(particles, frame_no)         include/snow/export.hpp:8, src/export.cpp:10-22
 *
 * Records are the 26-double particle records of snow_gpu.h.  The files have
 * the reference's format: groups.csv (group_id,vx,vy,vz,mass) and
 * particles.csv (group_id,x,y,z), a header line each, blank lines ignored;
 * frames go to output/frame_<6-digit frame>.csv under the current directory
 * with header "x,y,z" and rows (x, -z, y).
 */
#ifndef SNOW_IO_H
#define SNOW_IO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Parses both files and returns the particle count; when `records` is not NULL
 * and `capacity` >= that count, also writes the records (V_p0 = 0, F_E = F_P =
 * I, as assemble_particles leaves them).  Returns -1 on a file or format error
 * (the reference's std::runtime_error text is in snow_io_last_error()) and -2
 * when the count exceeds `capacity`. */
int64_t snow_io_import(const char* groups_csv, const char* particles_csv, double* records,
                       int64_t capacity);

/* Writes output/frame_<frame_no>.csv for n records.  0 on success, -1 on error. */
int snow_io_export(const double* records, int64_t n, int frame_no);

/* Text of the last error on the calling thread. */
const char* snow_io_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* SNOW_IO_H */
