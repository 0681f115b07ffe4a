// CSV particle import and frame export with the reference's semantics
// (src/import.cpp, src/export.cpp): the same files, columns, skipped header and
// blank lines, field rules and error messages.  The parser reads each file in
// one piece and converts numbers with std::from_chars where the text is a
// plain decimal (falling back to std::stoi/std::stod, the reference's
// conversions, for anything else), instead of a stringstream per field.
#include <algorithm>
#include <charconv>
#include <cstdint>
#include <cstring>
#include <exception>
#include <fcntl.h>
#include <fstream>
#include <iomanip>
#include <iterator>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <thread>
#include <vector>

#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "snow/export.hpp"
#include "snow/import.hpp"
#include "snow_host_detail.hpp"
#include "snow_io.h"

namespace
{
std::string read_file(const std::string& filename)
{
    std::ifstream file(filename, std::ios::binary | std::ios::ate);
    if (!file.is_open()) throw std::runtime_error{"File not open: " + filename};
    const std::streamoff size = file.tellg();
    if (size < 0)  // not seekable (a pipe): read it as a stream
    {
        file.clear();
        return std::string(std::istreambuf_iterator<char>(file), std::istreambuf_iterator<char>());
    }
    std::string text(static_cast<std::size_t>(size), '\0');
    file.seekg(0);
    file.read(text.data(), size);
    text.resize(static_cast<std::size_t>(file.gcount()));
    return text;
}

// Runs parse_line over lines [1, size) (line 0 is the header) in contiguous
// parts on several threads, each into its own vector, and returns the
// results in file order.  An exception is rethrown from the first line that
// raised one in file order -- the one a sequential read stops at -- so the
// error is the reference's.
template <typename T, typename F>
std::vector<T> parse_body(const std::vector<std::string_view>& lines, F&& parse_line)
{
    constexpr std::size_t kLinesPerPart = 32768;
    const std::size_t body = lines.size() - 1;
    const std::size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const std::size_t parts = std::max<std::size_t>(1, std::min<std::size_t>({hw, 32, body / kLinesPerPart}));
    std::vector<std::vector<T>> out(parts);
    std::vector<std::exception_ptr> err(parts);
    auto work = [&](std::size_t k) {
        const std::size_t lo = 1 + body * k / parts, hi = 1 + body * (k + 1) / parts;
        try
        {
            out[k].reserve(hi - lo);
            for (std::size_t i = lo; i < hi; ++i)
                if (!lines[i].empty()) out[k].push_back(parse_line(lines[i]));
        }
        catch (...)
        {
            err[k] = std::current_exception();
        }
    };
    std::vector<std::thread> pool;
    for (std::size_t k = 1; k < parts; ++k) pool.emplace_back(work, k);
    work(0);
    for (auto& t : pool) t.join();
    for (const auto& e : err)
        if (e) std::rethrow_exception(e);
    if (parts == 1) return std::move(out[0]);
    std::size_t total = 0;
    for (const auto& v : out) total += v.size();
    std::vector<T> all;
    all.reserve(total);
    for (auto& v : out) all.insert(all.end(), v.begin(), v.end());
    return all;
}

// Lines as std::getline yields them: split at '\n', no empty final segment.
std::vector<std::string_view> lines_of(const std::string& text)
{
    std::vector<std::string_view> out;
    std::size_t pos = 0;
    while (pos < text.size())
    {
        const std::size_t nl = text.find('\n', pos);
        if (nl == std::string::npos)
        {
            out.emplace_back(text.data() + pos, text.size() - pos);
            break;
        }
        out.emplace_back(text.data() + pos, nl - pos);
        pos = nl + 1;
    }
    return out;
}

// Comma-separated fields of one line, read as std::getline(row, field, ',')
// reads them: a read past the last character fails ("Missing"); a trailing
// '\r' is dropped; an empty field is an error ("Empty").
class Fields
{
public:
    explicit Fields(std::string_view line) : line_(line) {}
    std::string_view next(const char* column)
    {
        if (pos_ >= line_.size()) throw std::runtime_error{std::string("Missing CSV field: ") + column};
        const std::size_t comma = line_.find(',', pos_);
        std::string_view f = comma == std::string_view::npos ? line_.substr(pos_) : line_.substr(pos_, comma - pos_);
        pos_ = comma == std::string_view::npos ? line_.size() : comma + 1;
        if (!f.empty() && f.back() == '\r') f.remove_suffix(1);
        if (f.empty()) throw std::runtime_error{std::string("Empty CSV field: ") + column};
        return f;
    }

private:
    std::string_view line_;
    std::size_t pos_ = 0;
};

bool plain_number(std::string_view f)
{
    const char c = f.front();
    if (!(c == '-' || c == '.' || (c >= '0' && c <= '9'))) return false;
    return f.find_first_of("xX") == std::string_view::npos;
}

int to_int(std::string_view f)
{
    int v = 0;
    if (plain_number(f) && f.find('.') == std::string_view::npos)
    {
        const auto r = std::from_chars(f.data(), f.data() + f.size(), v);
        if (r.ec == std::errc()) return v;
    }
    return std::stoi(std::string(f));  // the reference's conversion and exceptions
}

double to_double(std::string_view f)
{
    double v = 0.0;
    if (plain_number(f))
    {
        const auto r = std::from_chars(f.data(), f.data() + f.size(), v);
        if (r.ec == std::errc() && r.ptr != f.data()) return v;
    }
    return std::stod(std::string(f));
}
}  // namespace

std::map<int, ParticleGroup> import_groups(const std::string& filename)
{
    const std::string text = read_file(filename);
    const auto lines = lines_of(text);
    if (lines.empty()) throw std::runtime_error{"Group data file is empty: " + filename};
    std::map<int, ParticleGroup> groups;
    for (std::size_t k = 1; k < lines.size(); ++k)
    {
        if (lines[k].empty()) continue;
        Fields row(lines[k]);
        const int id = to_int(row.next("group_ID"));
        const double vx = to_double(row.next("v_x"));
        const double vy = to_double(row.next("v_y"));
        const double vz = to_double(row.next("v_z"));
        const double m = to_double(row.next("m"));
        if (!groups.emplace(id, ParticleGroup{Eigen::Vector3d{vx, vy, vz}, m}).second)
            throw std::runtime_error{"Duplicate group id: " + std::to_string(id)};
    }
    return groups;
}

std::vector<ParticleSeed> import_particle_seeds(const std::string& filename)
{
    const std::string text = read_file(filename);
    const auto lines = lines_of(text);
    if (lines.empty()) throw std::runtime_error{"Particle data file is empty: " + filename};
    return parse_body<ParticleSeed>(lines, [](std::string_view line) {
        Fields row(line);
        const int id = to_int(row.next("group_ID"));
        const double x = to_double(row.next("x"));
        const double y = to_double(row.next("y"));
        const double z = to_double(row.next("z"));
        return ParticleSeed{id, Eigen::Vector3d{x, y, z}};
    });
}

std::vector<Particle> assemble_particles(const std::vector<ParticleSeed>& seeds,
                                         const std::map<int, ParticleGroup>& groups)
{
    std::vector<Particle> particles;
    particles.reserve(seeds.size());
    for (const ParticleSeed& s : seeds)
    {
        const auto it = groups.find(s.group_id);
        if (it == groups.end())
            throw std::runtime_error{"Particle references undefined group id: " + std::to_string(s.group_id)};
        particles.emplace_back(s.position, it->second.velocity, it->second.mass, 0.0);
    }
    return particles;
}

namespace
{
// A file's bytes for parsing: a regular file is mapped read-only, so its pages
// are read in by the threads that parse them; anything else is read whole.
class FileBytes
{
public:
    explicit FileBytes(const std::string& filename)
    {
        const int fd = ::open(filename.c_str(), O_RDONLY);
        if (fd < 0) throw std::runtime_error{"File not open: " + filename};
        struct stat st{};
        if (::fstat(fd, &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0)
        {
            void* m = ::mmap(nullptr, static_cast<std::size_t>(st.st_size), PROT_READ, MAP_PRIVATE, fd, 0);
            if (m != MAP_FAILED)
            {
                map_ = m;
                size_ = static_cast<std::size_t>(st.st_size);
            }
        }
        ::close(fd);
        if (!map_) buf_ = read_file(filename);
    }
    ~FileBytes()
    {
        if (map_) ::munmap(map_, size_);
    }
    FileBytes(const FileBytes&) = delete;
    FileBytes& operator=(const FileBytes&) = delete;
    std::string_view view() const { return map_ ? std::string_view(static_cast<const char*>(map_), size_) : buf_; }

private:
    void* map_ = nullptr;
    std::size_t size_ = 0;
    std::string buf_;
};
}  // namespace

namespace
{
// A particle line's group prototype and position.
struct Seed
{
    const Particle* proto;
    double x, y, z;
};
// particles.csv parsed in parts: each part's seeds in file order.
struct ParsedParticles
{
    std::map<int, Particle> proto;  // one particle per group, copied for each of its particles
    std::vector<std::vector<Seed>> parts;
    std::size_t total = 0;
};

// Runs work(k) for k in [0, parts) on that many threads (k = 0 on this one).
template <typename F>
void run_parts(std::size_t parts, F&& work)
{
    std::vector<std::thread> pool;
    for (std::size_t k = 1; k < parts; ++k) pool.emplace_back(work, k);
    work(0);
    for (auto& t : pool) t.join();
}

// import_particles (src/import.cpp:131-136) up to the assembly, in one
// parallel pass over particles.csv: the body after the header line is cut
// into byte ranges at line starts, and each thread parses its lines into its
// own part.  The errors are the sequential ones: a malformed line anywhere
// comes before an undefined group id (the reference reads every seed before
// assembling), and of each kind the first in file order is reported.
ParsedParticles parse_particles(const std::string& filename_group, const std::string& filename_particle_seed)
{
    ParsedParticles res;
    const auto groups = import_groups(filename_group);
    const FileBytes file(filename_particle_seed);
    const std::string_view text = file.view();
    if (text.empty()) throw std::runtime_error{"Particle data file is empty: " + filename_particle_seed};
    const std::size_t header_end = text.find('\n');
    const std::size_t body = header_end == std::string_view::npos ? text.size() : header_end + 1;
    for (const auto& [id, g] : groups)
        res.proto.emplace(id, Particle(Eigen::Vector3d::Zero(), g.velocity, g.mass, 0.0));

    constexpr std::size_t kBytesPerPart = std::size_t(1) << 20;
    const std::size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const std::size_t parts =
        std::max<std::size_t>(1, std::min<std::size_t>({hw, 32, (text.size() - body) / kBytesPerPart}));
    std::vector<std::size_t> cut(parts + 1, text.size());
    cut[0] = body;
    for (std::size_t k = 1; k < parts; ++k)
    {
        std::size_t b = std::max(body + (text.size() - body) * k / parts, cut[k - 1]);
        if (b > body && b < text.size() && text[b - 1] != '\n')
        {
            const std::size_t nl = text.find('\n', b);
            b = nl == std::string_view::npos ? text.size() : nl + 1;
        }
        cut[k] = b;
    }
    res.parts.resize(parts);
    std::vector<std::exception_ptr> parse_error(parts);
    std::vector<char> undefined(parts, 0);
    std::vector<int> undefined_id(parts, 0);
    const auto& proto = res.proto;
    run_parts(parts, [&](std::size_t k) {
        std::vector<Seed>& seeds = res.parts[k];
        seeds.reserve((cut[k + 1] - cut[k]) / 24 + 1);
        try
        {
            for (std::size_t pos = cut[k]; pos < cut[k + 1];)
            {
                const std::size_t nl = text.find('\n', pos);
                const std::size_t end = std::min(nl == std::string_view::npos ? text.size() : nl, cut[k + 1]);
                const std::string_view line = text.substr(pos, end - pos);
                pos = end + 1;
                if (line.empty()) continue;
                Fields row(line);
                const int id = to_int(row.next("group_ID"));
                const double x = to_double(row.next("x"));
                const double y = to_double(row.next("y"));
                const double z = to_double(row.next("z"));
                const auto it = proto.find(id);
                if (it == proto.end())
                {
                    if (!undefined[k]) undefined_id[k] = id;
                    undefined[k] = 1;
                    continue;
                }
                seeds.push_back(Seed{&it->second, x, y, z});
            }
        }
        catch (...)
        {
            parse_error[k] = std::current_exception();
        }
    });
    for (const auto& e : parse_error)
        if (e) std::rethrow_exception(e);
    for (std::size_t k = 0; k < parts; ++k)
        if (undefined[k])
            throw std::runtime_error{"Particle references undefined group id: " + std::to_string(undefined_id[k])};
    for (const auto& seeds : res.parts) res.total += seeds.size();
    return res;
}

// Writes the parsed particles as records into `out` (total x 26 doubles), each
// part on its own thread.
void fill_records(const ParsedParticles& pp, double* out)
{
    std::vector<std::size_t> offset(pp.parts.size() + 1, 0);
    for (std::size_t k = 0; k < pp.parts.size(); ++k) offset[k + 1] = offset[k] + pp.parts[k].size();
    run_parts(pp.parts.size(), [&](std::size_t k) {
        double* rec = out + SNOW_RECORD_DOUBLES * offset[k];
        for (const Seed& sd : pp.parts[k])
        {
            std::memcpy(rec, sd.proto, sizeof(Particle));
            rec[0] = sd.x;
            rec[1] = sd.y;
            rec[2] = sd.z;
            rec += SNOW_RECORD_DOUBLES;
        }
    });
}
}  // namespace

// The parsed particles, assembled into the vector in file order; its storage
// is faulted in on all threads first, so that the one pass that fills it runs
// at memory speed.
std::vector<Particle> import_particles(const std::string& filename_group, const std::string& filename_particle_seed)
{
    const ParsedParticles pp = parse_particles(filename_group, filename_particle_seed);
    std::vector<Particle> all;
    all.reserve(pp.total);
    if (pp.total > 0)
    {
        unsigned char* raw = reinterpret_cast<unsigned char*>(all.data());
        const std::size_t bytes = pp.total * sizeof(Particle);
        const std::uintptr_t a = (reinterpret_cast<std::uintptr_t>(raw) + 4095) & ~std::uintptr_t(4095);
        const std::uintptr_t e = (reinterpret_cast<std::uintptr_t>(raw) + bytes) & ~std::uintptr_t(4095);
        if (e > a) ::madvise(reinterpret_cast<void*>(a), e - a, MADV_HUGEPAGE);
        const std::size_t parts = pp.parts.size();
        run_parts(parts, [&](std::size_t k) {
            const std::size_t lo = bytes * k / parts, hi = bytes * (k + 1) / parts;
            std::memset(raw + lo, 0, hi - lo);
        });
    }
    for (const auto& seeds : pp.parts)
        for (const Seed& sd : seeds)
        {
            all.push_back(*sd.proto);
            Particle& q = all.back();
            q.x_p[0] = sd.x;
            q.x_p[1] = sd.y;
            q.x_p[2] = sd.z;
        }
    return all;
}

namespace
{
// One number as the default stream formatting writes it (export.cpp:13-19:
// operator<< on a double, precision 6, %g style), via std::to_chars in its
// general format with the same precision.
char* put_number(char* at, double v)
{
    return std::to_chars(at, at + 32, v, std::chars_format::general, 6).ptr;
}

// Rows [lo, hi) of a frame: "x,-z,y\n" per particle; `stride` doubles from one
// particle's x to the next one's (26 for records, 3 for positions).
char* put_rows(char* at, const double* xyz, std::size_t stride, std::size_t lo, std::size_t hi)
{
    for (std::size_t i = lo; i < hi; ++i)
    {
        const double* p = xyz + stride * i;
        at = put_number(at, p[0]);
        *at++ = ',';
        at = put_number(at, p[2] * -1);
        *at++ = ',';
        at = put_number(at, p[1]);
        *at++ = '\n';
    }
    return at;
}

// output/frame_<frame>.csv with header "x,y,z" and rows (x, -z, y), default
// stream formatting (export.cpp:10-22).  Large frames are formatted by several
// threads, each into its own buffer, and written in order in one pass.
void write_frame(const double* xyz, std::size_t stride, std::size_t n, int frame_no)
{
    std::ostringstream name;
    name << "output/frame_" << std::setw(6) << std::setfill('0') << frame_no << ".csv";
    std::ofstream file{name.str(), std::ios::binary};
    constexpr std::size_t kRowBytes = 3 * 32, kRowsPerThread = 16384;
    const std::size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const std::size_t parts = std::max<std::size_t>(1, std::min<std::size_t>({hw, 32, n / kRowsPerThread}));
    std::vector<std::string> out(parts);
    std::vector<std::size_t> used(parts, 0);
    auto work = [&](std::size_t k) {
        const std::size_t lo = n * k / parts, hi = n * (k + 1) / parts;
        out[k].resize((hi - lo) * kRowBytes);
        used[k] = put_rows(out[k].data(), xyz, stride, lo, hi) - out[k].data();
    };
    std::vector<std::thread> pool;
    for (std::size_t k = 1; k < parts; ++k) pool.emplace_back(work, k);
    work(0);
    for (auto& t : pool) t.join();
    file.write("x,y,z\n", 6);
    for (std::size_t k = 0; k < parts; ++k) file.write(out[k].data(), static_cast<std::streamsize>(used[k]));
}

std::mutex g_export_mu;
std::vector<std::thread> g_exports;
}  // namespace

void export_particles(const std::vector<Particle>& particles, int frame_no)
{
    // A vector kept on the GPU by resident stepping: its positions are read back.
    const std::size_t n = particles.size();
    std::unique_ptr<double[]> fresh;
    if (n > 0)
    {
        fresh.reset(new double[3 * n]);
        if (snow_host_resident_positions(particles, fresh.get()))
        {
            write_frame(fresh.get(), 3, n, frame_no);
            return;
        }
    }
    write_frame(reinterpret_cast<const double*>(particles.data()), SNOW_RECORD_DOUBLES, n, frame_no);
}

namespace snow::gpu
{
void export_particles_async(const std::vector<Particle>& particles, int frame_no)
{
    // the positions now (from the GPU when the vector is resident), the file later
    const std::size_t n = particles.size();
    std::shared_ptr<double[]> xyz(new double[3 * std::max<std::size_t>(n, 1)]);
    if (n > 0 && !snow_host_resident_positions(particles, xyz.get()))
        for (std::size_t i = 0; i < n; ++i)
            std::memcpy(&xyz[3 * i], &particles[i].x_p[0], 3 * sizeof(double));
    std::lock_guard<std::mutex> lock(g_export_mu);
    g_exports.emplace_back([xyz, n, frame_no] { write_frame(xyz.get(), 3, n, frame_no); });
}

void wait_exports()
{
    std::vector<std::thread> jobs;
    {
        std::lock_guard<std::mutex> lock(g_export_mu);
        jobs.swap(g_exports);
    }
    for (auto& t : jobs) t.join();
}
}  // namespace snow::gpu

// ---------------------------------------------------------------- C ABI
// include/snow_io.h: the importer and the frame writer above for callers
// that bind C (ctypes, cgo, JNI).

namespace
{
thread_local std::string g_io_error;
}

extern "C" int64_t snow_io_import(const char* groups_csv, const char* particles_csv, double* records,
                                  int64_t capacity)
{
    try
    {
        if (!groups_csv || !particles_csv) throw std::runtime_error("snow_io_import: NULL file name");
        // parsed on all threads and written straight into the caller's records
        const ParsedParticles pp = parse_particles(groups_csv, particles_csv);
        const auto n = static_cast<int64_t>(pp.total);
        if (records)
        {
            if (n > capacity) return -2;
            fill_records(pp, records);
        }
        return n;
    }
    catch (const std::exception& e)
    {
        g_io_error = e.what();
        return -1;
    }
}

extern "C" int snow_io_export(const double* records, int64_t n, int frame_no)
{
    try
    {
        if (n < 0 || (n > 0 && !records)) throw std::runtime_error("snow_io_export: bad record array");
        write_frame(records, SNOW_RECORD_DOUBLES, static_cast<std::size_t>(n), frame_no);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_io_error = e.what();
        return -1;
    }
}

extern "C" const char* snow_io_last_error(void) { return g_io_error.c_str(); }
