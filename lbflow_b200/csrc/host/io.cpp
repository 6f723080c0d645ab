// File formats (see io.h).
#include "io.h"

#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>

namespace lbfhost {

std::vector<uint8_t> loadGeometry(const std::string& path, std::size_t n)
{
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("FileRaw::Load() - Can not open file for input.");
    std::vector<uint8_t> g(n);
    const std::size_t got = n ? std::fread(g.data(), 1, n, f) : 0;
    std::fclose(f);
    if (got != n) throw std::runtime_error("FileRaw::Load() - Failed to read from raw file");
    return g;
}

std::string stepName(const std::string& outPath, std::size_t t, const char* ext)
{
    std::ostringstream os;
    os << outPath << "." << std::setw(10) << std::setfill('0') << t << ext;
    return os.str();
}

namespace {
// Output file written sequentially with write(2) straight from the caller's
// buffer (no stdio copy), with every failure reported.
class Sink {
public:
    Sink(const std::string& path, const char* openError) : fd_(::open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644))
    {
        if (fd_ < 0) throw std::runtime_error(openError);
    }
    ~Sink() { if (fd_ >= 0) ::close(fd_); }
    void put(const void* p, std::size_t bytes, const char* error)
    {
        const char* c = static_cast<const char*>(p);
        while (bytes) {
            const ssize_t w = ::write(fd_, c, bytes);
            if (w <= 0) throw std::runtime_error(error);
            c += w;
            bytes -= (std::size_t)w;
        }
    }
    void close(const char* error)
    {
        const int fd = fd_;
        fd_ = -1;
        if (::close(fd) != 0) throw std::runtime_error(error);
    }
private:
    int fd_;
};

const char kSaveError[] = "FileRaw::Save() - Failed to save to file";
}  // namespace

namespace {
// VTK ImageData XML header up to the start of the appended data.
std::string vtiHeader(const std::vector<std::size_t>& sz, const std::vector<std::string>& scalars,
                      const std::string& vector, int components)
{
    const std::size_t D = sz.size();
    std::size_t N = 1;
    for (std::size_t n : sz) N *= n;
    // Extents are listed x first (reference order reversed), padded to 3D.
    std::ostringstream ext;
    for (std::size_t d = D; d > 0; --d) ext << "0 " << sz[d - 1] - 1 << " ";
    for (std::size_t d = 3 - D; d > 0; --d) ext << "0 0 ";
    std::ostringstream h;
    h << "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">"
      << "<ImageData WholeExtent=\" " << ext.str() << "\" Origin=\"0 0 0\" Spacing=\"1 1 1\">"
      << "<Piece Extent=\"" << ext.str() << "\"><PointData Scalars=\"";
    for (const std::string& s : scalars) h << s << " ";
    h << "\" Vectors=\"" << vector << " \" >";
    std::size_t offset = 0;
    for (const std::string& s : scalars) {
        h << "<DataArray type=\"Float64\" Name=\"" << s << "\" format=\"appended\" offset=\""
          << offset << "\"/>";
        offset += N * sizeof(double) + sizeof(uint64_t);
    }
    h << "<DataArray type=\"Float64\" Name=\"" << vector << "\" NumberOfComponents=\"" << components
      << "\" format=\"appended\" offset=\"" << offset << "\"/>";
    h << "</PointData><CellData></CellData></Piece></ImageData><AppendedData encoding=\"raw\">_";
    return h.str();
}
}  // namespace

void writeVtiBlocks(const std::string& path, const std::vector<std::size_t>& sz,
                    const std::vector<std::string>& scalars, const std::string& vector, int components,
                    const double* data)
{
    std::size_t N = 1;
    for (std::size_t n : sz) N *= n;
    const std::string head = vtiHeader(sz, scalars, vector, components);
    Sink f(path, "FileRaw::Save() - Can not open file for output.");
    f.put(head.data(), head.size(), kSaveError);
    std::size_t at = 0;
    for (std::size_t k = 0; k < scalars.size(); ++k, at += N) {
        const uint64_t len = N * sizeof(double);
        f.put(&len, sizeof len, kSaveError);
        f.put(data + at, len, kSaveError);
    }
    const uint64_t len = N * components * sizeof(double);
    f.put(&len, sizeof len, kSaveError);
    f.put(data + at, len, kSaveError);
    const char foot[] = "</AppendedData></VTKFile>";
    f.put(foot, sizeof foot - 1, kSaveError);
    f.close(kSaveError);
}

void writeCheckpoint(const std::string& path, const double* f, std::size_t count)
{
    // prepareRestart (simulator.cpp:335-343): truncate, drop the old sidecar.
    std::remove((path + ".meta").c_str());
    Sink out(path, "Cannot create restart population file.");
    out.put(f, count * sizeof(double), kSaveError);
    out.close(kSaveError);
}

void writeCheckpointMeta(const std::string& path, std::size_t t, std::size_t phases, std::size_t D,
                         std::size_t Q, const std::vector<std::size_t>& sz)
{
    std::ofstream out(path + ".meta", std::ios::trunc);
    out << "DRLAB_OUTGOING_V1\n" << t << ' ' << phases << ' ' << D << ' ' << Q << '\n';
    for (std::size_t n : sz) out << n << ' ';
    out << '\n' << "NEXT_STREAM " << t + 1 << '\n' << "INITIAL_COLLISION_INCLUDED " << t + 1 << '\n'
        << "CONVERGENCE_HISTORY_RESET_ON_LOAD\n";
    if (!out) throw std::runtime_error("Cannot write restart metadata.");
}

void validateCheckpoint(const std::string& path, std::size_t t, std::size_t phases, std::size_t D,
                        std::size_t Q, const std::vector<std::size_t>& sz)
{
    std::ifstream in(path + ".meta");
    std::string format;
    std::size_t st = 0, sp = 0, sd = 0, sq = 0;
    in >> format >> st >> sp >> sd >> sq;
    if (!in || format != "DRLAB_OUTGOING_V1" || st != t || sp != phases || sd != D || sq != Q)
        throw std::runtime_error("Missing or incompatible restart metadata; historical unlabeled checkpoints are not accepted.");
    std::size_t N = 1;
    for (std::size_t n : sz) {
        std::size_t stored = 0;
        in >> stored;
        if (!in || n != stored) throw std::runtime_error("Restart grid dimensions differ.");
        N *= n;
    }
    std::ifstream data(path, std::ios::binary | std::ios::ate);
    const std::size_t expected = N * Q * phases * sizeof(double);
    if (!data || data.tellg() != static_cast<std::streamoff>(expected))
        throw std::runtime_error("Restart population file has an invalid length.");
}

std::vector<double> readCheckpoint(const std::string& path, std::size_t count)
{
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("FileRaw::Load() - Can not open file for input.");
    std::vector<double> v(count);
    const std::size_t got = count ? std::fread(v.data(), sizeof(double), count, f) : 0;
    std::fclose(f);
    if (got != count) throw std::runtime_error("FileRaw::Load() - Failed to read from raw file");
    return v;
}

}  // namespace lbfhost
