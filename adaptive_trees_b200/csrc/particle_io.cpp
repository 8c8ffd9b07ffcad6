// particle_io.cpp -- readers for the particle files and dataset manifests the
// reference's tests and benchmarks use (tests/particle_io.hpp;
// benchmarks/drivers/common.hpp:62-175), so the same inputs can feed this
// engine.  Host code only.
//
// Particle files:
//   * text: one particle per row, four numeric columns in the order charge x y
//     z ("cxyz") or x y z charge ("xyzc"), or the word ESC for an escaped
//     particle that keeps its slot; blank rows and rows starting with '#' are
//     skipped; a leading '+' on a number is accepted;
//   * binary ("bin"): x y z as three doubles per particle; a NaN x marks an
//     escaped particle.
// Escaped particles get the escape coordinate (the largest double) on all
// three axes, which the trees treat as outside every box.
// Manifests: rows "dataset <name>", "slots <n>", "box <6 numbers>" and
// "frame <index> <id> <format> <path>"; relative frame paths are taken from
// the manifest's directory.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "adaptive_trees_b200.h"
#include "particle_io.hpp"

namespace aot
{
namespace io
{
constexpr double kEscaped = std::numeric_limits<double>::max();

std::vector<char> slurp(const std::string &path)
{
    std::FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) throw std::runtime_error("cannot open " + path);
    std::fseek(fp, 0, SEEK_END);
    const long size = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    std::vector<char> buf(size > 0 ? size_t(size) + 1 : 1, '\0');
    const size_t got = size > 0 ? std::fread(buf.data(), 1, size_t(size), fp) : 0;
    std::fclose(fp);
    if (size > 0 && got != size_t(size)) throw std::runtime_error("short read on " + path);
    buf[got] = '\0';
    buf.resize(got + 1);
    return buf;
}

// xyz of every particle of a text file; `offset` is the column of x (1 for cxyz, 0 for xyzc)
void readText(const std::string &path, int offset, std::vector<double> &x, std::vector<double> &y,
              std::vector<double> &z)
{
    std::vector<char> buf = slurp(path);
    char *p = buf.data();
    char *end = p + buf.size() - 1;
    size_t line = 0;
    while (p < end)
    {
        char *eol = static_cast<char *>(std::memchr(p, '\n', size_t(end - p)));
        if (!eol) eol = end;
        *eol = '\0';  // numbers never run into the next row
        ++line;
        char *q = p;
        p = eol + 1;
        while (*q && std::isspace(static_cast<unsigned char>(*q))) ++q;
        if (*q == '\0' || *q == '#') continue;
        if (std::strncmp(q, "ESC", 3) == 0)
        {
            q += 3;
            while (*q && std::isspace(static_cast<unsigned char>(*q))) ++q;
            if (*q != '\0' && *q != '#')
                throw std::invalid_argument(path + ":" + std::to_string(line) + ": unexpected text after ESC");
            x.push_back(kEscaped);
            y.push_back(kEscaped);
            z.push_back(kEscaped);
            continue;
        }
        double v[4];
        for (double &c : v)
        {
            while (*q && std::isspace(static_cast<unsigned char>(*q))) ++q;
            if (*q == '+') ++q;
            char *next = q;
            c = std::strtod(q, &next);
            if (next == q || (*next && !std::isspace(static_cast<unsigned char>(*next)) && *next != '#'))
                throw std::invalid_argument(path + ":" + std::to_string(line) + ": expected four numbers or ESC");
            q = next;
        }
        x.push_back(v[offset]);
        y.push_back(v[offset + 1]);
        z.push_back(v[offset + 2]);
    }
}

void readBinary(const std::string &path, std::vector<double> &x, std::vector<double> &y, std::vector<double> &z)
{
    std::vector<char> buf = slurp(path);
    const size_t bytes = buf.size() - 1;
    if (bytes % (3 * sizeof(double))) throw std::invalid_argument("binary frame " + path + " is not xyz doubles");
    const size_t n = bytes / (3 * sizeof(double));
    x.resize(n);
    y.resize(n);
    z.resize(n);
    for (size_t i = 0; i < n; ++i)
    {
        double v[3];
        std::memcpy(v, buf.data() + i * sizeof(v), sizeof(v));
        const bool esc = std::isnan(v[0]);
        x[i] = esc ? kEscaped : v[0];
        y[i] = esc ? kEscaped : v[1];
        z[i] = esc ? kEscaped : v[2];
    }
}

int layoutOf(const std::string &format)
{
    if (format == "cxyz") return AO_LAYOUT_CHARGE_XYZ;
    if (format == "xyzc") return AO_LAYOUT_XYZ_CHARGE;
    if (format == "bin") return AO_LAYOUT_BINARY_XYZ;
    throw std::invalid_argument("unknown frame format " + format);
}

Manifest readManifest(const std::string &path)
{
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open manifest " + path);
    Manifest m;
    const size_t slash = path.find_last_of('/');
    const std::string dir = slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
    std::string line;
    while (std::getline(in, line))
    {
        std::istringstream ss(line);
        std::string tag;
        if (!(ss >> tag) || tag[0] == '#') continue;
        if (tag == "dataset") ss >> m.dataset;
        else if (tag == "slots") ss >> m.slots;
        else if (tag == "box")
        {
            for (double &b : m.box) ss >> b;
        }
        else if (tag == "frame")
        {
            Manifest::Frame f{};
            std::string format;
            ss >> f.index >> f.id >> format;
            f.layout = layoutOf(format);
            std::getline(ss >> std::ws, f.path);
            if (!f.path.empty() && f.path[0] != '/') f.path = dir + f.path;
            m.frames.push_back(f);
        }
    }
    if (m.frames.empty() || m.slots == 0) throw std::invalid_argument("manifest " + path + " lists no slots or frames");
    return m;
}
}  // namespace io
}  // namespace aot
