// particle_io.hpp -- readers of the reference's particle files and manifests (particle_io.cpp).
#pragma once

#include <string>
#include <vector>

namespace aot
{
namespace io
{
void readText(const std::string &path, int offset, std::vector<double> &x, std::vector<double> &y,
              std::vector<double> &z);
void readBinary(const std::string &path, std::vector<double> &x, std::vector<double> &y, std::vector<double> &z);

struct Manifest
{
    std::string dataset;
    size_t slots = 0;
    double box[6] = {0, 0, 0, 0, 0, 0};
    struct Frame
    {
        int index;
        long long id;
        int layout;
        std::string path;
    };
    std::vector<Frame> frames;
};
Manifest readManifest(const std::string &path);
}  // namespace io
}  // namespace aot
