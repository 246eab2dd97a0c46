// ref_driver_hogbom.cc -- TEST INFRASTRUCTURE ONLY: runs the reference's own HogbomGolden
// (current/tHogbomCleanOMP/HogbomGolden.cc, compiled unmodified from the reference tree by
// `make ref-hogbom`) on raw float images, as its driver tHogbomCleanOMP.cc:94-121 does.
//
//   ref_driver_hogbom <dirty.img> <psf.img> <model.out> <residual.out>
//
// Images are square raw float32 files (the reference's .img format, tHogbomCleanOMP.cc:43-55);
// the iteration count, gain and threshold are the reference's Parameters.h (1000, 0.1, 1e-5).
#include "HogbomGolden.h"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

static std::vector<float> read_image(const std::string& path)
{
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) {
        std::cerr << "cannot open " << path << std::endl;
        std::exit(1);
    }
    const std::streamsize bytes = f.tellg();
    f.seekg(0);
    std::vector<float> img(size_t(bytes) / sizeof(float));
    f.read(reinterpret_cast<char*>(img.data()), bytes);
    return img;
}

static void write_image(const std::string& path, const std::vector<float>& img)
{
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    f.write(reinterpret_cast<const char*>(img.data()), std::streamsize(img.size() * sizeof(float)));
}

int main(int argc, char** argv)
{
    if (argc != 5) {
        std::cerr << "usage: ref_driver_hogbom <dirty.img> <psf.img> <model.out> <residual.out>" << std::endl;
        return 1;
    }
    const std::vector<float> dirty = read_image(argv[1]);
    const std::vector<float> psf = read_image(argv[2]);
    const size_t dim = size_t(std::sqrt(double(dirty.size())));
    const size_t psf_dim = size_t(std::sqrt(double(psf.size())));
    if (dim * dim != dirty.size() || psf_dim * psf_dim != psf.size()) {
        std::cerr << "images must be square" << std::endl;
        return 1;
    }
    std::vector<float> model(dirty.size(), 0.0f), residual;
    HogbomGolden golden;
    golden.deconvolve(dirty, dim, psf, psf_dim, model, residual);
    write_image(argv[3], model);
    write_image(argv[4], residual);
    return 0;
}
