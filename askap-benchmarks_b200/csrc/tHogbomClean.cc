// tHogbomClean.cc -- tHogbomCleanOMP's driver (current/tHogbomCleanOMP/tHogbomCleanOMP.cc:81-124) on
// HogbomB200: reads the dirty and PSF images (raw float32, square; dirty.img and psf.img by default,
// as Parameters.h names them), cleans, writes residual.img and model.img, and prints the
// reference's report lines.  The loop time is the device time of the cleaning.
#include "HogbomB200.h"

#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace {
std::vector<float> readImage(const std::string& filename)
{
    struct stat results;
    if (stat(filename.c_str(), &results) != 0) {
        std::cerr << "Error: Could not stat " << filename << std::endl;
        std::exit(1);
    }
    std::vector<float> image(size_t(results.st_size) / sizeof(float));
    std::ifstream file(filename.c_str(), std::ios::in | std::ios::binary);
    file.read(reinterpret_cast<char*>(image.data()), results.st_size);
    return image;
}

void writeImage(const std::string& filename, const std::vector<float>& image)
{
    std::ofstream file(filename.c_str(), std::ios::out | std::ios::binary | std::ios::trunc);
    file.write(reinterpret_cast<const char*>(image.data()), std::streamsize(image.size() * sizeof(float)));
}

size_t checkSquare(const std::vector<float>& vec)
{
    const size_t size = vec.size();
    const size_t singleDim = size_t(std::sqrt(double(size)));
    if (singleDim * singleDim != size) {
        std::cerr << "Error: Image is not square" << std::endl;
        std::exit(1);
    }
    return singleDim;
}
}  // namespace

int main(int argc, char* argv[])
{
    const std::string dirtyFile = argc > 1 ? argv[1] : "dirty.img";
    const std::string psfFile = argc > 2 ? argv[2] : "psf.img";
    const std::string outDir = argc > 3 ? std::string(argv[3]) + "/" : "";
    std::cout << "Reading dirty image and psf image" << std::endl;
    const std::vector<float> dirty = readImage(dirtyFile);
    const size_t dim = checkSquare(dirty);
    const std::vector<float> psf = readImage(psfFile);
    const size_t psfDim = checkSquare(psf);
    HogbomB200 clean;
    std::cout << "Iterations = " << 1000 << std::endl;
    std::cout << "Image dimensions = " << dim << "x" << dim << std::endl;
    std::vector<float> model(dirty.size(), 0.0f), residual;
    try {
        std::cout << "+++++ Forward processing (B200) +++++" << std::endl;
        clean.deconvolve(dirty, dim, psf, psfDim, model, residual);
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }
    const double time = clean.deviceSeconds();
    const int n = clean.iterations() > 0 ? clean.iterations() : 1;
    std::cout << "    Time " << time << " (s) " << std::endl;
    std::cout << "    Time per cycle " << time / n * 1000 << " (ms)" << std::endl;
    std::cout << "    Cleaning rate  " << n / time << " (iterations per second)" << std::endl;
    std::cout << "Done" << std::endl;
    writeImage(outDir + "residual.img", residual);
    writeImage(outDir + "model.img", model);
    return 0;
}
