// Test program for tests/test_dropin.py: the C++ Benchmark class (askap-benchmarks_b200/csrc,
// the mirror of attic/tConvolveMPI/Benchmark.h:55-99) on one problem.  It runs init, runGrid and
// runDegrid, then the std::vector forms initC, gridKernel (into a zeroed grid) and degridKernel (of
// that grid), and writes every result as raw little-endian arrays into the output directory:
//   C.c64 grid.c64 outdata.c64 (the std::vector forms), obj_grid.c64 obj_outdata.c64 (the object's
//   passes) and meta.txt (support, overSample, wCellSize).
// Usage: cpp_attic_check nSamples wSize nChan gSize cellSize outdir
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "Benchmark.h"

namespace {
void write(const std::string& path, const std::vector<Value>& v)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(Value)));
}
}  // namespace

int main(int argc, char* argv[])
{
    if (argc != 7) {
        std::fprintf(stderr, "usage: cpp_attic_check nSamples wSize nChan gSize cellSize outdir\n");
        return 2;
    }
    tcv_config cfg;
    tcv_config_default(&cfg);
    cfg.n_samples = std::atoll(argv[1]);
    cfg.w_size = std::atoi(argv[2]);
    cfg.n_chan = std::atoi(argv[3]);
    cfg.g_size = std::atoi(argv[4]);
    cfg.cell_size = std::atof(argv[5]);
    const std::string dir = argv[6];
    Benchmark b(cfg);
    b.init();
    b.runGrid();
    b.runDegrid();
    b.sync();
    write(dir + "/obj_grid.c64", b.gridValues());
    write(dir + "/obj_outdata.c64", b.outdata());

    // the reference's frequencies (attic/tConvolveMPI/Benchmark.cc:86-90)
    std::vector<Coord> freq(cfg.n_chan);
    for (int i = 0; i < cfg.n_chan; ++i) freq[i] = (1.4e9 - 2.0e5 * Coord(i) / Coord(cfg.n_chan)) / 2.998e8;
    int support = 0, overSample = 0;
    Coord wCellSize = 0;
    std::vector<Value> C;
    b.initC(freq, cfg.cell_size, cfg.w_size, support, overSample, wCellSize, C);
    std::vector<Value> grid(size_t(cfg.g_size) * cfg.g_size, Value(0.f, 0.f));
    b.gridKernel(support, C, grid, cfg.g_size);
    std::vector<Value> out;
    b.degridKernel(grid, cfg.g_size, support, C, out);
    write(dir + "/C.c64", C);
    write(dir + "/grid.c64", grid);
    write(dir + "/outdata.c64", out);
    std::ofstream m(dir + "/meta.txt");
    m << std::setprecision(17) << support << " " << overSample << " " << wCellSize << " " << b.getSupport() << "\n";
    return 0;
}
