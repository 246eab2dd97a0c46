// tConvolve.cc -- benchmark driver on the B200 Benchmark class.
//
// Same flow and rate lines as the reference driver (attic/tConvolveMPI/tConvolveMPI.cc:78-122):
// init, timed runGrid, timed runDegrid (degridding the grid just produced), with
//   griddings = nSamples * nChan * sSize^2 (per process)
// and the "Gridding rate ... (million grid points per second)" lines.  One process drives one GPU
// (the reference's MPI ranks are independent replicas; run one process per GPU for more).
// Options follow attic/tConvolveOMP/tConvolveOMP.cc:416-466 (-n -w -c -f) plus -g (gSize),
// -s (cellSize), -t (table form: c64 r32 cbf16 rbf16 cf16 rf16), -r (timed repeats), -d (device).
#include "Benchmark.h"

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

namespace {
void usage()
{
    std::cout << "usage: tConvolve [-h] [option]\n"
                 "-n num\t number of data samples (default 160000)\n"
                 "-w num\t number of lookup planes in w projection (default 33)\n"
                 "-c num\t number of spectral channels (default 1)\n"
                 "-f val\t reduce the field of view by a factor of val (cellSize *= val)\n"
                 "-g num\t grid size in pixels (default 4096)\n"
                 "-s val\t cell size in wavelengths (default 5.0)\n"
                 "-t form\t table storage: c64 (default) r32 cbf16 rbf16 cf16 rf16\n"
                 "-r num\t timed repeats of each pass (default 1; the rate is per pass)\n"
                 "-d num\t CUDA device (default 0)\n";
}

int ctype_of(const std::string& s)
{
    const char* names[] = {"c64", "r32", "cbf16", "rbf16", "cf16", "rf16"};
    for (int i = 0; i < 6; ++i)
        if (s == names[i]) return i;
    return -1;
}

void report(const char* what, double time, double n_vis, double s_size)
{
    std::cout << "    Number of processes: 1" << std::endl;
    std::cout << "    Time " << time << " (s) " << std::endl;
    std::cout << "    Time per visibility spectral sample " << 1e6 * time / n_vis << " (us) " << std::endl;
    std::cout << "    Time per " << what << 1e9 * time / (n_vis * s_size * s_size) << " (ns) " << std::endl;
}
}  // namespace

int main(int argc, char* argv[])
{
    tcv_config cfg;
    tcv_config_default(&cfg);
    int repeats = 1;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-h") {
            usage();
            return 0;
        }
        if (a.size() != 2 || a[0] != '-' || i + 1 >= argc) {
            usage();
            return 1;
        }
        const char* v = argv[++i];
        switch (a[1]) {
            case 'n': cfg.n_samples = std::atoll(v); break;
            case 'w': cfg.w_size = std::atoi(v); break;
            case 'c': cfg.n_chan = std::atoi(v); break;
            case 'f': cfg.cell_size *= std::atof(v); break;
            case 'g': cfg.g_size = std::atoi(v); break;
            case 's': cfg.cell_size = std::atof(v); break;
            case 't': cfg.c_type = ctype_of(v); break;
            case 'r': repeats = std::atoi(v); break;
            case 'd': cfg.device = std::atoi(v); break;
            default: usage(); return 1;
        }
    }
    if (cfg.c_type < 0 || repeats < 1) {
        usage();
        return 1;
    }
    try {
        Benchmark bmark(cfg);
        bmark.init();
        bmark.sync();
        const double n_vis = double(cfg.n_samples) * cfg.n_chan;
        const double s_size = 2.0 * bmark.getSupport() + 1.0;
        const double griddings = n_vis * s_size * s_size;

        std::cout << "+++++ Forward processing (B200) +++++" << std::endl;
        auto t0 = std::chrono::steady_clock::now();
        for (int r = 0; r < repeats; ++r) bmark.runGrid();
        bmark.sync();
        double time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() / repeats;
        report("gridding   ", time, n_vis, s_size);
        std::cout << "    Gridding rate   " << (griddings / 1000000) / time
                  << " (million grid points per second)" << std::endl;

        std::cout << "+++++ Reverse processing (B200) +++++" << std::endl;
        t0 = std::chrono::steady_clock::now();
        for (int r = 0; r < repeats; ++r) bmark.runDegrid();
        bmark.sync();
        time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() / repeats;
        report("degridding ", time, n_vis, s_size);
        std::cout << "    Degridding rate " << (griddings / 1000000) / time
                  << " (million grid points per second)" << std::endl;
        std::cout << "Done" << std::endl;
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
