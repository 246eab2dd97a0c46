// tConvolveCurrent.cc -- current/tConvolveMPI's driver (current/tConvolveMPI/tConvolveMPI.cc:61-186)
// on current::Benchmark: the continuum run then the spectral-line run on one object, runGrid and
// runDegrid each timed (with a device synchronisation before the clock stops), and the
// reference's report lines.  One process drives one GPU.  Options beyond the reference:
// -t picks the plan with tcv_cur_tune first (untimed set-up), -d the CUDA device.
#include "CurrentBenchmark.h"

#include <chrono>
#include <cstdlib>
#include <iostream>
#include <string>

int main(int argc, char* argv[])
{
    bool tune = false;
    int device = 0;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-t") {
            tune = true;
        } else if (a == "-d" && i + 1 < argc) {
            device = std::atoi(argv[++i]);
        } else {
            std::cout << "usage: tConvolveCurrent [-t] [-d device]" << std::endl;
            return 1;
        }
    }
    try {
        current::Benchmark bmark(device);
        bmark.setSort(0);
        const std::vector<float> rates = bmark.requiredRate();
        (void)rates;
        for (int run = 0; run < 2; ++run) {
            bmark.setMPIrank(0);
            bmark.setRunType(run);
            std::cout << "+++++ Test " << bmark.getRunType() << " +++++" << std::endl;
            bmark.init();
            if (tune) bmark.tune();
            const double ngridvis = double(bmark.nVisibilitiesGridded());
            const double ngridpix = double(bmark.nPixelsGridded());
            const double tgridpix = ngridpix;
            bmark.sync();
            auto t0 = std::chrono::steady_clock::now();
            bmark.runGrid();
            bmark.sync();
            double time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::cout << "  Forward processing" << std::endl;
            std::cout << "    Number of processes: 1" << std::endl;
            std::cout << "    Time " << time << " (s) " << std::endl;
            std::cout << "    Time per visibility spectral sample " << 1e6 * time / ngridvis << " (us) " << std::endl;
            std::cout << "    Time per gridding   " << 1e9 * time / ngridpix << " (ns) " << std::endl;
            std::cout << "    Gridding rate (per process)   " << (ngridvis / 1e6) / time << " (Mvis/sec)" << std::endl;
            std::cout << "    Gridding rate (per process)   " << (ngridpix / 1e6) / time << " (Mpix/sec)" << std::endl;
            std::cout << "    Gridding rate (total)      " << (tgridpix / 1e6) / time << " (Mpix/sec)" << std::endl;
            std::cout << "    " << (run == 0 ? "Continuum" : "Spectral") << " gridding performance (per process):   "
                      << (ngridpix / 1e6) / time << " (Mpix/sec)" << std::endl;
            t0 = std::chrono::steady_clock::now();
            bmark.runDegrid();
            bmark.sync();
            time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::cout << "  Reverse processing" << std::endl;
            std::cout << "    Number of processes: 1" << std::endl;
            std::cout << "    Time " << time << " (s) " << std::endl;
            std::cout << "    Time per visibility spectral sample " << 1e6 * time / ngridvis << " (us) " << std::endl;
            std::cout << "    Time per degridding " << 1e9 * time / ngridpix << " (ns) " << std::endl;
            std::cout << "    Degridding rate (per node) " << (ngridvis / 1e6) / time << " (Mvis/sec)" << std::endl;
            std::cout << "    Degridding rate (per node) " << (ngridpix / 1e6) / time << " (Mpix/sec)" << std::endl;
            std::cout << "    Degridding rate (total)    " << (tgridpix / 1e6) / time << " (Mpix/sec)" << std::endl;
            std::cout << "    " << (run == 0 ? "Continuum" : "Spectral")
                      << " degridding performance (per process):   " << (ngridpix / 1e6) / time << " (Mpix/sec)"
                      << std::endl;
            std::cout << "Done" << std::endl;
        }
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
