// tMajor.cc -- tMajorACC's driver (current/tMajorACC/tMajorACC.cc:889-1635) on the tcv_major_* object:
// the program's options (-n samples, -w w-planes, -c channels, -f cell-size factor; plus -g grid size,
// -M major and -m minor cycles, -d device), its set-up, the major cycles, and its timing report
// (device time per stage, per major cycle).
#include <cstdlib>
#include <iostream>
#include <string>

#include "tconvolve.h"

namespace {
void usage()
{
    std::cout << "usage: tMajor [-h] [option]\n"
                 "-n num\t change the number of data samples to num.\n"
                 "-w num\t change the number of lookup planes in w projection to num.\n"
                 "-c num\t change the number of spectral channels to num.\n"
                 "-f val\t reduce the field of view by a factor of val (=> reduce the kernel size).\n"
                 "-g num\t grid size (default 4096); -M num major cycles (5); -m num minor cycles (100); "
                 "-d num device\n";
}

int fail(tcv_major_ctx* m, tcv_status s, const char* what)
{
    std::cerr << "Error: " << what << " failed: " << tcv_status_string(s);
    if (m) std::cerr << " (" << tcv_major_last_error(m) << ")";
    std::cerr << std::endl;
    if (m) tcv_major_destroy(m);
    return 1;
}

void rates(const char* title, double t, double nv, double griddings, const char* what)
{
    std::cout << title << std::endl;
    std::cout << "    Time per major cycle " << t << " (s) " << std::endl;
    std::cout << "    Time per visibility sample " << 1e6 * t / nv << " (us) " << std::endl;
    std::cout << "    Time per " << what << "   " << 1e9 * t / griddings << " (ns) " << std::endl;
}
}  // namespace

int main(int argc, char* argv[])
{
    tcv_major_config cfg;
    tcv_major_config_default(&cfg);
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a.size() != 2 || a[0] != '-' || (a != "-h" && i + 1 >= argc)) {
            usage();
            return 1;
        }
        if (a == "-h") {
            usage();
            return 0;
        }
        const char* v = argv[++i];
        switch (a[1]) {
            case 'n': cfg.n_samples = std::atol(v); break;
            case 'w': cfg.w_size = std::atoi(v); break;
            case 'c': cfg.n_chan = std::atoi(v); break;
            case 'f': cfg.cell_size *= std::atof(v); break;
            case 'g': cfg.g_size = std::atoi(v); break;
            case 'M': cfg.n_major = std::atoi(v); break;
            case 'm': cfg.n_minor = std::atoi(v); break;
            case 'd': cfg.device = std::atoi(v); break;
            default: usage(); return 1;
        }
    }
    std::cout << "nSamples = " << cfg.n_samples << "\nnChan = " << cfg.n_chan << "\nwSize = " << cfg.w_size
              << "\ncellSize = " << cfg.cell_size << std::endl;
    tcv_major_ctx* m = nullptr;
    tcv_status s = tcv_major_create(&cfg, &m);
    if (s != TCV_OK) return fail(nullptr, s, "tcv_major_create");
    if ((s = tcv_major_init(m)) != TCV_OK) return fail(m, s, "tcv_major_init");
    for (int it = 0; it < cfg.n_major; ++it) {
        std::cout << "cycle " << it << std::endl;
        if ((s = tcv_major_run_cycle(m)) != TCV_OK) return fail(m, s, "tcv_major_run_cycle");
    }
    double ms[TCV_MAJOR_STAGES];
    int cycles = 0;
    if ((s = tcv_major_stage_ms(m, ms, &cycles)) != TCV_OK) return fail(m, s, "tcv_major_stage_ms");
    int support = 0;
    int64_t nv = 0;
    tcv_major_info(m, &support, &nv, nullptr, nullptr);
    const double sz = 2.0 * support + 1.0, griddings = double(nv) * sz * sz, n = cycles > 0 ? cycles : 1;
    std::cout << "\n+++++ B200 times +++++\n" << std::endl;
    rates("Gridding PSF", ms[TCV_MAJOR_PSF_GRID] * 1e-3, double(nv), griddings, "gridding");
    std::cout << "    Gridding rate   " << griddings / 1e6 / (ms[TCV_MAJOR_PSF_GRID] * 1e-3)
              << " (million grid points per second)" << std::endl;
    rates("Gridding data", ms[TCV_MAJOR_GRID] * 1e-3 / n, double(nv), griddings, "gridding");
    std::cout << "    Gridding rate   " << griddings / 1e6 / (ms[TCV_MAJOR_GRID] * 1e-3 / n)
              << " (million grid points per second)" << std::endl;
    std::cout << "Inverse FFTs\n    Time per major cycle " << ms[TCV_MAJOR_IFFT] * 1e-3 / n << " (s) " << std::endl;
    const double th = ms[TCV_MAJOR_HOGBOM] * 1e-3 / n;
    std::cout << "Hogbom clean\n    Time per major cycle " << th << " (s) \n    Time per minor cycle "
              << th / cfg.n_minor * 1000 << " (ms)\n    Cleaning rate  " << cfg.n_minor / th
              << " (iterations per second)" << std::endl;
    std::cout << "Forward FFT\n    Time per major cycle " << ms[TCV_MAJOR_FFT] * 1e-3 / n << " (s) " << std::endl;
    rates("Degridding data", ms[TCV_MAJOR_DEGRID] * 1e-3 / n, double(nv), griddings, "degridding");
    std::cout << "    Degridding rate   " << griddings / 1e6 / (ms[TCV_MAJOR_DEGRID] * 1e-3 / n)
              << " (million grid points per second)" << std::endl;
    std::cout << std::endl;
    tcv_major_destroy(m);
    return 0;
}
