// ref_driver.cc -- drives the reference's own Benchmark class (attic/tConvolveMPI/Benchmark.cc,
// compiled unmodified from the reference tree by oracle/Makefile) to produce golden outputs and
// to time the reference CPU path on this host.
//
// TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline, never the product).
//
// The Benchmark header is a build-time copy of attic/tConvolveMPI/Benchmark.h with the problem
// constants (lines 39-46) substituted per configuration and its private section made public, so
// that this driver can read the grid, the samples and the table, and inject visibilities.
//
// Modes:
//   ref_driver dump <outdir> [vis.bin]
//       init(); optionally replace samples[].data with complex64 values from vis.bin; runGrid();
//       runDegrid(); write u/v/w (f64), iu/iv/coff (i32), C, grid, outdata (complex64) and meta.txt.
//   ref_driver time <threads> <samples_per_thread> <steps> [warmup]
//       tConvolveMT-style replicas (attic/tConvolveMT/tConvolveMT.cc:65-123): one init(), then
//       <threads> replicas, each owning a private grid and the first <samples_per_thread>
//       samples, run the reference gridKernel and then degridKernel concurrently.  Prints one
//       line per step: "step <i> grid_s <t> degrid_s <t> updates <u>".
#include "Benchmark.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

namespace {

template <typename T>
void write_vec(const std::string& path, const std::vector<T>& v)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(T)));
    if (!f) {
        std::cerr << "cannot write " << path << std::endl;
        std::exit(2);
    }
}

int dump(const std::string& outdir, const char* vis_path)
{
    Benchmark b;
    b.init();
    const size_t n = b.samples.size();
    if (vis_path) {
        std::vector<Value> vis(n);
        std::ifstream f(vis_path, std::ios::binary);
        f.read(reinterpret_cast<char*>(vis.data()), std::streamsize(n * sizeof(Value)));
        if (!f) {
            std::cerr << "cannot read " << n << " visibilities from " << vis_path << std::endl;
            return 2;
        }
        for (size_t i = 0; i < n; ++i) b.samples[i].data = vis[i];
    }
    b.runGrid();
    b.runDegrid();

    std::vector<int> iu(n), iv(n), coff(n);
    std::vector<Value> data(n);
    for (size_t i = 0; i < n; ++i) {
        iu[i] = b.samples[i].iu;
        iv[i] = b.samples[i].iv;
        coff[i] = b.samples[i].cOffset;
        data[i] = b.samples[i].data;
    }
    write_vec(outdir + "/u.f64", b.u);
    write_vec(outdir + "/v.f64", b.v);
    write_vec(outdir + "/w.f64", b.w);
    write_vec(outdir + "/iu.i32", iu);
    write_vec(outdir + "/iv.i32", iv);
    write_vec(outdir + "/coff.i32", coff);
    write_vec(outdir + "/data.c64", data);
    write_vec(outdir + "/C.c64", b.C);
    write_vec(outdir + "/grid.c64", b.grid);
    write_vec(outdir + "/outdata.c64", b.outdata);
    std::ofstream meta(outdir + "/meta.txt");
    meta.precision(17);
    meta << "nSamples " << nSamples << "\nnChan " << nChan << "\nwSize " << wSize << "\ngSize "
         << gSize << "\ncellSize " << cellSize << "\nbaseline " << baseline << "\nsupport "
         << b.getSupport() << "\noverSample " << b.overSample << "\nwCellSize " << b.wCellSize
         << "\n";
    return 0;
}

int timing(int threads, int per_thread, int steps, int warmup)
{
    Benchmark main_b;
    main_b.init();
    const int support = main_b.getSupport();
    const int s = 2 * support + 1;
    if (per_thread > int(main_b.samples.size())) per_thread = int(main_b.samples.size());

    std::vector<Benchmark> rep(threads);
    for (int t = 0; t < threads; ++t) {
        rep[t].samples.assign(main_b.samples.begin(), main_b.samples.begin() + per_thread);
        rep[t].outdata.assign(per_thread, Value(0.0f));
        rep[t].grid.assign(size_t(gSize) * gSize, Value(0.0f));
    }
    const double updates = double(per_thread) * double(s) * double(s) * double(threads);
    std::cout << "threads " << threads << " samples_per_thread " << per_thread << " support "
              << support << std::endl;

    for (int step = 0; step < warmup + steps; ++step) {
        std::vector<std::thread> pool;
        auto t0 = std::chrono::steady_clock::now();
        for (int t = 0; t < threads; ++t)
            pool.emplace_back([&, t] { rep[t].gridKernel(support, main_b.C, rep[t].grid, gSize); });
        for (auto& th : pool) th.join();
        auto t1 = std::chrono::steady_clock::now();
        pool.clear();
        for (int t = 0; t < threads; ++t)
            pool.emplace_back(
                [&, t] { rep[t].degridKernel(rep[t].grid, gSize, support, main_b.C, rep[t].outdata); });
        for (auto& th : pool) th.join();
        auto t2 = std::chrono::steady_clock::now();
        if (step >= warmup)
            std::printf("step %d grid_s %.6f degrid_s %.6f updates %.0f\n", step - warmup,
                        std::chrono::duration<double>(t1 - t0).count(),
                        std::chrono::duration<double>(t2 - t1).count(), updates);
        std::fflush(stdout);
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc >= 3 && std::strcmp(argv[1], "dump") == 0)
        return dump(argv[2], argc >= 4 ? argv[3] : nullptr);
    if (argc >= 5 && std::strcmp(argv[1], "time") == 0)
        return timing(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]),
                      argc >= 6 ? std::atoi(argv[5]) : 1);
    std::cerr << "usage: ref_driver dump <outdir> [vis.bin] | time <threads> <per_thread> <steps> [warmup]"
              << std::endl;
    return 1;
}
