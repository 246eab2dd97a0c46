// ref_driver_current.cc -- drives the reference's own current/tConvolveMPI Benchmark class
// (current/tConvolveMPI/Benchmark.cc, compiled unmodified from the reference tree by
// oracle/Makefile) to produce golden outputs of the variable-support path and to time it.
//
// TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline, never the product).
//
// The header is a build-time copy of current/tConvolveMPI/Benchmark.h with its private section
// made public, so that this driver can read the grid, the offsets and the table.
//
// Modes:
//   ref_driver_current dump <run_type> <sort> <outdir> [earlier run types...]
//       The earlier run types are init()ed first on the same object, as tConvolveMPI's loop does
//       (current/tConvolveMPI/tConvolveMPI.cc:85-92), so the generator state carries over.
//       Then init(); runGrid(); runDegrid(); and u/v/w (f64), iu/iv/wplane/coff/ssize/coff0
//       (i32), C, grid, outdata (complex64) and meta.txt are written.
//   ref_driver_current time <run_type> <threads> <steps> [max_samples]
//       One init(), then <threads> replicas (private grid, the first max_samples samples each)
//       run gridKernel then degridKernel concurrently per step; prints
//       "step <i> grid_s <t> degrid_s <t> pixels <n>".
#include "Benchmark.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
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

int dump(int run_type, int sort, const std::string& out, const std::vector<int>& earlier)
{
    Benchmark b;
    b.setMPIrank(1);  // not rank 0: the reference prints only on rank 0
    b.setSort(sort);
    for (int r : earlier) {
        b.setRunType(r);
        b.init();
    }
    b.setRunType(run_type);
    b.init();
    b.runGrid();
    b.runDegrid();
    write_vec(out + "/u.bin", b.u);
    write_vec(out + "/v.bin", b.v);
    write_vec(out + "/w.bin", b.w);
    write_vec(out + "/iu.bin", b.iu);
    write_vec(out + "/iv.bin", b.iv);
    write_vec(out + "/wplane.bin", b.wPlane);
    write_vec(out + "/coff.bin", b.cOffset);
    write_vec(out + "/ssize.bin", b.sSize);
    write_vec(out + "/coff0.bin", b.cOffset0);
    write_vec(out + "/C.bin", b.C);
    write_vec(out + "/grid.bin", b.grid1);
    write_vec(out + "/outdata.bin", b.outdata1);
    std::ofstream m(out + "/meta.txt");
    m.precision(17);
    m << "nSamples " << b.nSamples << "\nwSize " << b.wSize << "\ngSize " << b.gSize << "\noverSample "
      << b.overSample << "\nsupport " << b.m_support << "\nwCellSize " << b.wCellSize << "\nuvCellSize "
      << b.uvCellSize << "\nnPixelsGridded " << b.nPixelsGridded() << "\nnext " << b.next << "\n";
    return 0;
}

int time_mode(int run_type, int threads, int steps, long max_samples)
{
    Benchmark b;
    b.setMPIrank(1);
    b.setSort(0);
    b.setRunType(run_type);
    b.init();
    const long n = std::min<long>(long(b.data.size()), max_samples > 0 ? max_samples : long(b.data.size()));
    b.data.resize(size_t(n));
    b.outdata1.resize(size_t(n));
    long pixels = 0;
    for (long d = 0; d < n; ++d) pixels += long(b.sSize[b.wPlane[d]]) * b.sSize[b.wPlane[d]];
    std::vector<Benchmark> reps(size_t(threads), b);
    for (int s = 0; s < steps; ++s) {
        auto t0 = std::chrono::steady_clock::now();
        std::vector<std::thread> th;
        for (auto& r : reps) th.emplace_back([&r] { r.runGrid(); });
        for (auto& t : th) t.join();
        auto t1 = std::chrono::steady_clock::now();
        th.clear();
        for (auto& r : reps) th.emplace_back([&r] { r.runDegrid(); });
        for (auto& t : th) t.join();
        auto t2 = std::chrono::steady_clock::now();
        std::printf("step %d grid_s %.6f degrid_s %.6f pixels %ld\n", s,
                    std::chrono::duration<double>(t1 - t0).count(), std::chrono::duration<double>(t2 - t1).count(),
                    pixels * threads);
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc >= 5 && std::string(argv[1]) == "dump") {
        std::vector<int> earlier;
        for (int i = 5; i < argc; ++i) earlier.push_back(std::atoi(argv[i]));
        return dump(std::atoi(argv[2]), std::atoi(argv[3]), argv[4], earlier);
    }
    if (argc >= 5 && std::string(argv[1]) == "time")
        return time_mode(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]), argc > 5 ? std::atol(argv[5]) : 0);
    std::cerr << "usage: ref_driver_current dump <run_type> <sort> <outdir> [earlier...] | "
                 "time <run_type> <threads> <steps> [max_samples]" << std::endl;
    return 1;
}
