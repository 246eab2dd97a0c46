// Test program for tests/test_drivers.py: the std::vector forms of current::Benchmark (gridKernel,
// degridKernel, initC) against the object's own passes on the spectral-line run.  Prints
// "grid_equal <0|1> degrid_equal <0|1> c_equal <0|1>" and exits 0.
#include <cstring>
#include <iostream>
#include <vector>

#include "CurrentBenchmark.h"

int main()
{
    current::Benchmark b;
    b.setRunType(1);
    b.init();
    b.runGrid();
    b.runDegrid();
    b.sync();
    const std::vector<current::Value> grid = b.gridValues(), out = b.outdata();
    const tcv_cur_geometry g = b.geometry();
    int support = 0, os = 0;
    current::Coord wcs = 0;
    std::vector<current::Value> c;
    b.initC(g.uv_cell_size, g.w_size, support, os, wcs, c);
    std::vector<current::Value> grid2(size_t(g.g_size) * g.g_size, current::Value(0.f, 0.f)), out2;
    b.gridKernel(c, grid2, g.g_size);
    b.degridKernel(grid2, g.g_size, c, out2);
    std::vector<current::Value> c_dev(size_t(g.c_len));
    tcv_cur_get_c(b.context(), reinterpret_cast<float*>(c_dev.data()), g.c_len);
    const bool ge = grid2.size() == grid.size() && std::memcmp(grid2.data(), grid.data(), grid.size() * 8) == 0;
    const bool de = out2.size() == out.size() && std::memcmp(out2.data(), out.data(), out.size() * 8) == 0;
    const bool ce = c.size() == c_dev.size() && std::memcmp(c.data(), c_dev.data(), c.size() * 8) == 0;
    std::cout << "grid_equal " << ge << " degrid_equal " << de << " c_equal " << ce << std::endl;
    return 0;
}
