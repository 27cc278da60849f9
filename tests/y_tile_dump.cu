// Prints the y-pass column-tile parameters of ibpm.jl_b200/csrc/dst_kernels.cuh
// (the constexpr helpers the kernel itself uses) for every transform length,
// scalar type and plan, one line each:
//   N esize PL TW TP run pad_every col_stride tile_elems off(0..N-2)...
// Host code only: it launches nothing and runs without a GPU.
// tests/test_y_tile_layout.py compiles and runs it.
#include <cstdio>

#include "dst_kernels.cuh"

using namespace ibpm::dstk;

template <int N, class T, int PL>
static void dump() {
    const int n2 = N - 1;
    std::printf("%d %d %d %d %d %d %d %d %d", N, (int)sizeof(T), PL, y_tile_w<N, T, PL>(), ct_tp(N, PL),
                y_scan_run<N, PL>(), y_pad_every<N, T, PL>(), y_col_stride<N, T, PL>(n2),
                y_tile_elems<N, T, PL>(n2));
    for (int j = 0; j < n2; ++j) std::printf(" %d", y_off<N, T, PL>(j));
    std::printf("\n");
}

template <int N>
static void dump_all() {
    dump<N, float, 0>();
    dump<N, float, 1>();
    dump<N, double, 0>();
    dump<N, double, 1>();
}

int main() {
    dump_all<32>();
    dump_all<64>();
    dump_all<128>();
    dump_all<192>();
    dump_all<200>();
    dump_all<256>();
    dump_all<384>();
    dump_all<400>();
    dump_all<512>();
    dump_all<768>();
    dump_all<1024>();
    dump_all<2048>();
    return 0;
}
