// layouts.cuh -- shared-memory index arithmetic of the TMA-staged solver
// kernels (fused red-black sweep, SpMV, restriction).  The kernels call
// these functions, and the host-compiled layout check
// (tests/cpp/layout_check.cpp) enumerates every index they can form for
// every thread and cell and checks it against the boxes' extents, so the
// check follows the code the kernels run.
#pragma once

#if defined(__CUDACC__)
#define LHI_LAYOUT_FN __host__ __device__ __forceinline__ constexpr
#else
#define LHI_LAYOUT_FN inline constexpr
#endif

namespace lhi {
namespace layout {

// ---- fused red-black sweep of one 8 x 8 x 32 tile (x, y, z); boxes of
// kZW values along z, starting 4 cells before the tile (TMA's 16-byte rule)
constexpr int kZW = 40;                 // z extent of the value boxes
constexpr int kMW = 64;                 // z extent of the mask box (starts 16 before)
constexpr int kZBox = 12 * 12 * kZW;    // z grown by two cells in x and y
constexpr int kRBox = 10 * 10 * kZW;    // r, diag, cz grown by one cell
constexpr int kCBox = 11 * 10 * kZW;    // cx (x from x0 - 2) and cy (y from y0 - 2)
constexpr int kMBox = 10 * 10 * kMW;
// neighbour steps inside the z box, and the -x / -y coefficient steps
constexpr int kZStepX = 12 * kZW, kZStepY = kZW;
constexpr int kCXStepX = 10 * kZW, kCYStepY = kZW;

// cell (lx, ly, lz) relative to the tile origin, lx, ly in [-1, 8], lz in [-1, 32]
LHI_LAYOUT_FN int rb_r(int lx, int ly, int lz) { return ((lx + 1) * 10 + (ly + 1)) * kZW + (lz + 4); }
LHI_LAYOUT_FN int rb_z(int lx, int ly, int lz) { return ((lx + 2) * 12 + (ly + 2)) * kZW + (lz + 4); }
LHI_LAYOUT_FN int rb_m(int lx, int ly, int lz) { return ((lx + 1) * 10 + (ly + 1)) * kMW + (lz + 16); }
LHI_LAYOUT_FN int rb_cx(int lx, int ly, int lz) { return ((lx + 2) * 10 + (ly + 1)) * kZW + (lz + 4); }
LHI_LAYOUT_FN int rb_cy(int lx, int ly, int lz) { return ((lx + 1) * 11 + (ly + 2)) * kZW + (lz + 4); }

// colour 0 ((x + y + z) even) on the tile grown by one cell: work item q of
// 10 x 10 rows of 17 cells; colour 1 on the tile: q of 8 x 8 rows of 16
constexpr int kRbColour0Items = 100 * 17, kRbColour1Items = 64 * 16;
LHI_LAYOUT_FN void rb_colour0(int q, int x0, int y0, int z0, int& lx, int& ly, int& lz) {
    const int row = q / 17, k = q - row * 17;
    lx = row / 10 - 1;
    ly = row - (row / 10) * 10 - 1;
    lz = ((x0 + lx + y0 + ly + z0 - 1) & 1) - 1 + 2 * k;
}
LHI_LAYOUT_FN void rb_colour1(int q, int x0, int y0, int z0, int& lx, int& ly, int& lz) {
    const int row = q >> 4, k = q & 15;
    lx = row >> 3;
    ly = row & 7;
    lz = ((x0 + lx + y0 + ly + z0 + 1) & 1) + 2 * k;
}
// the write-out: item q of 64 rows x 8 float4s, its first value in the z box
constexpr int kRbOutItems = 64 * 8;
LHI_LAYOUT_FN int rb_out(int q, int& lx, int& ly, int& c) {
    const int row = q >> 3;
    c = q & 7;
    lx = row >> 3;
    ly = row & 7;
    return rb_z(lx, ly, 4 * c);
}

// ---- SpMV and restriction of one tile: warp wp = x, lane = z, row ly = y;
// p / z box grown by one cell (z from z0 - 4), diag / mask / residual the
// tile, cx from x0 - 1, cy from y0 - 1, cz from z0 - 4
constexpr int kPBox = 10 * 10 * 40, kDBox = 8 * 8 * 32, kCXBox = 9 * 8 * 32, kCYBox = 8 * 9 * 32,
              kCZBox = 8 * 8 * 36;
constexpr int kPStepX = 400, kPStepY = 40;
LHI_LAYOUT_FN int sp_p(int wp, int ly, int lane) { return ((wp + 1) * 10 + (ly + 1)) * 40 + (lane + 4); }
LHI_LAYOUT_FN int sp_c(int wp, int ly, int lane) { return (wp * 8 + ly) * 32 + lane; }  // diag, mask, residual
LHI_LAYOUT_FN int sp_cx(int wp, int ly, int lane) { return sp_c(wp, ly, lane) + 256; }   // own +x face
LHI_LAYOUT_FN int sp_cx_minus(int wp, int ly, int lane) { return sp_c(wp, ly, lane); }
LHI_LAYOUT_FN int sp_cy(int wp, int ly, int lane) { return (wp * 9 + ly + 1) * 32 + lane; }
LHI_LAYOUT_FN int sp_cy_minus(int wp, int ly, int lane) { return (wp * 9 + ly) * 32 + lane; }
LHI_LAYOUT_FN int sp_cz(int wp, int ly, int lane) { return (wp * 8 + ly) * 36 + lane + 4; }
LHI_LAYOUT_FN int sp_cz_minus(int wp, int ly, int lane) { return (wp * 8 + ly) * 36 + lane + 3; }

// restriction: thread t owns coarse cell (i, j, k) of the tile's 4 x 4 x 16;
// child c8 = (a, b, c) in the reference's order, its index in the residual tile
LHI_LAYOUT_FN void rs_coarse(int t, int& i, int& j, int& k) {
    i = t >> 6;
    j = (t >> 4) & 3;
    k = t & 15;
}
LHI_LAYOUT_FN int rs_child(int i, int j, int k, int c8) {
    const int a = (c8 >> 2) & 1, b = (c8 >> 1) & 1, c = c8 & 1;
    return ((2 * i + a) * 8 + (2 * j + b)) * 32 + 2 * k + c;
}

}  // namespace layout
}  // namespace lhi
