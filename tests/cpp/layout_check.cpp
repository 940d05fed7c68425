// Host check of the shared-memory layouts of the TMA-staged solver kernels:
// every index the kernels form through csrc/layouts.cuh, for every thread,
// work item and tile parity, lies inside its box, and the work items cover
// their cells exactly once.  Built and run by tests/test_cpu_tile_layouts.py.
#include <cstdio>
#include <set>
#include <tuple>

#include "layouts.cuh"

using namespace lhi::layout;

static int failures = 0;
static void check(bool ok, const char* what, int a, int b, int c) {
    if (!ok && failures++ < 20) std::printf("FAIL %s (%d, %d, %d)\n", what, a, b, c);
}
static bool in(int i, int n) { return i >= 0 && i < n; }

// one cell of the fused sweep: every box read rb_eval can make
static void rb_cell(int lx, int ly, int lz) {
    const int r = rb_r(lx, ly, lz), z = rb_z(lx, ly, lz), m = rb_m(lx, ly, lz);
    const int cx = rb_cx(lx, ly, lz), cy = rb_cy(lx, ly, lz);
    check(in(r, kRBox) && in(r - 1, kRBox), "r / diag / cz box", lx, ly, lz);
    check(in(m, kMBox), "mask box", lx, ly, lz);
    check(in(cx, kCBox) && in(cx - kCXStepX, kCBox), "cx box", lx, ly, lz);
    check(in(cy, kCBox) && in(cy - kCYStepY, kCBox), "cy box", lx, ly, lz);
    for (int off : {0, kZStepX, -kZStepX, kZStepY, -kZStepY, 1, -1}) check(in(z + off, kZBox), "z box", lx, ly, lz);
}

int main() {
    // fused sweep, every parity of the tile origin
    for (int x0 : {0, 8}) for (int y0 : {0, 8}) for (int z0 : {0, 32, 64}) {
        std::set<std::tuple<int, int, int>> c0, c1, out;
        for (int q = 0; q < kRbColour0Items; ++q) {
            int lx, ly, lz;
            rb_colour0(q, x0, y0, z0, lx, ly, lz);
            check(lx >= -1 && lx <= 8 && ly >= -1 && ly <= 8 && lz >= -1 && lz <= 32, "colour 0 cell", lx, ly, lz);
            check(((x0 + lx + y0 + ly + z0 + lz) & 1) == 0, "colour 0 parity", lx, ly, lz);
            rb_cell(lx, ly, lz);
            c0.insert({lx, ly, lz});
        }
        int even = 0;
        for (int lx = -1; lx <= 8; ++lx) for (int ly = -1; ly <= 8; ++ly) for (int lz = -1; lz <= 32; ++lz)
            if (((x0 + lx + y0 + ly + z0 + lz) & 1) == 0) {
                ++even;
                check(c0.count({lx, ly, lz}) == 1, "colour 0 covers the grown tile", lx, ly, lz);
            }
        check(int(c0.size()) == kRbColour0Items && even == kRbColour0Items, "colour 0 once each", x0, y0, z0);
        for (int q = 0; q < kRbColour1Items; ++q) {
            int lx, ly, lz;
            rb_colour1(q, x0, y0, z0, lx, ly, lz);
            check(lx >= 0 && lx < 8 && ly >= 0 && ly < 8 && lz >= 0 && lz < 32, "colour 1 cell", lx, ly, lz);
            check(((x0 + lx + y0 + ly + z0 + lz) & 1) == 1, "colour 1 parity", lx, ly, lz);
            rb_cell(lx, ly, lz);
            c1.insert({lx, ly, lz});
        }
        check(int(c1.size()) == kRbColour1Items, "colour 1 covers the tile's odd cells once", x0, y0, z0);
        for (int q = 0; q < kRbOutItems; ++q) {
            int lx, ly, c;
            const int zo = rb_out(q, lx, ly, c);
            check(zo % 4 == 0 && in(zo, kZBox) && in(zo + 3, kZBox), "write-out float4", lx, ly, c);
            for (int j = 0; j < 4; ++j) {
                check(zo + j == rb_z(lx, ly, 4 * c + j), "write-out cell", lx, ly, 4 * c + j);
                out.insert({lx, ly, 4 * c + j});
            }
        }
        check(out.size() == 8u * 8u * 32u, "write-out covers the tile", x0, y0, z0);
    }
    // SpMV and the restriction's residual
    std::set<int> cells;
    for (int wp = 0; wp < 8; ++wp) for (int ly = 0; ly < 8; ++ly) for (int lane = 0; lane < 32; ++lane) {
        const int p = sp_p(wp, ly, lane);
        for (int off : {0, kPStepX, -kPStepX, kPStepY, -kPStepY, 1, -1}) check(in(p + off, kPBox), "p box", wp, ly, lane);
        check(in(sp_c(wp, ly, lane), kDBox), "diag / mask box", wp, ly, lane);
        check(in(sp_cx(wp, ly, lane), kCXBox) && in(sp_cx_minus(wp, ly, lane), kCXBox), "cx box", wp, ly, lane);
        check(in(sp_cy(wp, ly, lane), kCYBox) && in(sp_cy_minus(wp, ly, lane), kCYBox), "cy box", wp, ly, lane);
        check(in(sp_cz(wp, ly, lane), kCZBox) && in(sp_cz_minus(wp, ly, lane), kCZBox), "cz box", wp, ly, lane);
        cells.insert(sp_c(wp, ly, lane));
    }
    check(int(cells.size()) == kDBox, "the tile's cells once each", 0, 0, 0);
    std::set<int> children;
    for (int t = 0; t < 256; ++t) {
        int i, j, k;
        rs_coarse(t, i, j, k);
        for (int c8 = 0; c8 < 8; ++c8) {
            const int f = rs_child(i, j, k, c8);
            check(in(f, kDBox), "restriction child", i, j, k);
            children.insert(f);
        }
    }
    check(int(children.size()) == kDBox, "the coarse cells cover the fine tile once", 0, 0, 0);
    std::printf("%s: %d failures\n", failures ? "FAILED" : "ok", failures);
    return failures ? 1 : 0;
}
