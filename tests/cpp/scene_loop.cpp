// The reference's frame loop (main.cpp:48-62, without the GL render) on the
// C++ host surface of include/lhi_liquid.hpp: a 32^3 dam break in the unit
// cube, ROBUST solver keys, 20 steps of PreStep / Step / PostStep.  Prints
// one JSON line; exits non-zero on any failure.
#include <cmath>
#include <cstdio>
#include <vector>

#include "lhi_liquid.hpp"

using namespace lhi_b200;

int main() {
    const int n = 32;
    SolverParameter sp;
    sp.tolerance = Scalar(1e-6);
    sp.toleranceMode = LHI_TOL_RELATIVE;
    sp.cgVariant = LHI_CG_FLEXIBLE;
    sp.updateRegion = LHI_REGION_FLUID;
    sp.smoother = LHI_SMOOTHER_DAMPED_GS;
    sp.smoothingFactor = Scalar(1.0);
    sp.trueResidualEvery = 10;
    sp.maxIterations = 200;
    LiquidParameter lp;
    // mixed precision: FP32 grid and V-cycle, FP64 x and dot products (FP32 x
    // stalls near 1e-5 relative on the true residual)
    LiquidModel<3> model({0, 0, 0}, {1, 1, 1}, {n, n, n}, sp, lp, LHI_PRECISION_MIXED);
    // RectBoundary(0.5, 0.5 - dx, useInside) under an OperatorBoundary::None root
    lhi_boundary_node root{};
    root.kind = LHI_BOUNDARY_NONE;
    root.left = 1;
    root.right = -1;
    lhi_boundary_node walls{};
    walls.kind = LHI_BOUNDARY_RECT;
    walls.use_inside = 1;
    walls.left = walls.right = -1;
    for (int i = 0; i < 3; ++i) {
        walls.center[i] = 0.5;
        walls.half_extent[i] = 0.5 - 1.0 / n;
    }
    model.SetBoundary({root, walls});
    model.ComputeSolidPhi();
    // dam block [0, 0.4) x [0, 0.6) x [0, 1): 2x2x2 particles per cell
    std::vector<Scalar> pos;
    const double dx = 1.0 / n;
    for (int x = 0; x < n; ++x)
        for (int y = 0; y < n; ++y)
            for (int z = 0; z < n; ++z) {
                const double cx = (x + 0.5) * dx, cy = (y + 0.5) * dx, cz = (z + 0.5) * dx;
                if (x < 1 || y < 1 || z < 1 || z > n - 2 || cx >= 0.4 || cy >= 0.6) continue;
                for (int k = 0; k < 8; ++k) {
                    pos.push_back(Scalar(cx + ((k >> 2) & 1 ? 0.25 : -0.25) * dx));
                    pos.push_back(Scalar(cy + ((k >> 1) & 1 ? 0.25 : -0.25) * dx));
                    pos.push_back(Scalar(cz + (k & 1 ? 0.25 : -0.25) * dx));
                }
            }
    model.GetParticleSystem().SetParticles(pos);
    const Scalar dt = Scalar(1.0 / 480.0);
    int iters = 0;
    for (int step = 0; step < 20; ++step) {
        try {
            model.PreStep(dt);
            model.Step(dt);
            model.PostStep(dt);
        } catch (const std::runtime_error& e) {
            std::fprintf(stderr, "step %d: %s (graph: %s)\n", step, e.what(), lhi_solver_graph_error(model.Handle()));
            return 4;
        }
        lhi_solve_stats st{};
        Check(lhi_solver_get_stats(model.Handle(), &st), "lhi_solver_get_stats");
        if (st.status != LHI_OK) {
            std::fprintf(stderr, "step %d: solve status %d\n", step, st.status);
            return 2;
        }
        iters += st.iterations;
    }
    const std::vector<Scalar> p = model.GetParticleSystem().GetPositions();
    double ymin = 1e30, ymax = -1e30;
    for (size_t i = 1; i < p.size(); i += 3) {
        ymin = std::fmin(ymin, p[i]);
        ymax = std::fmax(ymax, p[i]);
    }
    // CorrectVolume, the opt-in step the reference has commented out: the
    // selected particles move, all stay inside the walls
    model.CorrectVolume(dt);
    const std::vector<Scalar> pc = model.GetParticleSystem().GetPositions();
    size_t moved = 0;
    bool inside = true;
    for (size_t i = 0; i < pc.size(); ++i) {
        moved += pc[i] != p[i];
        inside = inside && pc[i] > 0.0f && pc[i] < 1.0f;
    }
    std::printf("{\"particles\": %lld, \"pcg_iterations\": %d, \"ymin\": %.6f, \"ymax\": %.6f, \"cfl\": %.6f, "
                "\"correct_volume_moved\": %zu, \"graph_error\": \"%s\"}\n",
                (long long)model.GetParticleSystem().NumParticles(), iters, ymin, ymax, model.GetCFL(), moved,
                lhi_solver_graph_error(model.Handle()));
    return (ymax < 0.6 && ymin > 0.0 && moved > 0 && inside) ? 0 : 3;
}
