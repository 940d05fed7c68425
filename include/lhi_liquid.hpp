// lhi_liquid.hpp -- C++ host surface of the B200 liquid step, over the C-ABI
// of lhi.h.  Header-only; link with -llhi.
//
// It keeps the reference's class and method names so the reference's Scene
// loop (main.cpp:50-53: PreStep, Step, PostStep, GetCFL) runs unchanged on
// top of it:
//   lhi_b200::LiquidModel<3>    LiquidModel.h:14-61
//   lhi_b200::CGSolver<3>       PressureSolver.h:89-118
//   lhi_b200::ParticleSystem<3> ParticleSystem.h:24-60
//   lhi_b200::SolverParameter   SceneParameter.h:10-45 (+ the solver keys of lhi.h)
//   lhi_b200::LiquidParameter   SceneParameter.h:48-66
// Boundaries are the BaseBoundary<3> tree as lhi_boundary_node arrays
// (Boundary.h:6-96).  Every failing call throws std::runtime_error carrying
// lhi_last_error(), as the reference throws on its own errors
// (PressureSolver.cpp:769, ParticleSystem.cpp:73).  Scalars cross as float:
// the reference's Scalar (Definition.h:33).
#ifndef LHI_LIQUID_HPP_
#define LHI_LIQUID_HPP_

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "lhi.h"

namespace lhi_b200 {

using Scalar = float;
using Vector3 = std::array<Scalar, 3>;

inline void Check(int rc, const char* what) {
    if (rc != LHI_OK) throw std::runtime_error(std::string(what) + " failed: " + lhi_last_error());
}

// SolverParameter<3> (SceneParameter.h:10-45) plus the keys lhi.h adds.
struct SolverParameter {
    int maxIterations = 100;
    Scalar tolerance = Scalar(1e-5);
    int preconditionerType = LHI_PRECOND_MULTIGRID;  // None, Jacobi, Multigrid (+ Learned)
    int numLevel = 4;
    int numPreSmooth = 5;
    int numPostSmooth = 5;
    int numFinalSmooth = 20;
    Scalar smoothingFactor = Scalar(0.5);
    int toleranceMode = LHI_TOL_ABSOLUTE;
    int cgVariant = LHI_CG_REFERENCE;
    int trueResidualEvery = 0;
    int updateRegion = LHI_REGION_INTERIOR;
    int smoother = LHI_SMOOTHER_REFERENCE;

    lhi_solver_params ToAbi() const {
        lhi_solver_params p{};
        p.max_iterations = maxIterations;
        p.preconditioner = preconditionerType;
        p.tolerance = tolerance;
        p.num_level = numLevel;
        p.num_pre_smooth = numPreSmooth;
        p.num_post_smooth = numPostSmooth;
        p.num_final_smooth = numFinalSmooth;
        p.smoothing_factor = smoothingFactor;
        p.tolerance_mode = toleranceMode;
        p.cg_variant = cgVariant;
        p.true_residual_every = trueResidualEvery;
        p.update_region = updateRegion;
        p.smoother = smoother;
        return p;
    }
};

// LiquidParameter<3> (SceneParameter.h:48-66) and the SceneParameter<3>
// gravity the liquid model reads.
struct LiquidParameter {
    int numParticles = 0;
    Scalar viscosity = Scalar(0.001);  // parsed, unused by the liquid step
    Scalar density = Scalar(1000);
    Scalar surfaceTension = Scalar(0.0728);  // parsed, unused
    int correctCycle = 8;
    Scalar gravity = Scalar(-9.81);
};

template <int DIM> class ParticleSystem;
template <int DIM> class CGSolver;
template <int DIM> class LiquidModel;

// ParticleSystem<3>: positions / velocities in the caller's order.
template <> class ParticleSystem<3> {
public:
    explicit ParticleSystem(lhi_liquid* h) : h_(h) {}
    std::int64_t NumParticles() const {
        std::int64_t n = 0;
        Check(lhi_liquid_num_particles(h_, &n), "lhi_liquid_num_particles");
        return n;
    }
    // positions (and optionally velocities / affine matrices) as flat xyz triples
    void SetParticles(const std::vector<Scalar>& pos, const std::vector<Scalar>* vel = nullptr,
                      const std::vector<Scalar>* affine = nullptr) {
        if (pos.size() % 3) throw std::runtime_error("SetParticles: positions must be xyz triples");
        const std::int64_t n = std::int64_t(pos.size() / 3);
        if ((vel && vel->size() != pos.size()) || (affine && affine->size() != size_t(n) * 9))
            throw std::runtime_error("SetParticles: size mismatch");
        Check(lhi_liquid_set_particles(h_, n, pos.data(), vel ? vel->data() : nullptr,
                                       affine ? affine->data() : nullptr),
              "lhi_liquid_set_particles");
    }
    std::vector<Scalar> GetPositions() const { return Get(0); }
    std::vector<Scalar> GetVelocities() const { return Get(1); }
    // ParticleSystem<3>::SpawnParticles (ParticleSystem.cpp:45-64): lattice of
    // spacing 0.5 * radius over [minCoord, maxCoord), at most maxCount.
    void SpawnParticles(const Vector3& minCoord, const Vector3& maxCoord, Scalar radius, std::int64_t maxCount) {
        const double mn[3] = {minCoord[0], minCoord[1], minCoord[2]};
        const double mx[3] = {maxCoord[0], maxCoord[1], maxCoord[2]};
        std::int64_t n = 0;
        Check(lhi_scene_spawn_lattice(mn, mx, radius, maxCount, LHI_PRECISION_FP32, &n, nullptr),
              "lhi_scene_spawn_lattice");
        std::vector<Scalar> pos(size_t(n) * 3);
        Check(lhi_scene_spawn_lattice(mn, mx, radius, maxCount, LHI_PRECISION_FP32, &n, pos.data()),
              "lhi_scene_spawn_lattice");
        SetParticles(pos);
    }

private:
    std::vector<Scalar> Get(int which) const {
        const std::int64_t n = NumParticles();
        std::vector<Scalar> out(size_t(n) * 3);
        Check(lhi_liquid_get_particles(h_, which == 0 ? out.data() : nullptr, which == 1 ? out.data() : nullptr,
                                       nullptr),
              "lhi_liquid_get_particles");
        return out;
    }
    lhi_liquid* h_;
};

// CGSolver<3> (PressureSolver.h:89-118)
template <> class CGSolver<3> {
public:
    explicit CGSolver(lhi_liquid* h) : h_(h) {}
    void Init() { Check(lhi_solver_init(h_), "lhi_solver_init"); }
    void BuildRHS() { Check(lhi_solver_build_rhs(h_), "lhi_solver_build_rhs"); }
    void BuildLHS(Scalar liquidDensity, Scalar dt) { Check(lhi_solver_build_lhs(h_, liquidDensity, dt), "lhi_solver_build_lhs"); }
    void ApplyPreconditioner() { Check(lhi_solver_apply_preconditioner(h_), "lhi_solver_apply_preconditioner"); }
    // Solve (PressureSolver.cpp:839-934); returns the statistics, throws on NaN
    // and on a CUDA error; stopping at maxIterations is reported in status.
    lhi_solve_stats Solve(Scalar liquidDensity, Scalar dt) {
        lhi_solve_stats st{};
        const int rc = lhi_solver_solve(h_, liquidDensity, dt, &st);
        if (rc != LHI_OK && rc != LHI_E_NOT_CONVERGED) Check(rc, "lhi_solver_solve");
        return st;
    }
    // A x on one level (host buffers of that level's cell count)
    std::vector<Scalar> GetAx(const std::vector<Scalar>& x, int level = 0) {
        std::vector<Scalar> out(x.size());
        Check(lhi_solver_get_ax(h_, level, x.data(), out.data()), "lhi_solver_get_ax");
        return out;
    }

private:
    lhi_liquid* h_;
};

// LiquidModel<3> (LiquidModel.h:14-61) on the GPU.  SetBoundary keeps a copy
// of the boundary tree (the reference keeps a pointer, LiquidModel.h:68);
// ComputeSolidPhi evaluates it on the device.
template <> class LiquidModel<3> {
public:
    LiquidModel(const Vector3& minCoord, const Vector3& maxCoord, const std::array<int, 3>& gridDimension,
                const SolverParameter& solver, const LiquidParameter& liquid, int precision = LHI_PRECISION_FP32)
        : liquid_(liquid),
          minCoord_(minCoord),
          maxCoord_(maxCoord),
          h_(Create(minCoord, maxCoord, gridDimension, solver, liquid, precision)),
          ps_(h_),
          solver_(h_) {}
    ~LiquidModel() { lhi_liquid_destroy(h_); }
    LiquidModel(const LiquidModel&) = delete;
    LiquidModel& operator=(const LiquidModel&) = delete;

    // LiquidModel<3>::Init (LiquidModel.cpp:507-512): solid SDF, then the
    // lattice over the middle 40% of the domain (radius 2 dx), capped at
    // numParticles.
    void Init() {
        ComputeSolidPhi();
        double dx[3];
        Check(lhi_liquid_get_dx(h_, dx), "lhi_liquid_get_dx");
        Vector3 lo, hi;
        for (int i = 0; i < 3; ++i) {
            const Scalar off = Scalar(0.3) * (maxCoord_[i] - minCoord_[i]);
            lo[i] = minCoord_[i] + off;
            hi[i] = maxCoord_[i] - off;
        }
        ps_.SpawnParticles(lo, hi, Scalar(2) * Scalar(dx[0]), liquid_.numParticles);
    }
    void PreStep(Scalar dt) { Check(lhi_liquid_pre_step(h_, dt), "lhi_liquid_pre_step"); }
    void Step(Scalar dt) { Check(lhi_liquid_step(h_, dt), "lhi_liquid_step"); }
    void PostStep(Scalar dt) { Check(lhi_liquid_post_step(h_, dt), "lhi_liquid_post_step"); }

    void ComputeLiquidPhi() { Check(lhi_liquid_compute_liquid_phi(h_), "lhi_liquid_compute_liquid_phi"); }
    void ComputeSolidPhi() {
        if (boundary_.empty()) throw std::runtime_error("ComputeSolidPhi: no boundary set");
        Check(lhi_liquid_set_boundary(h_, boundary_.data(), std::int32_t(boundary_.size()), root_),
              "lhi_liquid_set_boundary");
    }
    void Particle2Grid() { Check(lhi_liquid_particle_to_grid(h_), "lhi_liquid_particle_to_grid"); }
    void Grid2Particle() { Check(lhi_liquid_grid_to_particle(h_), "lhi_liquid_grid_to_particle"); }
    void Projection(Scalar dt) { SolvePressure(dt); }
    void SolvePressure(Scalar dt) { Check(lhi_liquid_projection(h_, dt), "lhi_liquid_projection"); }
    void ApplyGravity(Scalar dt) { Check(lhi_liquid_apply_gravity(h_, dt), "lhi_liquid_apply_gravity"); }
    void AdvectParticle(Scalar dt) { Check(lhi_liquid_advect_particles(h_, dt), "lhi_liquid_advect_particles"); }
    void Extrapolate() { Check(lhi_liquid_extrapolate(h_), "lhi_liquid_extrapolate"); }
    // disabled in the reference's 3D step (LiquidModel.cpp:527)
    void CorrectVolume(Scalar) { throw std::runtime_error("CorrectVolume is disabled in the 3D liquid step"); }
    Scalar ComputeDivergence() const {
        double mean = 0, mx = 0;
        Check(lhi_liquid_compute_divergence(h_, &mean, &mx), "lhi_liquid_compute_divergence");
        return Scalar(mean);
    }
    Scalar GetCFL() const {
        double dt = 0;
        Check(lhi_liquid_get_cfl(h_, &dt), "lhi_liquid_get_cfl");
        return Scalar(dt);
    }
    void SetBoundary(std::vector<lhi_boundary_node> nodes, int root = 0) {
        boundary_ = std::move(nodes);
        root_ = root;
    }
    ParticleSystem<3>& GetParticleSystem() { return ps_; }
    CGSolver<3>& GetSolver() { return solver_; }
    lhi_liquid* Handle() const { return h_; }

private:
    static lhi_liquid* Create(const Vector3& minCoord, const Vector3& maxCoord, const std::array<int, 3>& dim,
                              const SolverParameter& solver, const LiquidParameter& liquid, int precision) {
        lhi_grid_desc g{};
        for (int i = 0; i < 3; ++i) {
            g.dim[i] = dim[i];
            g.min_coord[i] = minCoord[i];
            g.max_coord[i] = maxCoord[i];
        }
        const lhi_solver_params sp = solver.ToAbi();
        lhi_liquid_params lp{};
        lp.density = liquid.density;
        lp.gravity = liquid.gravity;
        lhi_liquid* h = nullptr;
        Check(lhi_liquid_create(&g, &sp, &lp, precision, &h), "lhi_liquid_create");
        return h;
    }

    LiquidParameter liquid_;
    Vector3 minCoord_, maxCoord_;
    lhi_liquid* h_ = nullptr;
    ParticleSystem<3> ps_;
    CGSolver<3> solver_;
    std::vector<lhi_boundary_node> boundary_;
    int root_ = 0;
};

}  // namespace lhi_b200

#endif  // LHI_LIQUID_HPP_
