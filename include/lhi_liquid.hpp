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
// LiquidModel<3> is built either from explicit grid / solver / liquid
// parameters or, like the reference (LiquidModel.cpp:480-486), from the
// reference's own Scene<3>: any object with its getters (GetMinCoord,
// GetMaxCoord, GetGridDimension, GetSolverParameter, GetLiquidParameter,
// GetGravity).  Boundaries are either the reference's BaseBoundary<3> objects
// (SetBoundary(BaseBoundary<3>*), evaluated on the host node by node as
// ComputeSolidPhi does, LiquidModel.cpp:563-572) or the same tree as
// lhi_boundary_node arrays (Boundary.h:6-96), evaluated on the device.
// Every failing call throws std::runtime_error carrying lhi_last_error(), as
// the reference throws on its own errors (PressureSolver.cpp:769,
// ParticleSystem.cpp:73).  Host buffers are float, the reference's Scalar
// (Definition.h:33): FP32 and mixed-precision handles.
#ifndef LHI_LIQUID_HPP_
#define LHI_LIQUID_HPP_

#include <array>
#include <cstdint>
#include <functional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
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
    bool correctVolume = false;  // Step ends with CorrectVolume (off, as in the reference's Step)
};

template <int DIM> class ParticleSystem;
template <int DIM> class CGSolver;
template <int DIM> class LiquidModel;

namespace detail {
// the argument type of a boundary's Compute(const VectorX<3>&) const
template <class M> struct ComputeArg;
template <class R, class C, class A> struct ComputeArg<R (C::*)(A) const> {
    using type = typename std::decay<A>::type;
};
}  // namespace detail

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
    std::vector<Scalar> GetAffineMatrices() const { return Get(2); }
    // ParticleSystem<3>::Resize (ParticleSystem.cpp:11-21): keeps the first
    // min(n, size) particles; new ones start at rest at the origin.
    void Resize(std::int64_t size) {
        if (size < 0) throw std::runtime_error("Resize: negative size");
        std::vector<Scalar> pos = Get(0), vel = Get(1), aff = Get(2);
        pos.resize(size_t(size) * 3, Scalar(0));
        vel.resize(size_t(size) * 3, Scalar(0));
        aff.resize(size_t(size) * 9, Scalar(0));
        SetParticles(pos, &vel, &aff);
    }
    // ParticleSystem<3>::LoadFromLine (ParticleSystem.cpp:88-103): positions
    // from one trajectory line, read as the reference reads it -- the first
    // token is skipped, and a missing token leaves that coordinate as it was.
    void LoadFromLine(const std::string& line) {
        std::vector<Scalar> pos = Get(0), vel = Get(1), aff = Get(2);
        std::istringstream ss(line);
        std::string token;
        std::getline(ss, token, ',');
        for (size_t i = 0; i < pos.size(); ++i)
            if (std::getline(ss, token, ',')) pos[i] = std::stof(token);
        SetParticles(pos, &vel, &aff);
    }
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
        if (which == 2) out.resize(size_t(n) * 9);
        if (n == 0) return out;
        Check(lhi_liquid_get_particles(h_, which == 0 ? out.data() : nullptr, which == 1 ? out.data() : nullptr,
                                       which == 2 ? out.data() : nullptr),
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

// LiquidModel<3> (LiquidModel.h:14-61) on the GPU.  SetBoundary(nodes) keeps a
// copy of a boundary tree, which ComputeSolidPhi evaluates on the device;
// SetBoundary(BaseBoundary<3>*) keeps the pointer, as the reference does
// (LiquidModel.h:57,68), and ComputeSolidPhi evaluates it on the host.
template <> class LiquidModel<3> {
public:
    // LiquidModel<3>::LiquidModel(const Scene<3>&) (LiquidModel.cpp:480-486):
    // grid from the scene's min / max coordinates and dimension, solver from
    // its SolverParameter (the reference's solver semantics), liquid from its
    // LiquidParameter and gravity.  SceneT is the reference's Scene<3> or
    // anything with the same getters.
    template <class SceneT, class = decltype(std::declval<const SceneT&>().GetSolverParameter())>
    explicit LiquidModel(const SceneT& scene, int precision = LHI_PRECISION_FP32)
        : LiquidModel(Vec3(scene.GetMinCoord()), Vec3(scene.GetMaxCoord()), Dim3(scene.GetGridDimension()),
                      SolverOf(scene.GetSolverParameter()), LiquidOf(scene), precision) {}

    LiquidModel(const Vector3& minCoord, const Vector3& maxCoord, const std::array<int, 3>& gridDimension,
                const SolverParameter& solver, const LiquidParameter& liquid, int precision = LHI_PRECISION_FP32)
        : liquid_(liquid),
          minCoord_(minCoord),
          maxCoord_(maxCoord),
          dim_(gridDimension),
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
    // LiquidModel<3>::ComputeSolidPhi (LiquidModel.cpp:563-611): nothing to do
    // without a boundary, as in the reference.
    void ComputeSolidPhi() {
        if (host_boundary_) {
            double dx[3];
            Check(lhi_liquid_get_dx(h_, dx), "lhi_liquid_get_dx");
            const Scalar h[3] = {Scalar(dx[0]), Scalar(dx[1]), Scalar(dx[2])};
            std::vector<Scalar> phi(size_t(dim_[0] + 1) * size_t(dim_[1] + 1) * size_t(dim_[2] + 1));
            size_t k = 0;
            for (int xi = 0; xi < dim_[0] + 1; ++xi)
                for (int yi = 0; yi < dim_[1] + 1; ++yi)
                    for (int zi = 0; zi < dim_[2] + 1; ++zi) {
                        // Vector3(xi, yi, zi).cwiseProduct(dx) + minCoord
                        const Scalar px = Scalar(xi) * h[0], py = Scalar(yi) * h[1], pz = Scalar(zi) * h[2];
                        phi[k++] = host_boundary_(px + minCoord_[0], py + minCoord_[1], pz + minCoord_[2]);
                    }
            Check(lhi_liquid_set_solid_phi(h_, phi.data()), "lhi_liquid_set_solid_phi");
            return;
        }
        if (boundary_.empty()) return;
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
    // LiquidModel<3>::CorrectVolume (LiquidModel.cpp:1086-1132); the reference's
    // Step has the call commented out (LiquidModel.cpp:527), so it runs only
    // when called (or with LiquidParameter::correctVolume set)
    void CorrectVolume(Scalar dt) { Check(lhi_liquid_correct_volume(h_, dt), "lhi_liquid_correct_volume"); }
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
        host_boundary_ = nullptr;
    }
    // LiquidModel<3>::SetBoundary(BaseBoundary<3>*) (LiquidModel.h:57): a
    // non-owning pointer to the reference's boundary object (or any type with
    // Scalar Compute(const Vector&) const); NULL clears it.
    template <class B, class = decltype(&B::Compute)> void SetBoundary(B* boundary) {
        boundary_.clear();
        if (!boundary) {
            host_boundary_ = nullptr;
            return;
        }
        using V = typename detail::ComputeArg<decltype(&B::Compute)>::type;
        host_boundary_ = [boundary](Scalar x, Scalar y, Scalar z) { return Scalar(boundary->Compute(V(x, y, z))); };
    }
    // LiquidModel<3>::Render (LiquidModel.cpp:1136-1160) draws the particles
    // with OpenGL; there is no display here, so this is a no-op.
    void Render() const {}
    ParticleSystem<3>& GetParticleSystem() { return ps_; }
    CGSolver<3>& GetSolver() { return solver_; }
    lhi_liquid* Handle() const { return h_; }

private:
    template <class V> static Vector3 Vec3(const V& v) { return {Scalar(v[0]), Scalar(v[1]), Scalar(v[2])}; }
    template <class V> static std::array<int, 3> Dim3(const V& v) { return {int(v[0]), int(v[1]), int(v[2])}; }
    // SolverParameter<3> (SceneParameter.h:10-45): the reference's keys; the
    // solver keys lhi.h adds keep their defaults (the reference's semantics).
    template <class P> static SolverParameter SolverOf(const P& s) {
        SolverParameter o;
        o.maxIterations = int(s.maxIterations);
        o.tolerance = Scalar(s.tolerance);
        o.preconditionerType = int(s.preconditionerType);  // PrecondType::None, Jacobi, Multigrid = 0, 1, 2
        o.numLevel = int(s.numLevel);
        o.numPreSmooth = int(s.numPreSmooth);
        o.numPostSmooth = int(s.numPostSmooth);
        o.numFinalSmooth = int(s.numFinalSmooth);
        o.smoothingFactor = Scalar(s.smoothingFactor);
        return o;
    }
    template <class SceneT> static LiquidParameter LiquidOf(const SceneT& scene) {
        const auto& l = scene.GetLiquidParameter();
        LiquidParameter o;
        o.numParticles = int(l.numParticles);
        o.viscosity = Scalar(l.viscosity);
        o.density = Scalar(l.density);
        o.surfaceTension = Scalar(l.surfaceTension);
        o.correctCycle = int(l.correctCycle);
        o.gravity = Scalar(scene.GetGravity());
        return o;
    }
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
        lp.correct_volume = liquid.correctVolume ? 1 : 0;
        lp.correct_cycle = liquid.correctCycle;
        lhi_liquid* h = nullptr;
        Check(lhi_liquid_create(&g, &sp, &lp, precision, &h), "lhi_liquid_create");
        return h;
    }

    LiquidParameter liquid_;
    Vector3 minCoord_, maxCoord_;
    std::array<int, 3> dim_;
    lhi_liquid* h_ = nullptr;
    ParticleSystem<3> ps_;
    CGSolver<3> solver_;
    std::vector<lhi_boundary_node> boundary_;
    int root_ = 0;
    std::function<Scalar(Scalar, Scalar, Scalar)> host_boundary_;
};

}  // namespace lhi_b200

#endif  // LHI_LIQUID_HPP_
