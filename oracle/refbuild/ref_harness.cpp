// ref_harness.cpp -- C entry points that drive the reference's own liquid
// path (LiquidModel<3>, CGSolver<3>, Grid<3>, ParticleSystem<3> compiled from
// the reference tree).  TEST INFRASTRUCTURE ONLY: used to pin the oracle.
//
// Scene<3>'s constructor (Scene.cpp:13-20) is restated here so that the hair
// model, which the liquid path never touches, need not be compiled: a
// HairModel<3> stand-in with the same constructor signature takes its place.
// Private members are opened with a macro so the harness can read the grid
// and solver arrays for parity dumps; class layouts are unchanged.
#include <windows.h>  // the shim: all standard headers first, then min/max

#define private public
#define protected public
#include "LiquidModel.h"
#include "Renderer.h"
#include "Scene.h"
#undef private
#undef protected

#include "lhi.h"

#include <cstdint>
#include <cstring>

template <> class HairModel<3> {
public:
    explicit HairModel(const Scene<3>&) {}
};

// Scene<3>::Scene (Scene.cpp:13-20)
template <>
Scene<3>::Scene(const std::string& configFile)
    : m_solverParams(configFile), m_sceneParams(configFile), m_liquidParams(configFile), m_hairParams(configFile),
      m_liquidModel(std::make_unique<LiquidModel<3>>(*this)), m_hairModel(std::make_unique<HairModel<3>>(*this)) {
    m_boundary.SetChild(new RectBoundary<3>(VectorX<3>::Zero(), VectorX<3>::Ones() * 0.9, true));
    m_liquidModel->SetBoundary(&m_boundary);
}

template <> Scene<3>::~Scene() {}

// Headless: no shader program is ever created.
GLuint Renderer::CreateShaderProgram(const char*, const char*) { return 0; }

namespace {

struct RefState {
    std::unique_ptr<Scene<3>> scene;
    std::vector<BaseBoundary<3>*> tree;  // owned by the root's destructor chain; leaked on purpose
};

LiquidModel<3>& LM(void* h) { return static_cast<RefState*>(h)->scene->GetLiquidModel(); }

BaseBoundary<3>* build_node(const lhi_boundary_node* nodes, int32_t count, int32_t idx) {
    if (idx < 0 || idx >= count) return nullptr;
    const lhi_boundary_node& n = nodes[idx];
    Vector3 c(Scalar(n.center[0]), Scalar(n.center[1]), Scalar(n.center[2]));
    Vector3 h(Scalar(n.half_extent[0]), Scalar(n.half_extent[1]), Scalar(n.half_extent[2]));
    BaseBoundary<3>* b = nullptr;
    switch (n.kind) {
        case LHI_BOUNDARY_RECT: b = new RectBoundary<3>(c, h, n.use_inside != 0); break;
        case LHI_BOUNDARY_SOLID: b = new SolidBoundary<3>(c, n.use_inside != 0); break;
        case LHI_BOUNDARY_UNION: b = new OperatorBoundary<3>(OperatorBoundary<3>::OperatorType::Union); break;
        case LHI_BOUNDARY_INTERSECTION:
            b = new OperatorBoundary<3>(OperatorBoundary<3>::OperatorType::Intersection);
            break;
        case LHI_BOUNDARY_SUBTRACT: b = new OperatorBoundary<3>(OperatorBoundary<3>::OperatorType::Substract); break;
        default: b = new OperatorBoundary<3>(OperatorBoundary<3>::OperatorType::None); break;
    }
    if (n.kind >= LHI_BOUNDARY_UNION) {
        b->SetLeftChild(build_node(nodes, count, n.left));
        b->SetRightChild(build_node(nodes, count, n.right));
    }
    return b;
}

template <class A> void copy_out(const A& arr, void* out) {
    std::memcpy(out, arr.m_container.data(), arr.m_container.size() * sizeof(Scalar));
}
template <class A> void copy_in(A& arr, const void* in) {
    std::memcpy(arr.m_container.data(), in, arr.m_container.size() * sizeof(Scalar));
}

Array3<Scalar>* grid_field(LiquidModel<3>& lm, int f, int level) {
    Grid<3>& g = lm.m_grid;
    CGSolver<3>& s = lm.m_solver;
    switch (f) {
        case LHI_FIELD_VX: return &g.vx;
        case LHI_FIELD_VY: return &g.vy;
        case LHI_FIELD_VZ: return &g.vz;
        case LHI_FIELD_WX: return &g.wx;
        case LHI_FIELD_WY: return &g.wy;
        case LHI_FIELD_WZ: return &g.wz;
        case LHI_FIELD_LIQUID_WX: return &g.liquidWx;
        case LHI_FIELD_LIQUID_WY: return &g.liquidWy;
        case LHI_FIELD_LIQUID_WZ: return &g.liquidWz;
        case LHI_FIELD_TEMP_VX: return &g.tempVx;
        case LHI_FIELD_TEMP_VY: return &g.tempVy;
        case LHI_FIELD_TEMP_VZ: return &g.tempVz;
        case LHI_FIELD_PRESSURE: return &g.pressure;
        case LHI_FIELD_LIQUID_PHI: return &g.liquidPhi;
        case LHI_FIELD_SOLID_PHI: return &g.solidPhi;
        case LHI_FIELD_RHS: return &s.m_rhs;
        case LHI_FIELD_X: return &s.m_x;
        case LHI_FIELD_P: return &s.m_p;
        case LHI_FIELD_R: return (level >= 0 && level < s.m_maxLevel) ? &s.m_r[level] : nullptr;
        case LHI_FIELD_Z: return (level >= 0 && level < s.m_maxLevel) ? &s.m_z[level] : nullptr;
        case LHI_FIELD_ADIAG: return (level >= 0 && level < s.m_maxLevel) ? &s.m_Adiag[level] : nullptr;
        default: return nullptr;
    }
}

}  // namespace

extern "C" {

#define REF_API __attribute__((visibility("default")))

REF_API void* ref_create(const char* json_path) {
    try {
        auto* st = new RefState();
        st->scene = std::make_unique<Scene<3>>(std::string(json_path));
        return st;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_create: %s\n", e.what());
        return nullptr;
    }
}

REF_API void ref_destroy(void* h) { delete static_cast<RefState*>(h); }

REF_API void ref_get_dx(void* h, double dx[3]) {
    const Vector3& d = LM(h).m_grid.dx;
    for (int i = 0; i < 3; ++i) dx[i] = d[i];
}

// LiquidModel<3>::Init (LiquidModel.cpp:507-512): ComputeSolidPhi + SpawnParticles
REF_API int ref_init(void* h) {
    LM(h).Init();
    return 0;
}

REF_API int ref_set_boundary(void* h, const lhi_boundary_node* nodes, int32_t count, int32_t root) {
    BaseBoundary<3>* b = build_node(nodes, count, root);
    LM(h).SetBoundary(b);
    LM(h).ComputeSolidPhi();
    return 0;
}

REF_API int ref_compute_solid_phi(void* h) {
    LM(h).ComputeSolidPhi();
    return 0;
}

REF_API int ref_set_particles(void* h, int64_t n, const float* pos, const float* vel, const float* aff) {
    ParticleSystem<3>& ps = LM(h).GetParticleSystem();
    ps.Resize(Integer(n));
    for (int64_t i = 0; i < n; ++i) {
        ps.SetPosition(Integer(i), Vector3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]));
        ps.SetVelocity(Integer(i), vel ? Vector3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]) : Vector3::Zero());
        Matrix3 C = Matrix3::Zero();
        if (aff)
            for (int k = 0; k < 9; ++k) C.data()[k] = aff[9 * i + k];
        ps.SetAffineMatrix(Integer(i), C);
    }
    return 0;
}

REF_API int64_t ref_num_particles(void* h) { return LM(h).GetParticleSystem().NumParticles(); }

REF_API int ref_get_particles(void* h, float* pos, float* vel, float* aff) {
    ParticleSystem<3>& ps = LM(h).GetParticleSystem();
    for (Integer i = 0; i < ps.NumParticles(); ++i) {
        for (int k = 0; k < 3; ++k) {
            if (pos) pos[3 * size_t(i) + k] = ps.GetPosition(i)[k];
            if (vel) vel[3 * size_t(i) + k] = ps.GetVelocity(i)[k];
        }
        if (aff)
            for (int k = 0; k < 9; ++k) aff[9 * size_t(i) + k] = ps.GetAffineMatrix(i).data()[k];
    }
    return 0;
}

REF_API int ref_get_radius(void* h, float* radius) {
    ParticleSystem<3>& ps = LM(h).GetParticleSystem();
    for (Integer i = 0; i < ps.NumParticles(); ++i) radius[i] = ps.GetRadius(i);
    return 0;
}

REF_API int ref_get_field(void* h, int32_t field, int32_t level, void* out) {
    LiquidModel<3>& lm = LM(h);
    if (field == LHI_FIELD_IS_VALID) {
        const auto& v = lm.m_grid.isValid.m_container;
        uint8_t* o = static_cast<uint8_t*>(out);
        for (size_t i = 0; i < v.size(); ++i) o[i] = v[i] ? 1 : 0;
        return 0;
    }
    if (field == LHI_FIELD_ACOEF) {
        CGSolver<3>& s = lm.m_solver;
        if (level < 0 || level >= s.m_maxLevel) return LHI_E_INVALID_ARG;
        const auto& c = s.m_Acoef[level].m_container;
        float* o = static_cast<float*>(out);
        for (size_t i = 0; i < c.size(); ++i)
            for (int k = 0; k < 6; ++k) o[6 * i + k] = c[i][k];
        return 0;
    }
    Array3<Scalar>* a = grid_field(lm, field, level);
    if (!a) return LHI_E_INVALID_ARG;
    copy_out(*a, out);
    return 0;
}

REF_API int ref_set_field(void* h, int32_t field, int32_t level, const void* in) {
    LiquidModel<3>& lm = LM(h);
    if (field == LHI_FIELD_IS_VALID) {
        auto& v = lm.m_grid.isValid.m_container;
        const uint8_t* p = static_cast<const uint8_t*>(in);
        for (size_t i = 0; i < v.size(); ++i) v[i] = p[i] != 0;
        return 0;
    }
    Array3<Scalar>* a = grid_field(lm, field, level);
    if (!a) return LHI_E_INVALID_ARG;
    copy_in(*a, in);
    return 0;
}

REF_API int ref_clear(void* h) {
    LM(h).m_grid.Clear();
    return 0;
}
REF_API int ref_compute_liquid_phi(void* h) {
    LM(h).ComputeLiquidPhi();
    return 0;
}
REF_API int ref_particle_to_grid(void* h) {
    LM(h).Particle2Grid();
    return 0;
}
REF_API int ref_apply_gravity(void* h, float dt) {
    LM(h).ApplyGravity(dt);
    return 0;
}
REF_API int ref_solve_pressure(void* h, float dt) {
    LM(h).SolvePressure(dt);
    return 0;
}
REF_API int ref_extrapolate(void* h) {
    LM(h).Extrapolate();
    return 0;
}
REF_API int ref_grid_to_particle(void* h) {
    LM(h).Grid2Particle();
    return 0;
}
REF_API int ref_advect_particles(void* h, float dt) {
    LM(h).AdvectParticle(dt);
    return 0;
}
REF_API int ref_pre_step(void* h, float dt) {
    LM(h).PreStep(dt);
    return 0;
}
REF_API int ref_step(void* h, float dt) {
    LM(h).Step(dt);
    return 0;
}
REF_API int ref_post_step(void* h, float dt) {
    LM(h).PostStep(dt);
    return 0;
}
REF_API double ref_compute_divergence(void* h) { return double(LM(h).ComputeDivergence()); }
REF_API double ref_get_cfl(void* h) { return double(LM(h).GetCFL()); }

REF_API int ref_solver_init(void* h) {
    LM(h).m_solver.Init();
    return 0;
}
REF_API int ref_solver_build_rhs(void* h) {
    LM(h).m_solver.BuildRHS();
    return 0;
}
REF_API int ref_solver_build_lhs(void* h, float density, float dt) {
    LM(h).m_solver.BuildLHS(density, dt);
    return 0;
}
REF_API int ref_solver_apply_preconditioner(void* h) {
    LM(h).m_solver.ApplyPreconditioner();
    return 0;
}
REF_API int ref_solver_solve(void* h, float density, float dt) {
    LM(h).m_solver.Solve(density, dt);
    return 0;
}
REF_API int ref_solver_get_ax(void* h, int32_t level, const float* x, float* out) {
    CGSolver<3>& s = LM(h).m_solver;
    if (level < 0 || level >= s.m_maxLevel) return LHI_E_INVALID_ARG;
    Vector3i d = LM(h).m_grid.dimension / (1 << level);
    Array3<Scalar> g(d);
    std::memcpy(g.m_container.data(), x, g.m_container.size() * sizeof(Scalar));
    for (int xi = 0; xi < d.x(); ++xi)
        for (int yi = 0; yi < d.y(); ++yi)
            for (int zi = 0; zi < d.z(); ++zi) out[(size_t(xi) * d.y() + yi) * d.z() + zi] = s.GetAx(g, xi, yi, zi, level);
    return 0;
}

}  // extern "C"
