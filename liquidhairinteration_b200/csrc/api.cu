// api.cu -- the C-ABI of include/lhi.h: argument checking, error reporting
// (thread-local last error, int status codes) and dispatch to the handle's
// precision-specific implementation.  No exception crosses the boundary.
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>
#include <new>
#include <string>

#include "impl.cuh"
#include "lhi.h"
#include "net.cuh"

struct lhi_liquid {
    std::unique_ptr<lhi::LiquidBase> impl;
};

struct lhi_net {
    std::unique_ptr<lhi::LearnedNet> impl;
    cudaStream_t stream = nullptr;
    ~lhi_net() {
        impl.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace lhi {
std::atomic<long long> g_kernel_launches{0};
int divergence_noalloc(const int32_t dim[3], double dx, int32_t precision, const void* liquid_phi,
                       const void* liquid_wx, const void* liquid_wy, const void* liquid_wz, const void* vx,
                       const void* vy, const void* vz, void* stream, double* mean, double* max_abs);
}

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int from_cuda(const lhi::CudaError& e) {
    int code = (e.code == cudaErrorMemoryAllocation) ? LHI_E_OOM : LHI_E_CUDA;
    return fail(code, e.what());
}

template <class F> int guarded(F f) {
    try {
        return f();
    } catch (const lhi::CudaError& e) {
        return from_cuda(e);
    } catch (const std::invalid_argument& e) {
        return fail(LHI_E_INVALID_ARG, e.what());
    } catch (const std::bad_alloc& e) {
        return fail(LHI_E_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(LHI_E_CUDA, e.what());
    }
}

#define NEED_HANDLE(h) \
    if (!(h) || !(h)->impl) return fail(LHI_E_INVALID_ARG, "null handle")

// Converts the caller's boundary tree (root + child indices, BaseBoundary
// ownership layout of Boundary.h) into post-order so the device evaluates
// each node once, children first.
void emit(const lhi_boundary_node* nodes, int32_t count, int32_t idx, lhi::BoundaryProgram& prog, int depth,
          int* slot) {
    if (idx < 0 || idx >= count) throw std::invalid_argument("boundary tree: child index out of range");
    if (depth > 64) throw std::invalid_argument("boundary tree: too deep (cycle?)");
    const lhi_boundary_node& n = nodes[idx];
    int l = -1, r = -1;
    switch (n.kind) {
        case LHI_BOUNDARY_RECT:
        case LHI_BOUNDARY_SOLID: break;
        case LHI_BOUNDARY_UNION:
        case LHI_BOUNDARY_INTERSECTION:
        case LHI_BOUNDARY_SUBTRACT:
            emit(nodes, count, n.left, prog, depth + 1, &l);
            emit(nodes, count, n.right, prog, depth + 1, &r);
            break;
        case LHI_BOUNDARY_NONE: emit(nodes, count, n.left, prog, depth + 1, &l); break;
        default: throw std::invalid_argument("boundary tree: unknown node kind");
    }
    if (prog.count >= lhi::kMaxBoundaryNodes) throw std::invalid_argument("boundary tree: more than 32 nodes");
    int k = prog.count++;
    prog.kind[k] = n.kind;
    prog.use_inside[k] = n.use_inside;
    prog.left[k] = l;
    prog.right[k] = r;
    for (int i = 0; i < 3; ++i) {
        prog.center[k][i] = n.center[i];
        prog.half[k][i] = n.half_extent[i];
    }
    *slot = k;
}

}  // namespace

extern "C" {

void lhi_set_error_message(const char* msg) { g_last_error = msg ? msg : ""; }

LHI_API const char* lhi_last_error(void) { return g_last_error.c_str(); }

LHI_API int lhi_liquid_create(const lhi_grid_desc* grid, const lhi_solver_params* solver,
                              const lhi_liquid_params* liquid, int32_t precision, lhi_liquid** out) {
    if (!grid || !solver || !liquid || !out) return fail(LHI_E_INVALID_ARG, "null argument");
    *out = nullptr;
    return guarded([&]() -> int {
        std::unique_ptr<lhi_liquid> h(new lhi_liquid());
        switch (precision) {
            case LHI_PRECISION_FP32:
                h->impl.reset(new lhi::LiquidImpl<float, float>(*grid, *solver, *liquid, precision));
                break;
            case LHI_PRECISION_MIXED:
                h->impl.reset(new lhi::LiquidImpl<float, double>(*grid, *solver, *liquid, precision));
                break;
            case LHI_PRECISION_FP64:
                h->impl.reset(new lhi::LiquidImpl<double, double>(*grid, *solver, *liquid, precision));
                break;
            default: return fail(LHI_E_INVALID_ARG, "unknown precision");
        }
        *out = h.release();
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_destroy(lhi_liquid* h) {
    if (!h) return LHI_OK;
    return guarded([&]() -> int {
        delete h;
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_precision(const lhi_liquid* h, int32_t* precision) {
    NEED_HANDLE(h);
    if (!precision) return fail(LHI_E_INVALID_ARG, "null argument");
    *precision = h->impl->precision();
    return LHI_OK;
}

LHI_API int lhi_liquid_sync(lhi_liquid* h) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        h->impl->sync();
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_get_dx(const lhi_liquid* h, double dx[3]) {
    NEED_HANDLE(h);
    if (!dx) return fail(LHI_E_INVALID_ARG, "null argument");
    h->impl->dx(dx);
    return LHI_OK;
}

LHI_API int lhi_liquid_set_boundary(lhi_liquid* h, const lhi_boundary_node* nodes, int32_t count, int32_t root) {
    NEED_HANDLE(h);
    if (!nodes || count <= 0) return fail(LHI_E_INVALID_ARG, "empty boundary tree");
    return guarded([&]() -> int {
        lhi::BoundaryProgram prog;
        std::memset(&prog, 0, sizeof(prog));
        int slot = -1;
        emit(nodes, count, root, prog, 0, &slot);
        prog.root = slot;
        h->impl->set_boundary(prog);
        h->impl->sync();
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_set_solid_phi(lhi_liquid* h, const void* node_phi) {
    NEED_HANDLE(h);
    if (!node_phi) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        h->impl->set_solid_phi(node_phi);
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_set_particles(lhi_liquid* h, int64_t n, const void* pos, const void* vel, const void* affine) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        h->impl->set_particles(n, pos, vel, affine);
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_get_particles(lhi_liquid* h, void* pos, void* vel, void* affine) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        h->impl->get_particles(pos, vel, affine);
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_num_particles(const lhi_liquid* h, int64_t* n) {
    NEED_HANDLE(h);
    if (!n) return fail(LHI_E_INVALID_ARG, "null argument");
    *n = h->impl->num_particles();
    return LHI_OK;
}

#define STAGE(name, call)                 \
    LHI_API int name {                    \
        NEED_HANDLE(h);                   \
        return guarded([&]() -> int {     \
            call;                         \
            return LHI_OK;                \
        });                               \
    }

STAGE(lhi_liquid_clear(lhi_liquid* h), h->impl->clear())
STAGE(lhi_liquid_sort_particles(lhi_liquid* h), h->impl->sort_particles())
STAGE(lhi_liquid_compute_liquid_phi(lhi_liquid* h), h->impl->compute_liquid_phi())
STAGE(lhi_liquid_particle_to_grid(lhi_liquid* h), h->impl->particle_to_grid())
STAGE(lhi_liquid_apply_gravity(lhi_liquid* h, double dt), h->impl->apply_gravity(dt))
STAGE(lhi_liquid_velocity_update(lhi_liquid* h, double dt), h->impl->velocity_update(dt))
STAGE(lhi_liquid_extrapolate(lhi_liquid* h), h->impl->extrapolate())
STAGE(lhi_liquid_grid_to_particle(lhi_liquid* h), h->impl->grid_to_particle())
STAGE(lhi_liquid_advect_particles(lhi_liquid* h, double dt), h->impl->advect(dt))
STAGE(lhi_liquid_post_step(lhi_liquid* h, double dt), (void)dt; h->impl->sync())
STAGE(lhi_solver_init(lhi_liquid* h), h->impl->solver_init())
STAGE(lhi_solver_build_rhs(lhi_liquid* h), h->impl->build_rhs())
STAGE(lhi_solver_build_lhs(lhi_liquid* h, double density, double dt), h->impl->build_lhs(density, dt))
STAGE(lhi_solver_apply_preconditioner(lhi_liquid* h), h->impl->apply_preconditioner())

// Projection and step report a NaN in the solve; a solve that stops at the
// iteration cap is not an error here (the reference carries on as well), its
// status is available from lhi_solver_get_stats.
LHI_API int lhi_liquid_projection(lhi_liquid* h, double dt) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        int st = h->impl->projection(dt);
        if (st == LHI_E_NAN) return fail(LHI_E_NAN, "pressure solve produced NaN/Inf");
        if (st == LHI_E_TIMEOUT) return fail(LHI_E_TIMEOUT, "a bounded wait of the solver kernels ran out");
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_pre_step(lhi_liquid* h, double dt) {
    NEED_HANDLE(h);
    return guarded([&]() -> int { return h->impl->pre_step(dt); });
}

LHI_API int lhi_liquid_step(lhi_liquid* h, double dt) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        int st = h->impl->step(dt);
        if (st == LHI_E_NAN) return fail(LHI_E_NAN, "pressure solve produced NaN/Inf");
        if (st == LHI_E_TIMEOUT) return fail(LHI_E_TIMEOUT, "a bounded wait of the solver kernels ran out");
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_compute_divergence(lhi_liquid* h, double* mean, double* max_abs) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        h->impl->divergence(mean, max_abs);
        return LHI_OK;
    });
}

LHI_API int lhi_divergence_noalloc(const int32_t dim[3], double dx, int32_t precision, const void* liquid_phi,
                                   const void* liquid_wx, const void* liquid_wy, const void* liquid_wz,
                                   const void* vx, const void* vy, const void* vz, void* stream, double* mean,
                                   double* max_abs) {
    return guarded([&]() -> int {
        return lhi::divergence_noalloc(dim, dx, precision, liquid_phi, liquid_wx, liquid_wy, liquid_wz, vx, vy,
                                       vz, stream, mean, max_abs);
    });
}

// ------------------------------------------------------------ network
LHI_API int lhi_net_create(uint64_t seed, lhi_net** out) {
    if (!out) return fail(LHI_E_INVALID_ARG, "null argument");
    *out = nullptr;
    return guarded([&]() -> int {
        std::unique_ptr<lhi_net> n(new lhi_net());
        LHI_CUDA(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking));
        n->impl.reset(new lhi::LearnedNet(seed));
        *out = n.release();
        return LHI_OK;
    });
}

LHI_API int lhi_net_destroy(lhi_net* net) {
    if (!net) return LHI_OK;
    return guarded([&]() -> int {
        delete net;
        return LHI_OK;
    });
}

LHI_API int lhi_net_num_params(int64_t* count) {
    if (!count) return fail(LHI_E_INVALID_ARG, "null argument");
    *count = lhi::net_param_count();
    return LHI_OK;
}

LHI_API int lhi_net_get_params(lhi_net* net, float* out) {
    if (!net || !out) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        net->impl->get_params(out);
        return LHI_OK;
    });
}

LHI_API int lhi_net_set_relu(lhi_net* net, int32_t relu) {
    if (!net) return fail(LHI_E_INVALID_ARG, "null argument");
    net->impl->relu_ = relu != 0;
    return LHI_OK;
}

LHI_API int lhi_net_set_sparse(lhi_net* net, int32_t on) {
    if (!net) return fail(LHI_E_INVALID_ARG, "null argument");
    net->impl->sparse_enabled_ = on != 0;
    return LHI_OK;
}

LHI_API int lhi_net_save(lhi_net* net, const char* path) {
    if (!net || !path) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        const long long n = lhi::net_param_count();
        std::vector<float> p(static_cast<size_t>(n));
        net->impl->get_params(p.data());
        FILE* f = std::fopen(path, "wb");
        if (!f) return fail(LHI_E_INVALID_ARG, std::string("cannot open ") + path);
        const int64_t cnt = n;
        bool ok = std::fwrite("LHINET01", 1, 8, f) == 8 && std::fwrite(&cnt, 8, 1, f) == 1 &&
                  std::fwrite(p.data(), 4, size_t(n), f) == size_t(n);
        ok = (std::fclose(f) == 0) && ok;
        return ok ? LHI_OK : fail(LHI_E_INVALID_ARG, std::string("write failed: ") + path);
    });
}

LHI_API int lhi_net_load(lhi_net* net, const char* path) {
    if (!net || !path) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        FILE* f = std::fopen(path, "rb");
        if (!f) return fail(LHI_E_INVALID_ARG, std::string("cannot open ") + path);
        char tag[8];
        int64_t cnt = 0;
        const long long n = lhi::net_param_count();
        std::vector<float> p(static_cast<size_t>(n));
        bool ok = std::fread(tag, 1, 8, f) == 8 && std::memcmp(tag, "LHINET01", 8) == 0 && std::fread(&cnt, 8, 1, f) == 1 &&
                  cnt == n && std::fread(p.data(), 4, size_t(n), f) == size_t(n);
        std::fclose(f);
        if (!ok) return fail(LHI_E_INVALID_ARG, std::string("not a network parameter file of this layout: ") + path);
        net->impl->set_params(p.data());
        return LHI_OK;
    });
}

LHI_API int lhi_net_set_params(lhi_net* net, const float* in) {
    if (!net || !in) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        net->impl->set_params(in);
        return LHI_OK;
    });
}

namespace {
// device copies of host inputs for the host-buffer network entry points
struct NetHostArgs {
    float* r = nullptr;
    uint8_t* type = nullptr;
    uint8_t* solid = nullptr;
    float* z = nullptr;
    float* dz = nullptr;
    ~NetHostArgs() {
        cudaFree(r);
        cudaFree(type);
        cudaFree(solid);
        cudaFree(z);
        cudaFree(dz);
    }
};

long long net_dims_check(const int32_t dims[3]) {
    if (!dims) throw std::invalid_argument("null dims");
    for (int a = 0; a < 3; ++a)
        if (dims[a] < 4 || dims[a] > 4096) throw std::invalid_argument("network grid axes must be in [4, 4096]");
    return (long long)dims[0] * dims[1] * dims[2];
}

void net_upload(NetHostArgs& d, long long n, const float* r, const uint8_t* type, const uint8_t* solid, cudaStream_t s) {
    LHI_CUDA(cudaMalloc(&d.r, sizeof(float) * n));
    LHI_CUDA(cudaMalloc(&d.type, size_t(n)));
    LHI_CUDA(cudaMalloc(&d.z, sizeof(float) * n));
    LHI_CUDA(cudaMemcpyAsync(d.r, r, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    LHI_CUDA(cudaMemcpyAsync(d.type, type, size_t(n), cudaMemcpyHostToDevice, s));
    if (solid) {
        LHI_CUDA(cudaMalloc(&d.solid, size_t(n)));
        LHI_CUDA(cudaMemcpyAsync(d.solid, solid, size_t(n), cudaMemcpyHostToDevice, s));
    }
}
}  // namespace

LHI_API int lhi_solver_set_network(lhi_liquid* h, lhi_net* net, int32_t fallback_iterations) {
    NEED_HANDLE(h);
    if (!net) return fail(LHI_E_INVALID_ARG, "null network");
    return guarded([&]() -> int {
        h->impl->set_network(net->impl.get(), fallback_iterations);
        return LHI_OK;
    });
}

LHI_API int lhi_solver_learned_stats(lhi_liquid* h, int32_t* network_iterations, int32_t* fallback_iteration) {
    NEED_HANDLE(h);
    if (!network_iterations || !fallback_iteration) return fail(LHI_E_INVALID_ARG, "null argument");
    h->impl->learned_stats(network_iterations, fallback_iteration);
    return LHI_OK;
}

LHI_API int lhi_solver_record_residuals(lhi_liquid* h, int32_t max_snapshots) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        h->impl->record_residuals(max_snapshots);
        return LHI_OK;
    });
}

LHI_API int lhi_solver_num_snapshots(lhi_liquid* h, int32_t* count) {
    NEED_HANDLE(h);
    if (!count) return fail(LHI_E_INVALID_ARG, "null argument");
    *count = h->impl->num_snapshots();
    return LHI_OK;
}

LHI_API int lhi_solver_get_snapshot(lhi_liquid* h, int32_t index, float* out) {
    NEED_HANDLE(h);
    if (!out) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        h->impl->get_snapshot(index, out);
        return LHI_OK;
    });
}

LHI_API int lhi_net_train(lhi_net* net, lhi_liquid* h, int32_t steps, int32_t batch, double lr, uint64_t seed,
                          double* first_loss, double* last_loss) {
    NEED_HANDLE(h);
    if (!net || !first_loss || !last_loss) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        h->impl->train(net->impl.get(), steps, batch, lr, seed, first_loss, last_loss);
        return LHI_OK;
    });
}

LHI_API int lhi_net_tensor_core_selftest(int32_t n, int32_t k, const uint16_t* a, const uint16_t* b, float* d,
                                         int32_t* stage) {
    if (!a || !b || !d || !stage) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        int st = 0;
        const int rc = lhi::umma_selftest(a, b, n, k, d, &st);
        *stage = st;
        return rc == LHI_OK ? LHI_OK : fail(rc, "tensor-core self-test timed out at stage " + std::to_string(st));
    });
}

LHI_API int lhi_net_forward_host(lhi_net* net, const int32_t dims[3], const float* r, const uint8_t* type,
                                 const uint8_t* solid, double scale, float* z) {
    if (!net || !r || !type || !z) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        const long long n = net_dims_check(dims);
        NetHostArgs d;
        net_upload(d, n, r, type, solid, net->stream);
        const int dd[3] = {dims[0], dims[1], dims[2]};
        if (net->impl->sparse_enabled_) net->impl->plan_sparse(dd, d.type, net->stream);
        net->impl->forward(dd, d.r, d.type, d.solid, d.z, scale, net->stream, true);
        LHI_CUDA(cudaMemcpyAsync(z, d.z, sizeof(float) * n, cudaMemcpyDeviceToHost, net->stream));
        LHI_CUDA(cudaStreamSynchronize(net->stream));
        const int st = net->impl->check_status(net->stream);
        if (st != LHI_OK)
            return fail(st, "tensor-core pipeline wait timed out (kernel " + std::to_string(net->impl->last_timeout_[0]) +
                                ", step " + std::to_string(net->impl->last_timeout_[1]) + ", block " +
                                std::to_string(net->impl->last_timeout_[2]) + ")");
        return LHI_OK;
    });
}

LHI_API int lhi_net_backward_host(lhi_net* net, const int32_t dims[3], const float* r, const uint8_t* type,
                                  const uint8_t* solid, double scale, const float* dz, float* grad) {
    if (!net || !r || !type || !dz || !grad) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        const long long n = net_dims_check(dims);
        NetHostArgs d;
        net_upload(d, n, r, type, solid, net->stream);
        LHI_CUDA(cudaMalloc(&d.dz, sizeof(float) * n));
        LHI_CUDA(cudaMemcpyAsync(d.dz, dz, sizeof(float) * n, cudaMemcpyHostToDevice, net->stream));
        const int dd[3] = {dims[0], dims[1], dims[2]};
        net->impl->zero_grad(net->stream);
        net->impl->forward(dd, d.r, d.type, d.solid, d.z, scale, net->stream);
        net->impl->backward(d.dz, net->stream);
        net->impl->get_grads(grad, net->stream);
        const int st = net->impl->check_status(net->stream);
        return st == LHI_OK ? LHI_OK : fail(st, "tensor-core pipeline wait timed out");
    });
}

LHI_API int lhi_liquid_get_cfl(lhi_liquid* h, double* dt_out) {
    NEED_HANDLE(h);
    if (!dt_out) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        *dt_out = h->impl->cfl();
        return LHI_OK;
    });
}

LHI_API int lhi_solver_solve(lhi_liquid* h, double density, double dt, lhi_solve_stats* stats) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        int st = h->impl->solve(density, dt);
        if (stats) *stats = h->impl->stats();
        if (st == LHI_E_NAN) return fail(LHI_E_NAN, "pressure solve produced NaN/Inf");
        if (st == LHI_E_NOT_CONVERGED) return fail(LHI_E_NOT_CONVERGED, "pressure solve hit the iteration cap");
        if (st == LHI_E_TIMEOUT) return fail(LHI_E_TIMEOUT, "a bounded wait of the solver kernels ran out");
        return LHI_OK;
    });
}

LHI_API int lhi_solver_get_stats(lhi_liquid* h, lhi_solve_stats* stats) {
    NEED_HANDLE(h);
    if (!stats) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        *stats = h->impl->stats();  // synchronises when an asynchronous solve is pending
        return LHI_OK;
    });
}

LHI_API int lhi_solver_get_ax(lhi_liquid* h, int32_t level, const void* x, void* out) {
    NEED_HANDLE(h);
    if (!x || !out) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        h->impl->get_ax(level, x, out);
        return LHI_OK;
    });
}

LHI_API int lhi_debug_set_stage_wait_limit(double ms) {
    if (!(ms >= 0.0) || ms > 1e6) return fail(LHI_E_INVALID_ARG, "wait limit must be in [0, 1e6] ms");
    return guarded([&]() -> int {
        lhi::set_stage_wait_limit_ns((unsigned long long)(ms * 1e6));
        lhi::set_net_wait_limit_ns((unsigned long long)(ms * 1e6));
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_correct_volume(lhi_liquid* h, double dt) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        h->impl->correct_volume(dt);
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_render(lhi_liquid* h, const lhi_render_params* params, float* ndc, uint8_t* rgba) {
    NEED_HANDLE(h);
    if (!params) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        h->impl->render(*params, ndc, rgba);
        return LHI_OK;
    });
}

LHI_API int lhi_solver_spmv(lhi_liquid* h, double* p_dot_ap, int32_t* tma_kernel) {
    NEED_HANDLE(h);
    if (!p_dot_ap) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        int tma = 0;
        *p_dot_ap = h->impl->spmv_p(&tma);
        if (tma_kernel) *tma_kernel = tma;
        return LHI_OK;
    });
}

LHI_API int lhi_solver_active_tiles(lhi_liquid* h, int32_t level, int32_t* active, int32_t* total,
                                    int32_t* coarse) {
    NEED_HANDLE(h);
    if (!active || !total || !coarse) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        h->impl->active_tiles(level, active, total, coarse);
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_field_size(const lhi_liquid* h, int32_t field, int32_t level, int64_t* count,
                                  int32_t* elem_bytes) {
    NEED_HANDLE(h);
    if (!count || !elem_bytes) return fail(LHI_E_INVALID_ARG, "null argument");
    int rc = h->impl->field_size(field, level, count, elem_bytes);
    if (rc) return fail(rc, "unknown field or level");
    return LHI_OK;
}

LHI_API int lhi_liquid_get_field(lhi_liquid* h, int32_t field, int32_t level, void* out) {
    NEED_HANDLE(h);
    if (!out) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        h->impl->get_field(field, level, out);
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_set_field(lhi_liquid* h, int32_t field, int32_t level, const void* in) {
    NEED_HANDLE(h);
    if (!in) return fail(LHI_E_INVALID_ARG, "null argument");
    return guarded([&]() -> int {
        h->impl->set_field(field, level, in);
        return LHI_OK;
    });
}

LHI_API const char* lhi_solver_graph_error(lhi_liquid* h) {
    if (!h || !h->impl) return "null handle";
    return h->impl->graph_error().c_str();
}

LHI_API int lhi_liquid_set_async(lhi_liquid* h, int32_t on) {
    NEED_HANDLE(h);
    h->impl->set_async(on != 0);
    return LHI_OK;
}

LHI_API int lhi_liquid_stream(lhi_liquid* h, void** stream) {
    NEED_HANDLE(h);
    if (!stream) return fail(LHI_E_INVALID_ARG, "null argument");
    *stream = reinterpret_cast<void*>(h->impl->stream());
    return LHI_OK;
}

LHI_API int lhi_kernel_launch_count(int64_t* count) {
    if (!count) return fail(LHI_E_INVALID_ARG, "null argument");
    *count = lhi::g_kernel_launches.load();
    return LHI_OK;
}

LHI_API int lhi_liquid_profile(lhi_liquid* h, int32_t enable) {
    NEED_HANDLE(h);
    return guarded([&]() -> int {
        lhi::Profiler& p = h->impl->profiler();
        if (enable) p.reset();
        else p.drain();
        p.on = enable != 0;
        return LHI_OK;
    });
}

LHI_API int lhi_liquid_profile_read(lhi_liquid* h, int32_t category, int64_t* launches, double* total_ms) {
    NEED_HANDLE(h);
    if (category < 0 || category >= LHI_KERNEL_COUNT) return fail(LHI_E_INVALID_ARG, "unknown kernel category");
    return guarded([&]() -> int {
        lhi::Profiler& p = h->impl->profiler();
        p.drain();
        if (launches) *launches = p.launches[category];
        if (total_ms) *total_ms = p.ms[category];
        return LHI_OK;
    });
}

}  // extern "C"
