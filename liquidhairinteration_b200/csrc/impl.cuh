// impl.cuh -- device state and host orchestration of one liquid handle.
//
// LiquidImpl<T, TX> owns every device buffer of one scene: the MAC grid of
// Grid<3> (Grid.h:146-171) in the reference's x-major / z-fastest layout, the
// particle state as structure-of-arrays kept physically sorted by cell, and
// the multigrid levels of CGSolver<3> (PressureSolver.h:121-145) with the
// 7-point matrix stored per face instead of per row.
//   T  : grid, particle, matrix and V-cycle scalar (float or double)
//   TX : scalar of the outer CG iterate x (double in the mixed mode)
#pragma once

#include <string>
#include <type_traits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "common.cuh"
#include "lhi.h"
#include "net.cuh"
#include "tma.cuh"

// One window offset of the liquid SDF's gather: a lower bound (with a safety
// margin) of |x_c - x_p| - r over every particle of the window cell at this
// offset from cell c, and the offset packed as (ox + 16) | (oy + 16) << 8 |
// (oz + 16) << 16.
struct LphiOffset {
    double lb;
    int32_t off;
    int32_t pad;
};

namespace lhi {

constexpr int kMaxBoundaryNodes = 32;
constexpr int kMaxLevels = 10;

// Boundary tree in evaluation (post-) order: children precede parents.
struct BoundaryProgram {
    int count;
    int root;
    int kind[kMaxBoundaryNodes];
    int use_inside[kMaxBoundaryNodes];
    int left[kMaxBoundaryNodes];
    int right[kMaxBoundaryNodes];
    double center[kMaxBoundaryNodes][3];
    double half[kMaxBoundaryNodes][3];
};

// Device-resident PCG state: scalars, control flags and the per-level
// active-tile counts, read back by the host in one copy.
struct SolveScalars {
    double rz_old;    // r.z of the previous iteration
    double rz_new;
    double denom;     // p.Ap over the update region
    double res2;      // sum r^2 over the update region (recursive or true residual)
    double apz;       // Ap.z over the update region (flexible beta)
    double rr_all;    // sum r^2 over all cells (initial residual)
    double true2;     // sum (b - A x)^2 over the update region
    double div[3];    // divergence diagnostic: sum, count, max |div|
    double vmax;      // max |v| over particles (CFL)
    double alpha;
    double beta;
    double threshold; // stopping threshold on ||r||
    double residual0; // ||r0|| over all cells
    double residual;  // last ||r|| the stopping rule saw
    double red[4];    // spare reduction outputs
    int iter;         // PCG iterations taken
    int stop;         // 1 once the loop has ended: every loop kernel returns at once
    int status;       // LHI_OK / LHI_E_NOT_CONVERGED / LHI_E_NAN
    int true_now;     // this iteration recomputes r = b - A x
    int tile_count[kMaxLevels];
    int timeout;      // a bounded wait on a shared-memory staging copy gave up
    int p2g_overflow;  // P2G: particles outside the cell they were sorted into (listed for a second kernel)
};

// Active-tile set of one level: 8 x 8 x 32-cell tiles (x, y, z) holding a
// cell with phi <= 0 at that level, or covering an active tile of the next
// finer level; listed in increasing tile index.
constexpr int kTileX = 8, kTileY = 8, kTileZ = 32;
constexpr int kTileThreads = 256;  // 8 warps: warp w takes x = x0 + w, lane = z - z0
constexpr int kDefaultCoarseCells = 4096;  // levels below the finest this small go to one CTA
constexpr size_t kCoarseSmemBytes = 224 * 1024;  // shared memory of that CTA
constexpr int kCoarseThreads = 1024;

struct GridGeom {
    int nx, ny, nz;
};

template <class T> struct LevelDev {
    int nx, ny, nz;
    long long n;
    T* diag = nullptr;
    T* cf[3] = {nullptr, nullptr, nullptr};  // coefficient of the +x/+y/+z face of each cell
    uint8_t* type = nullptr;                 // 0 air (phi>0), 1 phi==0, 2 fluid (phi<0)
    T* phi = nullptr;                        // GetApproxLiquidPhi at this level
    T* r = nullptr;
    T* z = nullptr;
    T h[3];                                  // level spacing: factor * dx
    int tdim[3] = {0, 0, 0};                 // tiles per axis
    int ntiles = 0;
    uint8_t* tile_flag = nullptr;            // ntiles
    int32_t* tiles = nullptr;                // active tile ids, count in SolveScalars::tile_count
    // fused red-black sweep (FP32 levels whose nz is a multiple of 4)
    bool fused = false;
    T* zb = nullptr;                         // the sweep writes here, then z and zb swap
    uint8_t* mask = nullptr;                 // neighbour mask per cell, [nx][ny][mpitch]
    int mpitch = 0;
    CUtensorMap tm_z, tm_zb, tm_r, tm_d, tm_cx, tm_cy, tm_cz, tm_m;
    // one-tile boxes of the TMA restriction: z (and zb) grown by one cell,
    // r, diag, the coefficients with the -x / -y / -z faces, the mask
    CUtensorMap ts_z, ts_zb, ts_r, ts_d, ts_cx, ts_cy, ts_cz, ts_m;
};

// Optional per-category device timing: CUDA events on the handle's stream
// around every launch of a category while profiling is on.
struct Profiler {
    struct Rec {
        int cat;
        cudaEvent_t a, b;
    };
    bool on = false;
    std::vector<cudaEvent_t> pool;
    std::vector<Rec> recs;
    long long launches[LHI_KERNEL_COUNT] = {};
    double ms[LHI_KERNEL_COUNT] = {};
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        LHI_CUDA(cudaEventCreate(&e));
        return e;
    }
    // folds finished records into the totals (synchronises on the last one)
    void drain() {
        if (recs.empty()) return;
        LHI_CUDA(cudaEventSynchronize(recs.back().b));
        for (const Rec& r : recs) {
            float t = 0.f;
            LHI_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
            ms[r.cat] += t;
            launches[r.cat] += 1;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        recs.clear();
    }
    void reset() {
        drain();
        for (int i = 0; i < LHI_KERNEL_COUNT; ++i) {
            launches[i] = 0;
            ms[i] = 0.0;
        }
    }
    ~Profiler() {
        for (const Rec& r : recs) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    }
};

// Names of the LHI_KERNEL_* categories, as the NVTX ranges of the stages
// carry them (a profiler that records NVTX, such as Nsight Systems, shows
// each stage of a step under its name; without one the ranges cost nothing).
inline const char* kernel_category_name(int cat) {
    static const char* names[LHI_KERNEL_COUNT] = {"sort",          "liquid_phi", "p2g",     "g2p",     "extrapolate",
                                                  "grid",          "lhs",        "smooth_fine", "smooth_coarse",
                                                  "restrict",      "prolong",    "spmv",    "cg_vector"};
    return (cat >= 0 && cat < LHI_KERNEL_COUNT) ? names[cat] : "lhi";
}

class ProfScope {
public:
    ProfScope(Profiler& p, cudaStream_t s, int cat) : p_(p), s_(s), cat_(cat) {
        nvtxRangePushA(kernel_category_name(cat));
        if (p_.on) {
            a_ = p_.get();
            LHI_CUDA(cudaEventRecord(a_, s_));
        }
    }
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;
    ~ProfScope() {
        nvtxRangePop();
        if (!a_) return;
        cudaEvent_t b = nullptr;
        if (cudaEventCreate(&b) != cudaSuccess) return;
        if (!p_.pool.empty()) {
            cudaEventDestroy(b);
            b = p_.pool.back();
            p_.pool.pop_back();
        }
        cudaEventRecord(b, s_);
        p_.recs.push_back({cat_, a_, b});
    }

private:
    Profiler& p_;
    cudaStream_t s_;
    int cat_;
    cudaEvent_t a_ = nullptr;
};

// Polymorphic front so the C-ABI can hold any precision behind one pointer.
class LiquidBase {
public:
    virtual ~LiquidBase() {}
    virtual int precision() const = 0;
    virtual void dx(double out[3]) const = 0;
    virtual void set_boundary(const BoundaryProgram& prog) = 0;
    virtual void set_solid_phi(const void* host) = 0;
    virtual void set_particles(int64_t n, const void* pos, const void* vel, const void* aff) = 0;
    virtual void get_particles(void* pos, void* vel, void* aff) = 0;
    virtual int64_t num_particles() const = 0;
    virtual void clear() = 0;
    virtual void sort_particles() = 0;
    virtual void compute_liquid_phi() = 0;
    virtual void particle_to_grid() = 0;
    virtual void apply_gravity(double dt) = 0;
    virtual int projection(double dt) = 0;
    virtual void velocity_update(double dt) = 0;
    virtual void extrapolate() = 0;
    virtual void grid_to_particle() = 0;
    virtual void advect(double dt) = 0;
    virtual int pre_step(double dt) = 0;
    virtual int step(double dt) = 0;
    virtual void divergence(double* mean, double* max_abs) = 0;
    virtual double cfl() = 0;
    virtual void solver_init() = 0;
    virtual void build_rhs() = 0;
    virtual void build_lhs(double rho, double dt) = 0;
    virtual void apply_preconditioner() = 0;
    virtual int solve(double rho, double dt) = 0;
    virtual lhi_solve_stats stats() = 0;
    virtual void set_async(bool on) = 0;
    virtual const std::string& graph_error() const = 0;
    virtual void get_ax(int level, const void* x, void* out) = 0;
    virtual double spmv_p(int* tma) = 0;
    virtual void render(const lhi_render_params& rp, float* ndc_host, uint8_t* rgba_host) = 0;
    virtual void correct_volume(double dt) = 0;
    virtual void active_tiles(int level, int32_t* active, int32_t* total, int32_t* coarse) = 0;
    virtual void set_network(LearnedNet* net, int fallback_iterations) = 0;
    virtual void learned_stats(int32_t* net_iters, int32_t* fallback_at) = 0;
    virtual void record_residuals(int max_snapshots) = 0;
    virtual int num_snapshots() const = 0;
    virtual void get_snapshot(int index, float* host) = 0;
    virtual void train(LearnedNet* net, int steps, int batch, double lr, uint64_t seed, double* first,
                       double* last) = 0;
    virtual int field_size(int field, int level, int64_t* count, int32_t* eb) = 0;
    virtual void get_field(int field, int level, void* out) = 0;
    virtual void set_field(int field, int level, const void* in) = 0;
    virtual void sync() = 0;
    virtual cudaStream_t stream() const = 0;
    virtual Profiler& profiler() = 0;
};

template <class T, class TX> class LiquidImpl : public LiquidBase {
public:
    LiquidImpl(const lhi_grid_desc& g, const lhi_solver_params& sp, const lhi_liquid_params& lp, int precision);
    ~LiquidImpl() override;

    int precision() const override { return precision_; }
    void dx(double out[3]) const override {
        for (int i = 0; i < 3; ++i) out[i] = double(dx_[i]);
    }
    void set_boundary(const BoundaryProgram& prog) override;
    void set_solid_phi(const void* host) override;
    void set_particles(int64_t n, const void* pos, const void* vel, const void* aff) override;
    void get_particles(void* pos, void* vel, void* aff) override;
    int64_t num_particles() const override { return np_; }
    void clear() override;
    void sort_particles() override;
    void compute_liquid_phi() override;
    void particle_to_grid() override;
    void apply_gravity(double dt) override;
    int projection(double dt) override;
    void velocity_update(double dt) override;
    void extrapolate() override;
    void build_extrapolation_lists();
    void grid_to_particle() override;
    void advect(double dt) override;
    int pre_step(double dt) override;
    int step(double dt) override;
    void divergence(double* mean, double* max_abs) override;
    double cfl() override;
    void solver_init() override;
    void build_rhs() override;
    void build_lhs(double rho, double dt) override;
    void apply_preconditioner() override;
    int solve(double rho, double dt) override;
    lhi_solve_stats stats() override {
        if (stats_pending_) finish_stats();
        return stats_;
    }
    void set_async(bool on) override { async_ = on; }
    const std::string& graph_error() const override { return graph_error_.empty() ? tail_error_ : graph_error_; }
    void finish_stats();
    void get_ax(int level, const void* x, void* out) override;
    double spmv_p(int* tma) override;
    void render(const lhi_render_params& rp, float* ndc_host, uint8_t* rgba_host) override;
    void correct_volume(double dt) override;
    void active_tiles(int level, int32_t* active, int32_t* total, int32_t* coarse) override;
    void set_network(LearnedNet* net, int fallback_iterations) override;
    void learned_stats(int32_t* net_iters, int32_t* fallback_at) override {
        *net_iters = learned_iters_;
        *fallback_at = fallback_at_;
    }
    void record_residuals(int max_snapshots) override;
    int num_snapshots() const override { return snap_count_; }
    void get_snapshot(int index, float* host) override {
        if (index < 0 || index >= snap_count_) throw std::invalid_argument("snapshot index out of range");
        const int slot = (snap_next_ - snap_count_ + index + snap_cap_) % snap_cap_;
        LHI_CUDA(cudaMemcpyAsync(host, snaps_ + size_t(slot) * size_t(ncell_), sizeof(float) * ncell_,
                                 cudaMemcpyDeviceToHost, stream_));
        LHI_CUDA(cudaStreamSynchronize(stream_));
    }
    void train(LearnedNet* net, int steps, int batch, double lr, uint64_t seed, double* first, double* last) override;
    void ensure_solid_cells();
    void ensure_net_type();
    void record_snapshot();
    int field_size(int field, int level, int64_t* count, int32_t* eb) override;
    void get_field(int field, int level, void* out) override;
    void set_field(int field, int level, const void* in) override;
    void sync() override { LHI_CUDA(cudaStreamSynchronize(stream_)); }
    cudaStream_t stream() const override { return stream_; }
    Profiler& profiler() override { return prof_; }
    ProfScope scope(int cat) { return ProfScope(prof_, stream_, cat); }

    // ---- internals shared by the .cu files
    void alloc_particles(int64_t cap);
    void ensure_sorted();
    void apply_order();
    void build_liquid_phi_table();
    void p2g_accumulate();
    void p2g_normalize(bool with_gravity, T gdt);
    void g2p(bool advect, T dt);
    bool smooth(int level, int sweeps, bool final_dot = false);  // true if the sweep formed the r.z / Ap.z sums
    void restrict_to(int level);
    void prolong_to(int level);
    void vcycle();
    void build_tiles();
    void setup_coarse();
    void setup_fused();  // second z buffers, masks and tensor maps of the fused sweep
    void build_masks();
    void setup_spmv();  // tensor maps of the finest level's TMA SpMV
    void enqueue_vcycle();
    void enqueue_vcycle_levels();
    void enqueue_precond();
    void enqueue_init(unsigned long long cond, int use_cond);
    void enqueue_body(unsigned long long cond, int use_cond);
    void enqueue_final();
    void build_solve_graph(bool with_init);
    void spmv(int level, const T* x, T* y);
    void get_acoef(int level, T* host_out);
    void device_sum_launch_prep();
    template <class F> void with_partials(F f);
    double read_scalar(const double* dptr);
    void read_scalars();

    int precision_;
    Profiler prof_;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;

    // grid (Grid<3>)
    int nx_, ny_, nz_;
    T min_[3], max_[3], dx_[3];
    T radius_, density_, gravity_;
    int extrap_iters_;
    // CorrectVolume (LiquidModel.cpp:1086-1132): on in Step, cycle, current step, calls so far
    bool correct_in_step_ = false;
    int correct_cycle_ = 8, correct_step_ = 0;
    unsigned long long correct_calls_ = 0;
    long long ncell_, nface_[3], nnode_;
    T* v_[3] = {};    // current vx, vy, vz
    T* tv_[3] = {};   // current tempVx, tempVy, tempVz
    T* w_[3] = {};
    T* lw_[3] = {};   // liquidWx/y/z
    T* pressure_ = nullptr;
    T* liquid_phi_ = nullptr;
    T* solid_phi_ = nullptr;
    uint8_t* valid_ = nullptr;  // isValid: 255 invalid, else the sweep it became valid
    // Extrapolation work lists per component (isValid node indices), rebuilt
    // after the solid fractions or isValid change: ext_u_ the nodes of the
    // component's range that some component's init can make invalid (the
    // only ones whose flag can differ from 0 there), ext_s_ those the
    // component's own init makes invalid (the only ones its sweeps change).
    int32_t* ext_u_[3] = {};
    int32_t* ext_s_[3] = {};
    long long ext_nu_[3] = {}, ext_ns_[3] = {};
    bool ext_dirty_ = true;
    uint8_t* occ_ = nullptr;    // 4^3-cell block occupancy for the liquid SDF
    int occ_dim_[3];
    LphiOffset* lphi_tab_ = nullptr;  // the liquid SDF's window offsets by ascending distance bound
    int lphi_n_ = 0;

    // particles (SoA, sorted by cell): 15 scalars + caller id, double-buffered
    int64_t np_ = 0, pcap_ = 0;
    T* pdata_[2] = {nullptr, nullptr};  // [15][pcap]: px py pz ux uy uz c0..c8
    int32_t* pid_[2] = {nullptr, nullptr};
    int pcur_ = 0;
    bool sorted_ = false;
    bool keys_fresh_ = false;  // keys_[0]/vals_[0] hold (cell key, identity) of the current order
    // The sort's permutation not applied yet: pdata_[pcur_] is in the order
    // before the sort, vals_[0] maps a sorted index to its place there, and
    // rows 0-2 of pdata_[pcur_ ^ 1] hold the positions in sorted order.  The
    // liquid SDF, P2G and G2P + advection read through it (G2P writes the
    // sorted state, which applies it); anything else applies it first.
    bool perm_pending_ = false;
    uint32_t* keys_[2] = {nullptr, nullptr};
    int32_t* vals_[2] = {nullptr, nullptr};
    int32_t* cell_count_ = nullptr;  // ncell + 1
    int32_t* cell_start_ = nullptr;  // ncell + 1
    // headless render: RGBA image and normalised device coordinates, sized on first use
    void* image_ = nullptr;
    long long image_cap_ = 0;
    float* ndc_ = nullptr;
    long long ndc_cap_ = 0;
    void* scan_tmp_ = nullptr;
    long long scan_tmp_bytes_ = 0;

    // solver (CGSolver<3>)
    lhi_solver_params sp_;
    int nlev_;
    LevelDev<T> lv_[kMaxLevels];
    int coarse_level_ = 0;   // first level solved by the single-CTA coarse kernel (nlev_ if none)
    size_t coarse_smem_ = 0; // its dynamic shared memory
    uint32_t* coarse_list_ = nullptr;  // per-colour update lists of the coarse levels
    long long coarse_list_off_[kMaxLevels] = {};
    int* coarse_counts_ = nullptr;
    bool spmv_tma_ = false;
    bool fuse_dot_ = false;   // the V-cycle being enqueued is the PCG body's preconditioner
    bool dot_fused_ = false;  // its last level-0 sweep formed r.z, Ap.z and beta
    CUtensorMap tm_sp_[6];  // p, diag, cx, cy, cz, mask boxes of the TMA SpMV
    int tile_grid_ = 0;      // persistent CTAs of the tile kernels
    cudaStream_t cur_ = nullptr;   // stream the enqueue helpers launch on
    cudaStream_t side_ = nullptr;  // capture stream of the graph's loop body
    cudaGraphExec_t solve_exec_ = nullptr;
    cudaGraphExec_t tail_exec_ = nullptr;  // the loop and final pass without init (FPCG after its fallback)
    std::string tail_error_;               // why the tail graph could not be built (the loop stays host-driven)
    bool fallback_body_ran_ = false;       // a V-cycle body of an FPCG fallback has run host-driven
    int tail_from_iter_ = -1;              // iteration at which the last solve's tail graph took over
    long long graph_init_kernels_ = 0, graph_body_kernels_ = 0, graph_final_kernels_ = 0;
    bool async_ = false;         // steps do not wait for the solve; statistics are read on demand
    bool stats_pending_ = false; // the last graph solve's statistics are still on the device
    bool last_solve_graph_ = false;
    bool solved_once_ = false;   // graphs are captured from the second solve on
    std::string graph_error_;    // why the solve graph could not be built (then solves run host-driven)
    // learned preconditioner
    LearnedNet* net_ = nullptr;
    int fallback_iters_ = 0;
    bool use_fallback_ = false;  // this solve switched to the V-cycle
    int learned_iters_ = 0;
    int fallback_at_ = -1;
    uint8_t* solid_cell_ = nullptr;  // cell-centre solid flag (mean of the 8 node SDFs < 0)
    bool solid_cell_fresh_ = false;
    uint8_t* net_type_ = nullptr;    // level-0 type with skipped rows (small diagonal) as 0
    bool net_type_fresh_ = false;
    bool net_plan_stale_ = true;     // the network's tile plan predates net_type_
    float* snaps_ = nullptr;         // recorded residuals [snap_cap_][ncell_]
    int snap_cap_ = 0, snap_count_ = 0, snap_next_ = 0;
    float* train_z_ = nullptr;
    float* train_dz_ = nullptr;
    float* train_e_ = nullptr;
    double* train_red_ = nullptr;    // [0] sum e^2, [1] sum r^2, [2] loss accumulator
    T* rhs_ = nullptr;
    // mixed mode (T = float, TX = double): the finest level's right-hand side
    // and matrix assembled in FP64 from the same float fields, for the outer
    // CG's true residual and final check, so the iteration converges to the
    // FP64 system's solution; the V-cycle and the loop's SpMV stay FP32
    static constexpr bool kHiResidual = std::is_same<T, float>::value && std::is_same<TX, double>::value;
    double dxd_[3] = {0, 0, 0};  // grid spacing in double, as an FP64 model of the same grid computes it
    double* rhs_hi_ = nullptr;
    double* diag_hi_ = nullptr;
    double* cf_hi_[3] = {nullptr, nullptr, nullptr};
    TX* x_ = nullptr;
    T* p_ = nullptr;
    T* ap_ = nullptr;
    SolveScalars* sc_ = nullptr;      // device
    SolveScalars* sc_host_ = nullptr; // pinned mirror
    double* partials_ = nullptr;
    unsigned* counter_ = nullptr;
    int sum_blocks_ = 0;
    lhi_solve_stats stats_{};

    T* p_ptr(int k) const { return pdata_[pcur_] + size_t(k) * size_t(pcap_); }
};

// limit of the solver kernels' waits on their TMA staging copies, on the current device (k_solver.cu)
void set_stage_wait_limit_ns(unsigned long long ns);

// device-wide exclusive scan (k_sort.cu)
void device_exclusive_scan_i32(const int32_t* in, int32_t* out, long long n, void* tmp, long long tmp_bytes,
                               cudaStream_t s);
long long scan_tmp_bytes(long long n);

}  // namespace lhi
