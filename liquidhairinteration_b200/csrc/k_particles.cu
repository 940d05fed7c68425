// k_particles.cu -- particle side of the liquid step.
//
//   keys -> counting sort -> permute : particles stay physically sorted by
//                                      cell (ties by particle id)
//   liquid SDF (ComputeLiquidPhi)    : per-cell gather over the sorted cells,
//                                      nearest window cells first
//   P2G (Particle2Grid)              : 8^3-cell tiles accumulated in shared
//                                      memory, flushed once per node
//   G2P + advection                  : 8^3-cell tiles of face velocities
//                                      staged in shared memory, one thread
//                                      per particle
#include <algorithm>

#include "impl.cuh"

namespace lhi {

template <class T> struct GridP {
    int nx, ny, nz;
    T mn[3], mx[3], dx[3];
    T idx[3];  // 1 / dx, for the gathers that need not be bit-exact
};

template <class T> __device__ __forceinline__ int cell_trunc(T p, T mn, T dx) {
    return int(X<T>::div(X<T>::sub(p, mn), dx));  // Point2Index: static_cast<Integer>
}

template <class T> __device__ __forceinline__ uint32_t cell_key(const GridP<T>& g, T x, T y, T z) {
    int cx = min(max(cell_trunc(x, g.mn[0], g.dx[0]), 0), g.nx - 1);
    int cy = min(max(cell_trunc(y, g.mn[1], g.dx[1]), 0), g.ny - 1);
    int cz = min(max(cell_trunc(z, g.mn[2], g.dx[2]), 0), g.nz - 1);
    return uint32_t((long long)(cx * g.ny + cy) * g.nz + cz);
}

// ------------------------------------------------------------------ keys
template <class T>
__global__ void k_keys(GridP<T> g, const T* __restrict__ pd, long long cap, long long n, uint32_t* __restrict__ keys,
                       int32_t* __restrict__ vals) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = cell_key(g, pd[i], pd[cap + i], pd[2 * cap + i]);
    vals[i] = int32_t(i);
}

template <class T>
__global__ void k_permute(const T* __restrict__ src, T* __restrict__ dst, long long cap,
                          const int32_t* __restrict__ sid, int32_t* __restrict__ did,
                          const int32_t* __restrict__ order, long long n) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    long long s = order[k];
#pragma unroll
    for (int c = 0; c < 15; ++c) dst[c * cap + k] = src[c * cap + s];
    did[k] = sid[s];
}

// The sorted positions alone (rows 0-2 of dst): the permutation of the rest
// waits for G2P, which reads through it and writes the sorted state.
template <class T>
__global__ void k_gather_pos(const T* __restrict__ src, T* __restrict__ dst, long long cap,
                             const int32_t* __restrict__ order, long long n) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    long long s = order[k];
#pragma unroll
    for (int c = 0; c < 3; ++c) dst[c * cap + k] = src[c * cap + s];
}

__global__ void k_cell_count(const uint32_t* __restrict__ keys, long long n, int32_t* __restrict__ count) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < n;
    uint32_t key = valid ? keys[i] : 0xffffffffu;
    unsigned peers = __match_any_sync(0xffffffffu, key);
    unsigned lane = threadIdx.x & 31;
    if (valid && (peers & ((1u << lane) - 1u)) == 0u) atomicAdd(&count[key], int(__popc(peers)));
}

// Counting-sort scatter: particle i goes to cell_start[key] + its rank among
// the particles of its cell.  Lanes of a warp with the same key take
// consecutive ranks in lane order from one atomic add; warps take their
// blocks of ranks in whatever order the atomics land, so k_cell_order then
// orders every cell by particle ID.
__global__ void k_rank_scatter(const uint32_t* __restrict__ keys, long long n, const int32_t* __restrict__ cs,
                               int32_t* __restrict__ cursor, uint32_t* __restrict__ skeys,
                               int32_t* __restrict__ order) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const uint32_t key = valid ? keys[i] : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const unsigned lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (valid && int(lane) == leader) base = atomicAdd(&cursor[key], int(__popc(peers)));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!valid) return;
    const long long pos = (long long)cs[key] + base + __popc(peers & ((1u << lane) - 1u));
    skeys[pos] = key;
    order[pos] = int32_t(i);
}

// Orders every cell's particles by particle ID (a sorting network in
// registers for up to 16, insertion sort up to 64, heap sort beyond).  The sorted order is then the stable sort
// of the caller's order by cell key whatever order the device held before,
// so every walk of the sorted lists (P2G's per-cell sums, CorrectVolume's
// neighbour sums) visits the particles in an order fixed by their state.
// Compare-exchange of (key, value) pairs: the smaller key first.
__device__ __forceinline__ void ce(int32_t& ka, int32_t& kb, int32_t& va, int32_t& vb) {
    const bool sw = ka > kb;
    const int32_t k0 = sw ? kb : ka, k1 = sw ? ka : kb, v0 = sw ? vb : va, v1 = sw ? va : vb;
    ka = k0;
    kb = k1;
    va = v0;
    vb = v1;
}

// A cell's indices sorted by particle id in registers: all loads issued at
// once, then Batcher's odd-even merge sort network (Batcher 1968) for 8 or
// 16 keys (19 / 63 compare-exchanges, checked exhaustively by the 0-1
// principle); the ids are distinct and the padding sorts last.
template <int N>
__device__ __forceinline__ void cell_order_net(int32_t* a, int len, const int32_t* __restrict__ pid) {
    int32_t v[N], k[N];
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = i < len ? a[i] : 0;
#pragma unroll
    for (int i = 0; i < N; ++i) k[i] = i < len ? pid[v[i]] : 0x7fffffff;
    if constexpr (N == 8) {
        ce(k[0], k[1], v[0], v[1]); ce(k[2], k[3], v[2], v[3]); ce(k[0], k[2], v[0], v[2]); ce(k[1], k[3], v[1], v[3]);
        ce(k[1], k[2], v[1], v[2]); ce(k[4], k[5], v[4], v[5]); ce(k[6], k[7], v[6], v[7]); ce(k[4], k[6], v[4], v[6]);
        ce(k[5], k[7], v[5], v[7]); ce(k[5], k[6], v[5], v[6]); ce(k[0], k[4], v[0], v[4]); ce(k[2], k[6], v[2], v[6]);
        ce(k[2], k[4], v[2], v[4]); ce(k[1], k[5], v[1], v[5]); ce(k[3], k[7], v[3], v[7]); ce(k[3], k[5], v[3], v[5]);
        ce(k[1], k[2], v[1], v[2]); ce(k[3], k[4], v[3], v[4]); ce(k[5], k[6], v[5], v[6]);
    } else {
        static_assert(N == 16, "networks for 8 and 16 keys");
        ce(k[0], k[1], v[0], v[1]); ce(k[2], k[3], v[2], v[3]); ce(k[0], k[2], v[0], v[2]); ce(k[1], k[3], v[1], v[3]);
        ce(k[1], k[2], v[1], v[2]); ce(k[4], k[5], v[4], v[5]); ce(k[6], k[7], v[6], v[7]); ce(k[4], k[6], v[4], v[6]);
        ce(k[5], k[7], v[5], v[7]); ce(k[5], k[6], v[5], v[6]); ce(k[0], k[4], v[0], v[4]); ce(k[2], k[6], v[2], v[6]);
        ce(k[2], k[4], v[2], v[4]); ce(k[1], k[5], v[1], v[5]); ce(k[3], k[7], v[3], v[7]); ce(k[3], k[5], v[3], v[5]);
        ce(k[1], k[2], v[1], v[2]); ce(k[3], k[4], v[3], v[4]); ce(k[5], k[6], v[5], v[6]); ce(k[8], k[9], v[8], v[9]);
        ce(k[10], k[11], v[10], v[11]); ce(k[8], k[10], v[8], v[10]); ce(k[9], k[11], v[9], v[11]);
        ce(k[9], k[10], v[9], v[10]); ce(k[12], k[13], v[12], v[13]); ce(k[14], k[15], v[14], v[15]);
        ce(k[12], k[14], v[12], v[14]); ce(k[13], k[15], v[13], v[15]); ce(k[13], k[14], v[13], v[14]);
        ce(k[8], k[12], v[8], v[12]); ce(k[10], k[14], v[10], v[14]); ce(k[10], k[12], v[10], v[12]);
        ce(k[9], k[13], v[9], v[13]); ce(k[11], k[15], v[11], v[15]); ce(k[11], k[13], v[11], v[13]);
        ce(k[9], k[10], v[9], v[10]); ce(k[11], k[12], v[11], v[12]); ce(k[13], k[14], v[13], v[14]);
        ce(k[0], k[8], v[0], v[8]); ce(k[4], k[12], v[4], v[12]); ce(k[4], k[8], v[4], v[8]);
        ce(k[2], k[10], v[2], v[10]); ce(k[6], k[14], v[6], v[14]); ce(k[6], k[10], v[6], v[10]);
        ce(k[2], k[4], v[2], v[4]); ce(k[6], k[8], v[6], v[8]); ce(k[10], k[12], v[10], v[12]);
        ce(k[1], k[9], v[1], v[9]); ce(k[5], k[13], v[5], v[13]); ce(k[5], k[9], v[5], v[9]);
        ce(k[3], k[11], v[3], v[11]); ce(k[7], k[15], v[7], v[15]); ce(k[7], k[11], v[7], v[11]);
        ce(k[3], k[5], v[3], v[5]); ce(k[7], k[9], v[7], v[9]); ce(k[11], k[13], v[11], v[13]);
        ce(k[1], k[2], v[1], v[2]); ce(k[3], k[4], v[3], v[4]); ce(k[5], k[6], v[5], v[6]); ce(k[7], k[8], v[7], v[8]);
        ce(k[9], k[10], v[9], v[10]); ce(k[11], k[12], v[11], v[12]); ce(k[13], k[14], v[13], v[14]);
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (i < len) a[i] = v[i];
}

__global__ void k_cell_order(const int32_t* __restrict__ cs, long long ncell, const int32_t* __restrict__ pid,
                             int32_t* __restrict__ order) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int s = cs[c], e = cs[c + 1];
    const int len = e - s;
    if (len <= 1) return;
    int32_t* a = order + s;
    if (len <= 8) {
        cell_order_net<8>(a, len, pid);
        return;
    }
    if (len <= 16) {
        cell_order_net<16>(a, len, pid);
        return;
    }
    if (len <= 64) {
        for (int i = 1; i < len; ++i) {
            const int32_t v = a[i];
            const int32_t kv = pid[v];
            int j = i - 1;
            while (j >= 0 && pid[a[j]] > kv) {
                a[j + 1] = a[j];
                --j;
            }
            a[j + 1] = v;
        }
        return;
    }
    auto sift = [&](int root, int end) {  // max-heap on pid[a[0, end)]
        while (true) {
            int ch = 2 * root + 1;
            if (ch >= end) return;
            if (ch + 1 < end && pid[a[ch + 1]] > pid[a[ch]]) ++ch;
            if (pid[a[root]] >= pid[a[ch]]) return;
            const int32_t t = a[root];
            a[root] = a[ch];
            a[ch] = t;
            root = ch;
        }
    };
    for (int r = len / 2 - 1; r >= 0; --r) sift(r, len);
    for (int end = len - 1; end > 0; --end) {
        const int32_t t = a[0];
        a[0] = a[end];
        a[end] = t;
        sift(0, end);
    }
}

__global__ void k_occupancy(const int32_t* __restrict__ cs, int nx, int ny, int nz, uint8_t* __restrict__ occ,
                            int ox, int oy, int oz) {
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long nc = (long long)nx * ny * nz;
    if (c >= nc) return;
    if (cs[c + 1] == cs[c]) return;
    int x, y, z;
    idx3(c, ny, nz, x, y, z);
    occ[((long long)(x >> 2) * oy + (y >> 2)) * oz + (z >> 2)] = 1;
}

// AoS host layout <-> SoA device layout
template <class T>
__global__ void k_aos_to_soa(const T* __restrict__ aos, T* __restrict__ pd, long long cap, int32_t* __restrict__ id,
                             long long n, int has_vel, int has_aff) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T* pos = aos;
    const T* vel = aos + 3 * n;
    const T* aff = aos + 6 * n;
    for (int k = 0; k < 3; ++k) pd[k * cap + i] = pos[3 * i + k];
    for (int k = 0; k < 3; ++k) pd[(3 + k) * cap + i] = has_vel ? vel[3 * i + k] : T(0);
    for (int k = 0; k < 9; ++k) pd[(6 + k) * cap + i] = has_aff ? aff[9 * i + k] : T(0);
    id[i] = int32_t(i);
}

template <class T>
__global__ void k_soa_to_aos(const T* __restrict__ pd, long long cap, const int32_t* __restrict__ id,
                             T* __restrict__ aos, long long n) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    long long i = id[k];
    T* pos = aos;
    T* vel = aos + 3 * n;
    T* aff = aos + 6 * n;
    for (int c = 0; c < 3; ++c) pos[3 * i + c] = pd[c * cap + k];
    for (int c = 0; c < 3; ++c) vel[3 * i + c] = pd[(3 + c) * cap + k];
    for (int c = 0; c < 9; ++c) aff[9 * i + c] = pd[(6 + c) * cap + k];
}

// ------------------------------------------------------------ liquid SDF
// LiquidModel<3>::ComputeLiquidPhi (LiquidModel.cpp:540-560) as a gather:
// cell c takes min(|x_c - x_p| - r) over particles p whose Point2Index cell
// lies within +-d of c.  The minimum does not depend on visiting order, so
// the result is bit-identical to the reference.  The window's cells are
// visited in ascending order of a lower bound of what their particles can
// give (the table, own cell first); the walk ends at the first bound above
// the current minimum, since no later cell can lower it.  Inside the liquid
// the cell's own particles already end it.
template <class T>
__global__ void __launch_bounds__(256) k_liquid_phi(GridP<T> g, const int32_t* __restrict__ cs,
                                                    const uint8_t* __restrict__ occ, int ox, int oy, int oz,
                                                    const T* __restrict__ pd, long long cap, T radius, int d0, int d1,
                                                    int d2, const LphiOffset* __restrict__ tab, int ntab,
                                                    T* __restrict__ phi) {
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long nc = (long long)g.nx * g.ny * g.nz;
    if (c >= nc) return;
    int cx, cy, cz;
    idx3(c, g.ny, g.nz, cx, cy, cz);
    const int x0 = max(0, cx - d0), x1 = min(g.nx - 1, cx + d0);
    const int y0 = max(0, cy - d1), y1 = min(g.ny - 1, cy + d1);
    const int z0 = max(0, cz - d2), z1 = min(g.nz - 1, cz + d2);
    bool any = false;
    for (int bx = x0 >> 2; bx <= (x1 >> 2) && !any; ++bx)
        for (int by = y0 >> 2; by <= (y1 >> 2) && !any; ++by)
            for (int bz = z0 >> 2; bz <= (z1 >> 2); ++bz)
                if (occ[((long long)bx * oy + by) * oz + bz]) {
                    any = true;
                    break;
                }
    if (!any) return;
    T cur = phi[c];
    // Index2Point: (index + 0.5) * dx + minCoord
    const T cpx = X<T>::add(X<T>::mul(X<T>::add(T(cx), T(0.5)), g.dx[0]), g.mn[0]);
    const T cpy = X<T>::add(X<T>::mul(X<T>::add(T(cy), T(0.5)), g.dx[1]), g.mn[1]);
    const T cpz = X<T>::add(X<T>::mul(X<T>::add(T(cz), T(0.5)), g.dx[2]), g.mn[2]);
    const T* px = pd;
    const T* py = pd + cap;
    const T* pz = pd + 2 * cap;
    for (int k = 0; k < ntab; ++k) {
        const LphiOffset e = tab[k];
        if (double(cur) < e.lb) break;
        const int wx = cx + (e.off & 255) - 16, wy = cy + ((e.off >> 8) & 255) - 16,
                  wz = cz + ((e.off >> 16) & 255) - 16;
        if (wx < x0 || wx > x1 || wy < y0 || wy > y1 || wz < z0 || wz > z1) continue;
        const long long w = ((long long)wx * g.ny + wy) * g.nz + wz;
        const int s = cs[w], en = cs[w + 1];
        if (s == en) continue;
        // the particles of a cell off the grid's outer layer were sorted
        // into it by their own unclamped Point2Index: all inside the window
        // (and the bound holds for particles clamped into an outer-layer
        // cell: they lie beyond it)
        const bool own = wx > 0 && wx < g.nx - 1 && wy > 0 && wy < g.ny - 1 && wz > 0 && wz < g.nz - 1;
        for (int p = s; p < en; ++p) {
            T qx = px[p], qy = py[p], qz = pz[p];
            if (!own) {
                int tx = cell_trunc(qx, g.mn[0], g.dx[0]);
                int ty = cell_trunc(qy, g.mn[1], g.dx[1]);
                int tz = cell_trunc(qz, g.mn[2], g.dx[2]);
                if (abs(tx - cx) > d0 || abs(ty - cy) > d1 || abs(tz - cz) > d2) continue;
            }
            T dist = X<T>::sqrt(sqnorm3(X<T>::sub(cpx, qx), X<T>::sub(cpy, qy), X<T>::sub(cpz, qz)));
            T ph = X<T>::sub(dist, radius);
            cur = (cur < ph) ? cur : ph;
        }
    }
    phi[c] = cur;
}

// ------------------------------------------------------------------ P2G
constexpr int kTile = 8;

// Per-axis node offsets around the particle's cell for face component a on
// axis i: the quadratic B-spline is non-zero for offsets [-1, 2] along the
// face normal and [-1, 1] across it; the reference's window +-d clips it.
__device__ __forceinline__ int off_lo(int d) { return max(-1, -d); }
__device__ __forceinline__ int off_hi(int i, int a, int d) { return min(i == a ? 2 : 1, d); }

// Quadratic B-spline weights (qweight) and the reference's gradient weights
// (gqweight) of the three nodes around a middle node at signed distance
// t = x - node in [-1/2, 1/2] (grid units): the nodes at -1, 0, +1 sit at
// distances t + 1, t, t - 1, which fall on the outer branch, the inner
// branch and the outer branch of both functions.
template <class T> __device__ __forceinline__ void axis_weights(T t, T w[3], T gw[3]) {
    const T l = T(0.5f) - t, r = T(0.5f) + t;
    w[0] = T(0.5f) * l * l;
    w[1] = T(0.75f) - t * t;
    w[2] = T(0.5f) * r * r;
    gw[0] = -l;
    gw[1] = T(-2.f) * fabs(t);
    gw[2] = -r;
}

// LiquidModel<3>::Particle2Grid accumulation (LiquidModel.cpp:614-701).
// One CTA per 8^3-cell tile.  Thread t owns cells t and t + 256 of the tile;
// for each face component it walks its cell's sorted particles and sums
// their weights and APIC values for the cell's fixed window of nodes (4
// along the component's axis, offsets -1..2; 3 across, offsets -1..1) in
// registers, then adds each window node once into the tile's shared-memory
// accumulators.  The lanes of a warp own distinct cells, so at any step they
// add to distinct nodes.  Finally each touched node goes to global memory
// with one add.  The per-axis weights and C.(x_p - x_node) terms are the
// reference's, rounded the same way; the per-node products are regrouped
// and fused (multiply-add), and particles are summed in another order, so
// P2G matches the reference to rounding, not bit for bit.
// A particle whose own truncated index (cast<Integer>, LiquidModel.cpp:629)
// is not the cell it was sorted into (only outside the grid, where the sort
// key is clamped) adds its window straight to global memory.
template <class T, int A>
__device__ void p2g_particle_global(const GridP<T>& g, const int d[3], const T q[3], const T g3[3], T vel, T C0, T C1,
                                    T C2, T* __restrict__ gw, T* __restrict__ gv) {
    const int hx = g.nx - 1 + (A == 0), hy = g.ny - 1 + (A == 1), hz = g.nz - 1 + (A == 2);
    int ci[3];
    for (int i = 0; i < 3; ++i) ci[i] = int(g3[i]);
    for (int ox = max(-1, -d[0]); ox <= min(A == 0 ? 2 : 1, d[0]); ++ox) {
        const int xi = ci[0] + ox;
        const T cx = (A == 0) ? T(xi) : X<T>::add(T(xi), T(0.5));
        const T e0 = X<T>::sub(g3[0], cx);
        if (xi < 0 || xi > hx || fabs(e0) >= T(1.5f)) continue;
        for (int oy = max(-1, -d[1]); oy <= min(A == 1 ? 2 : 1, d[1]); ++oy) {
            const int yi = ci[1] + oy;
            const T cy = (A == 1) ? T(yi) : X<T>::add(T(yi), T(0.5));
            const T e1 = X<T>::sub(g3[1], cy);
            if (yi < 0 || yi > hy || fabs(e1) >= T(1.5f)) continue;
            const T wxy = X<T>::mul(qweight(e0), qweight(e1));
            const T t0 = X<T>::mul(C0, X<T>::sub(q[0], X<T>::add(X<T>::mul(cx, g.dx[0]), g.mn[0])));
            const T t1 = X<T>::mul(C1, X<T>::sub(q[1], X<T>::add(X<T>::mul(cy, g.dx[1]), g.mn[1])));
            for (int oz = max(-1, -d[2]); oz <= min(A == 2 ? 2 : 1, d[2]); ++oz) {
                const int zi = ci[2] + oz;
                const T cz = (A == 2) ? T(zi) : X<T>::add(T(zi), T(0.5));
                const T e2 = X<T>::sub(g3[2], cz);
                if (zi < 0 || zi > hz || fabs(e2) >= T(1.5f)) continue;
                const T weight = X<T>::mul(wxy, qweight(e2));
                const T t2 = X<T>::mul(C2, X<T>::sub(q[2], X<T>::add(X<T>::mul(cz, g.dx[2]), g.mn[2])));
                const T val = X<T>::mul(weight, X<T>::add(vel, X<T>::add(t0, X<T>::add(t1, t2))));
                const long long gi = ((long long)xi * (g.ny + (A == 1)) + yi) * (g.nz + (A == 2)) + zi;
                atomicAdd(&gw[gi], weight);
                atomicAdd(&gv[gi], val);
            }
        }
    }
}

// The cell-sorted particle state as P2G reads it: the positions of sorted
// index k in pos (rows 0-2, stride cap), the other 12 scalars at row r of
// rest, index order ? order[k] : k (order: the sort's permutation while it
// is deferred).
template <class T> struct PView {
    const T* pos;
    const T* rest;
    const int32_t* order;
    long long cap;
};

template <class T> struct P2GOut {
    T* v[3];
    T* w[3];
};

__host__ __device__ constexpr int p2g_region(int a) {
    return (kTile + 2 + (a == 0)) * (kTile + 2 + (a == 1)) * (kTile + 2 + (a == 2));
}

// Staged particle records of the P2G warp loop (values of T), two per
// particle:
//   A (kP2GRecA values, 16-byte aligned: the lanes read wf and tf as vectors)
//     [0, 12)   wf[a][4]: face weights of component a along its own axis,
//               window slots -1..2 (node = cell + slot)
//     [12, 24)  tf[a][4] = C_aa * (x_a - face node a)
//     [24, 28)  unused (padding to 16 bytes)
//   B (kP2GRecB values, odd stride: the staging lanes' stores fall in
//     distinct banks)
//     [0, 27)   W[l], column l = 9a + 3s + t of the warp loop: the product of
//               the two cell-centre weights across component a (slot s on its
//               first other axis, t on the second; node centre = cell + slot + 0.5)
//     [27, 54)  B[l] = v_a + C_ab (x_b - centre b) + C_ac (x_c - centre c)
// The weights are the quadratic B-spline's in closed form around the
// particle's middle node (axis_weights); a node outside the reference's
// window (+-d) gets 0, as does a node at |e| >= 1.5 by the formula itself.
constexpr int kP2GRecA = 28;
constexpr int kP2GRecB = 55;
constexpr int kP2GWarps = 8;
constexpr int kP2GChunk = 16;  // particles staged at a time per warp
constexpr int kP2GStage = kP2GChunk * (kP2GRecA + kP2GRecB);  // values per warp

__device__ __forceinline__ void p2g_other_axes(int a, int& b, int& c) {
    b = (a == 0) ? 1 : 0;
    c = (a == 2) ? 1 : 2;
}

__device__ __forceinline__ void load4(const float* p, float v[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
}
__device__ __forceinline__ void load4(const double* p, double v[4]) {
    const double2 t0 = reinterpret_cast<const double2*>(p)[0], t1 = reinterpret_cast<const double2*>(p)[1];
    v[0] = t0.x;
    v[1] = t0.y;
    v[2] = t1.x;
    v[3] = t1.y;
}
__device__ __forceinline__ void store4(float* p, const float v[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store4(double* p, const double v[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// Computes the records of one particle (one lane per particle) and returns
// the z offset of its cell in the row, or -1 when its own truncated index
// (cast<Integer>, LiquidModel.cpp:629) is not the cell it was sorted into,
// or its grid coordinate is negative (both only outside the grid, where the
// sort key is clamped): such a particle is listed for k_p2g_overflow.
template <class T>
__device__ int p2g_stage(const GridP<T>& g, int d0, int d1, int d2, const PView<T>& pv, long long p, int rx, int ry,
                         int z0, int zend, T* ra, T* rb, int* __restrict__ ov_count, int32_t* __restrict__ ov_list) {
    const long long cap = pv.cap;
    const T q[3] = {pv.pos[p], pv.pos[cap + p], pv.pos[2 * cap + p]};
    T g3[3];
    int ci[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        // cwiseQuotient as a multiply (P2G equals the reference up to rounding; a particle whose cell then
        // differs from its sort key's takes the overflow path, which divides)
        g3[i] = (q[i] - g.mn[i]) * g.idx[i];
        ci[i] = int(g3[i]);  // cast<Integer>
    }
    if (ci[0] != rx || ci[1] != ry || ci[2] < z0 || ci[2] >= zend ||
        !(g3[0] >= T(0) && g3[1] >= T(0) && g3[2] >= T(0))) {
        ov_list[atomicAdd(ov_count, 1)] = int32_t(p);
        return -1;
    }
    const long long ps = pv.order ? (long long)pv.order[p] : p;
    T C[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) C[k] = pv.rest[(6 + k) * cap + ps];  // column-major: C[3a + i] = C(i, a)
    const int dd[3] = {d0, d1, d2};
    T wc[3][3], tc[3][2][3];  // centre weights per axis; C_ab (x_b - centre) per component and other axis
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T cb = T(ci[i]);  // integer grid coordinates are exact in T
        const T f = g3[i] - cb;  // exact, in [0, 1)
        const bool up = f >= T(0.5f);
        T w3[3], gu[3];
        axis_weights(g3[i] - (up ? cb + T(1) : cb), w3, gu);  // face nodes: middle node = nearest integer
        T wf[4], tf[4];
#pragma unroll
        for (int s2 = 0; s2 < 4; ++s2) {  // slot s2 = offset + 1 from the cell
            const int o = s2 - 1;
            T wv = up ? (s2 >= 1 ? w3[s2 - 1] : T(0)) : (s2 <= 2 ? w3[s2] : T(0));
            if (o < -dd[i] || o > dd[i]) wv = T(0);
            wf[s2] = wv;
            tf[s2] = C[4 * i] * (q[i] - fma(cb + T(o), g.dx[i], g.mn[i]));  // C(i, i)
        }
        store4(ra + 4 * i, wf);
        store4(ra + 12 + 4 * i, tf);
        axis_weights(f - T(0.5f), wc[i], gu);  // cell-centre nodes: middle node = this cell's centre
#pragma unroll
        for (int s2 = 0; s2 < 3; ++s2) {
            const int o = s2 - 1;
            if (o < -dd[i] || o > dd[i]) wc[i][s2] = T(0);
            const T dc = q[i] - fma(cb + T(o) + T(0.5f), g.dx[i], g.mn[i]);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a == i) continue;
                int b, c;
                p2g_other_axes(a, b, c);
                tc[a][b == i ? 0 : 1][s2] = C[3 * a + i] * dc;
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int b, c;
        p2g_other_axes(a, b, c);
        const T va = pv.rest[(3 + a) * cap + ps];
#pragma unroll
        for (int s2 = 0; s2 < 3; ++s2)
#pragma unroll
            for (int t2 = 0; t2 < 3; ++t2) {
                const int l = 9 * a + 3 * s2 + t2;
                rb[l] = wc[b][s2] * wc[c][t2];
                rb[27 + l] = va + tc[a][0][s2] + tc[a][1][t2];
            }
    }
    return ci[2] - z0;
}

// LiquidModel<3>::Particle2Grid accumulation (LiquidModel.cpp:614-701).
// One CTA per 8^3-cell tile, shared-memory accumulators for the tile's
// window nodes of the three face components.  A warp takes whole z rows of
// the tile: the particles of a row are contiguous in the sorted order.  The
// row's particles are staged 16 at a time (one lane per particle computes
// its per-axis weights and C.(x_p - x_node) terms once, for all three
// components, and the per-column products below), then the warp walks them
// run by run (a ballot over the staged cell offsets marks where each cell's
// particles start), two at a time within a run: lane l < 27 owns one
// column of 4 window nodes of one component (component l / 9, along that
// component's own axis; the 3 x 3 columns across it) and sums the weights
// and APIC values of the current cell's particles in registers.  When the
// walk reaches the next cell each lane adds its 4 nodes once into the
// tile's accumulators; at the end every touched node goes to global memory
// with one add.  The per-axis weights are the reference's B-spline in closed
// form; the per-node products are regrouped and fused and particles are
// summed in another order, so P2G matches the reference to rounding, not
// bit for bit.  No per-particle global atomics.
template <class T>
__global__ void __launch_bounds__(kP2GWarps * 32, sizeof(T) == 4 ? 3 : 1) k_p2g(GridP<T> g, const int32_t* __restrict__ cs, PView<T> pv,
                                                        int d0, int d1, int d2, P2GOut<T> out,
                                                        int* __restrict__ ov_count, int32_t* __restrict__ ov_list) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* acc = reinterpret_cast<T*>(smem_raw);
    __shared__ int any;
    const int x0 = blockIdx.z * kTile, y0 = blockIdx.y * kTile, z0 = blockIdx.x * kTile;
    const int zend = min(z0 + kTile, g.nz);
    const int R0 = p2g_region(0), R1 = p2g_region(1), R2 = p2g_region(2);
    const int ntot = 2 * (R0 + R1 + R2);
    static_assert(kP2GStage % 4 == 0 && kP2GRecA % 4 == 0, "records stay 16-byte aligned");
    T* stA = acc + ntot + (threadIdx.x >> 5) * kP2GStage;  // ntot is a multiple of 4
    T* stB = stA + kP2GChunk * kP2GRecA;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    if (threadIdx.x < kTile * kTile) {  // row (x0 + t / 8, y0 + t % 8)
        const int rx = x0 + (threadIdx.x >> 3), ry = y0 + (threadIdx.x & 7);
        if (rx < g.nx && ry < g.ny) {
            const long long c = ((long long)rx * g.ny + ry) * g.nz + z0;
            if (cs[c + (zend - z0)] > cs[c]) any = 1;
        }
    }
    __syncthreads();
    if (!any) return;
    for (int i = threadIdx.x; i < ntot; i += blockDim.x) acc[i] = T(0);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // this lane's column: component a, centre slots s (axis b) and t (axis c), face slots k along a
    const int a = lane / 9, s = (lane % 9) / 3, t = lane % 3;
    int b = 0, c = 0;
    p2g_other_axes(a < 3 ? a : 0, b, c);
    const bool col = lane < 27;
    const int ac = col ? a : 0;
    const int ey = kTile + 2 + (ac == 1), ez = kTile + 2 + (ac == 2);
    const int astride = (ac == 0) ? ey * ez : (ac == 1) ? ez : 1;
    // the column's first node relative to its cell, per axis (slot - 1, plus 1 for the halo): face slot 0
    // along a, centre slot s along b, t along c (b < c)
    const int ox = (ac == 0) ? 0 : s;
    const int oy = (ac == 1) ? 0 : (b == 1 ? s : t);
    const int oz = (ac == 2) ? 0 : t;
    // component a's weight and value accumulators: [w_0 | v_0 | w_1 | v_1 | w_2 | v_2]
    T* aw_s = acc + ((ac == 1) ? 2 * R0 : (ac == 2) ? 2 * (R0 + R1) : 0);
    T* av_s = aw_s + ((ac == 1) ? R1 : (ac == 2) ? R2 : R0);
    const int lw = col ? lane : 0;  // record offsets of this lane's column
    for (int row = warp; row < kTile * kTile; row += kP2GWarps) {
        const int rx = x0 + (row >> 3), ry = y0 + (row & 7);
        if (rx >= g.nx || ry >= g.ny) continue;
        const long long c0 = ((long long)rx * g.ny + ry) * g.nz + z0;
        const int pbeg = cs[c0], pend = cs[c0 + (zend - z0)];
        if (pend == pbeg) continue;
        int cur = -1;  // z offset of the cell being summed
        T aw[4] = {T(0), T(0), T(0), T(0)}, av[4] = {T(0), T(0), T(0), T(0)};
        auto flush = [&]() {
            if (cur < 0 || !col) return;
            // window node of slot (k, s, t) of cell (rx, ry, z0 + cur), local to the tile region
            const int base = (((rx - x0) + ox) * ey + (ry - y0) + oy) * ez + cur + oz;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                atomicAdd(&aw_s[base + k * astride], aw[k]);
                atomicAdd(&av_s[base + k * astride], av[k]);
                aw[k] = T(0);
                av[k] = T(0);
            }
        };
        auto add = [&](int j) {
            T wf[4], tf[4];
            load4(stA + j * kP2GRecA + 4 * ac, wf);
            load4(stA + j * kP2GRecA + 12 + 4 * ac, tf);
            const T W = stB[j * kP2GRecB + lw], B = stB[j * kP2GRecB + 27 + lw];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const T w = W * wf[k];
                aw[k] += w;
                av[k] = fma(w, B + tf[k], av[k]);
            }
        };
        for (int chunk = pbeg; chunk < pend; chunk += kP2GChunk) {
            const int n = min(kP2GChunk, pend - chunk);
            __syncwarp();
            int zo = -1;  // this lane's particle: z offset of its cell in the row (-1: overflow)
            if (lane < n)
                zo = p2g_stage<T>(g, d0, d1, d2, pv, chunk + lane, rx, ry, z0, zend, stA + lane * kP2GRecA,
                                  stB + lane * kP2GRecB, ov_count, ov_list);
            __syncwarp();
            // the chunk's runs of particles of one cell (sorted order: a cell's particles are contiguous);
            // every lane walks the same runs
            const int zprev = __shfl_up_sync(0xffffffffu, zo, 1);
            unsigned starts = __ballot_sync(0xffffffffu, lane < n && (lane == 0 || zprev != zo));
            while (starts) {
                const int sb = __ffs(starts) - 1;
                starts &= starts - 1;
                const int se = starts ? __ffs(starts) - 1 : n;
                const int run = __shfl_sync(0xffffffffu, zo, sb);
                if (run < 0) continue;  // overflow particles: k_p2g_overflow adds them
                if (run != cur) {
                    flush();
                    cur = run;
                }
                if (col) {
                    int j = sb;
                    for (; j + 1 < se; j += 2) {
                        add(j);
                        add(j + 1);
                    }
                    if (j < se) add(j);
                }
            }
        }
        flush();
    }
    __syncthreads();
    // flush: one global add per touched node
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2) {
        const int fy2 = kTile + 2 + (a2 == 1), fz2 = kTile + 2 + (a2 == 2);
        const int R = (a2 == 0) ? R0 : (a2 == 1) ? R1 : R2;
        const T* sw_a = acc + ((a2 == 1) ? 2 * R0 : (a2 == 2) ? 2 * (R0 + R1) : 0);
        const T* sv_a = sw_a + R;
        const int fy = g.ny + (a2 == 1), fz = g.nz + (a2 == 2);
        const int hx = g.nx - 1 + (a2 == 0);
        for (int i = threadIdx.x; i < R; i += blockDim.x) {
            T wv = sw_a[i], vv = sv_a[i];
            if (wv == T(0) && vv == T(0)) continue;
            int lz = i % fz2, ly = (i / fz2) % fy2, lx = i / (fy2 * fz2);
            int xi = x0 - 1 + lx, yi = y0 - 1 + ly, zi = z0 - 1 + lz;
            if (xi < 0 || xi > hx || yi < 0 || yi >= fy || zi < 0 || zi >= fz) continue;
            long long gi = ((long long)xi * fy + yi) * fz + zi;
            atomicAdd(&out.w[a2][gi], wv);
            atomicAdd(&out.v[a2][gi], vv);
        }
    }
}

// The particles k_p2g listed (outside the cell they were sorted into: off
// the grid) add their windows straight to global memory.
template <class T>
__global__ void k_p2g_overflow(GridP<T> g, PView<T> pv, int d0, int d1, int d2, P2GOut<T> out,
                               const int* __restrict__ ov_count, const int32_t* __restrict__ ov_list) {
    const int n = *ov_count;
    const int d[3] = {d0, d1, d2};
    const long long cap = pv.cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const long long p = ov_list[i];
        const long long ps = pv.order ? (long long)pv.order[p] : p;
        const T q[3] = {pv.pos[p], pv.pos[cap + p], pv.pos[2 * cap + p]};
        T g3[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) g3[k] = X<T>::div(X<T>::sub(q[k], g.mn[k]), g.dx[k]);
        T C[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) C[k] = pv.rest[(6 + k) * cap + ps];
        p2g_particle_global<T, 0>(g, d, q, g3, pv.rest[3 * cap + ps], C[0], C[1], C[2], out.w[0], out.v[0]);
        p2g_particle_global<T, 1>(g, d, q, g3, pv.rest[4 * cap + ps], C[3], C[4], C[5], out.w[1], out.v[1]);
        p2g_particle_global<T, 2>(g, d, q, g3, pv.rest[5 * cap + ps], C[6], C[7], C[8], out.w[2], out.v[2]);
    }
}

// v = !IsSmall(w) ? v / w : 0 (LiquidModel.cpp:703-720), optionally fused
// with ApplyGravity (LiquidModel.cpp:899-910) on the y component.
template <class T>
__global__ void k_p2g_normalize(T* __restrict__ v, const T* __restrict__ w, int fx, int fy, int fz, int gravity,
                                T gdt, int nx, int ny, int nz) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)fx * fy * fz;
    if (i >= n) return;
    T wv = w[i];
    T r = !is_small(wv) ? X<T>::div(v[i], wv) : T(0);
    if (gravity) {
        int x, y, z;
        idx3(i, fy, fz, x, y, z);
        if (x >= 1 && x < nx - 1 && y >= 1 && y < ny && z >= 1 && z < nz - 1) r = X<T>::add(r, gdt);
    }
    v[i] = r;
}

// ------------------------------------------------------------ G2P + advect
template <class T> struct SolidView {
    const T* phi;  // (nx+1)(ny+1)(nz+1)
};

template <class T> __device__ __forceinline__ bool in_grid(const GridP<T>& g, T x, T y, T z) {
    return g.mn[0] <= x && g.mn[1] <= y && g.mn[2] <= z && x <= g.mx[0] && y <= g.mx[1] && z <= g.mx[2];
}

// Grid<3>::GetSolidPhi for a point inside the grid (Grid.cpp:144-154)
// EXACT = false (the mixed-precision gather's advection): the grid
// coordinates by a multiply with 1 / dx, equal up to rounding.
template <class T, bool EXACT = true>
__device__ T solid_phi_in(const GridP<T>& g, const T* sp, T x, T y, T z) {
    T lx, ly, lz;
    if constexpr (EXACT) {
        lx = X<T>::div(X<T>::sub(x, g.mn[0]), g.dx[0]);
        ly = X<T>::div(X<T>::sub(y, g.mn[1]), g.dx[1]);
        lz = X<T>::div(X<T>::sub(z, g.mn[2]), g.dx[2]);
    } else {
        lx = (x - g.mn[0]) * g.idx[0];
        ly = (y - g.mn[1]) * g.idx[1];
        lz = (z - g.mn[2]) * g.idx[2];
    }
    int xi, yi, zi;
    T fx, fy, fz;
    barycentric(lx, 0, g.nx + 1, xi, fx);
    barycentric(ly, 0, g.ny + 1, yi, fy);
    barycentric(lz, 0, g.nz + 1, zi, fz);
    const long long sy = g.nz + 1, sx = (long long)(g.ny + 1) * (g.nz + 1);
    const T* b = sp + xi * sx + yi * sy + zi;
    return trilerp(b[0], b[sx], b[sy], b[sx + sy], b[1], b[sx + 1], b[sy + 1], b[sx + sy + 1], fx, fy, fz);
}

template <class T> __device__ void clamp_to_valid(const GridP<T>& g, T& x, T& y, T& z) {
    x = clampS(x, X<T>::add(g.mn[0], g.dx[0]), X<T>::sub(g.mx[0], g.dx[0]));
    y = clampS(y, X<T>::add(g.mn[1], g.dx[1]), X<T>::sub(g.mx[1], g.dx[1]));
    z = clampS(z, X<T>::add(g.mn[2], g.dx[2]), X<T>::sub(g.mx[2], g.dx[2]));
}

template <class T> __device__ void normalized3(T v0, T v1, T v2, T out[3]) {
    T n2 = sqnorm3(v0, v1, v2);
    if (n2 > T(0)) {
        T n = X<T>::sqrt(n2);
        out[0] = X<T>::div(v0, n);
        out[1] = X<T>::div(v1, n);
        out[2] = X<T>::div(v2, n);
    } else {
        out[0] = v0;
        out[1] = v1;
        out[2] = v2;
    }
}

// GetSolidGradient at a point whose +-eps neighbours are inside the grid
template <class T> __device__ void solid_grad_inner(const GridP<T>& g, const T* sp, T x, T y, T z, T out[3]) {
    const T eps = T(1e-4);
    T left = solid_phi_in(g, sp, X<T>::sub(x, eps), y, z);
    T right = solid_phi_in(g, sp, X<T>::add(x, eps), y, z);
    T bottom = solid_phi_in(g, sp, x, X<T>::sub(y, eps), z);
    T top = solid_phi_in(g, sp, x, X<T>::add(y, eps), z);
    T front = solid_phi_in(g, sp, x, y, X<T>::add(z, eps));
    T back = solid_phi_in(g, sp, x, y, X<T>::sub(z, eps));
    T dv = T(__dmul_rn(2.0, double(eps)));
    normalized3(X<T>::div(X<T>::sub(right, left), dv), X<T>::div(X<T>::sub(top, bottom), dv),
                X<T>::div(X<T>::sub(front, back), dv), out);
}

// Grid<3>::GetSolidPhi (Grid.cpp:128-155) for any point
template <class T> __device__ T solid_phi_at(const GridP<T>& g, const T* sp, T x, T y, T z) {
    if (in_grid(g, x, y, z)) return solid_phi_in(g, sp, x, y, z);
    T vx = x, vy = y, vz = z;
    clamp_to_valid(g, vx, vy, vz);
    T gr[3];
    solid_grad_inner(g, sp, vx, vy, vz, gr);
    T r = solid_phi_in(g, sp, vx, vy, vz);
    r = X<T>::add(r, X<T>::mul(gr[0], X<T>::sub(x, vx)));
    r = X<T>::add(r, X<T>::mul(gr[1], X<T>::sub(y, vy)));
    r = X<T>::add(r, X<T>::mul(gr[2], X<T>::sub(z, vz)));
    return r;
}

// Grid<3>::GetSolidGradient (Grid.cpp:175-192) for any point
template <class T> __device__ void solid_grad_at(const GridP<T>& g, const T* sp, T x, T y, T z, T out[3]) {
    if (!in_grid(g, x, y, z)) {
        clamp_to_valid(g, x, y, z);
        solid_grad_inner(g, sp, x, y, z, out);
        return;
    }
    const T eps = T(1e-4);
    T left = solid_phi_at(g, sp, X<T>::sub(x, eps), y, z);
    T right = solid_phi_at(g, sp, X<T>::add(x, eps), y, z);
    T bottom = solid_phi_at(g, sp, x, X<T>::sub(y, eps), z);
    T top = solid_phi_at(g, sp, x, X<T>::add(y, eps), z);
    T front = solid_phi_at(g, sp, x, y, X<T>::add(z, eps));
    T back = solid_phi_at(g, sp, x, y, X<T>::sub(z, eps));
    T dv = T(__dmul_rn(2.0, double(eps)));
    normalized3(X<T>::div(X<T>::sub(right, left), dv), X<T>::div(X<T>::sub(top, bottom), dv),
                X<T>::div(X<T>::sub(front, back), dv), out);
}

// Gather of one face component (LiquidModel.cpp:738-761 and its y/z twins).
// On each axis the window nodes that contribute (offset inside the clipped
// window, |e| < 1.5, node inside the face grid) are one run of at most 3
// consecutive nodes; the sum visits that run in the reference's ascending
// order.  The x.y weight products are formed once per (x, y) pair: the same
// products as the reference's (wX * wY) * wZ, so every term is bit-identical.
// FACTORED (the mixed-precision handles): the weights are separable, so the
// sums are taken axis by axis -- per (x, y) column S = sum wZ v and
// T = sum gZ v, then per x A = sum wY S, B = sum gY S, D = sum wY T, then
// v = sum wX A, C = (sum gX A, sum wX B, sum wX D) -- with fused
// multiply-adds: about a third of the arithmetic, the same value up to
// rounding.
// Where a gather reads the face velocities of one component: the global
// array (origin 0, the face grid's extents) or a tile's staged copy in
// shared memory (origin one node before the tile, the region's extents).
template <class T> struct VSrc {
    const T* v;
    int ox, oy, oz;
    long long fy, fz;
};

template <class T, int A, bool FACTORED>
__device__ __forceinline__ void g2p_component(const GridP<T>& g, const int d[3], const T g3[3], const int ci[3],
                                              const VSrc<T> vs, T& velA, T col[3]) {
    const int hmax[3] = {g.nx - 1 + (A == 0), g.ny - 1 + (A == 1), g.nz - 1 + (A == 2)};
    T ew[3][3], eg[3][3];
    int first[3], cnt[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int lo = off_lo(d[i]), hi = off_hi(i, A, d[i]);
        int kb = 4, ke = -1;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int o = k - 1;
            const int node = ci[i] + o;
            const T c = (i == A) ? T(node) : X<T>::add(T(node), T(0.5));
            const T e = X<T>::sub(g3[i], c);
            if (o >= lo && o <= hi && !(fabs(e) >= T(1.5f)) && node >= 0 && node <= hmax[i]) {
                kb = min(kb, k);
                ke = k;
            }
        }
        first[i] = ci[i] + kb - 1;
        cnt[i] = max(ke - kb + 1, 0);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int node = first[i] + j;
            const T c = (i == A) ? T(node) : X<T>::add(T(node), T(0.5));
            const T e = X<T>::sub(g3[i], c);
            ew[i][j] = j < cnt[i] ? qweight(e) : T(0);
            eg[i][j] = j < cnt[i] ? gqweight(e) : T(0);
        }
    }
    if constexpr (FACTORED) {
#pragma unroll
        for (int jx = 0; jx < 3; ++jx) {
            if (jx >= cnt[0]) break;
            T a = T(0), b = T(0), dd = T(0);
#pragma unroll
            for (int jy = 0; jy < 3; ++jy) {
                if (jy >= cnt[1]) break;
                const T* row = vs.v + ((long long)(first[0] + jx - vs.ox) * vs.fy + (first[1] + jy - vs.oy)) * vs.fz +
                               (first[2] - vs.oz);
                T s = T(0), t = T(0);
#pragma unroll
                for (int jz = 0; jz < 3; ++jz) {
                    if (jz >= cnt[2]) break;
                    const T val = row[jz];
                    s = fma(ew[2][jz], val, s);
                    t = fma(eg[2][jz], val, t);
                }
                a = fma(ew[1][jy], s, a);
                b = fma(eg[1][jy], s, b);
                dd = fma(ew[1][jy], t, dd);
            }
            velA = fma(ew[0][jx], a, velA);
            col[0] = fma(eg[0][jx], a, col[0]);
            col[1] = fma(ew[0][jx], b, col[1]);
            col[2] = fma(ew[0][jx], dd, col[2]);
        }
    } else {
#pragma unroll
    for (int jx = 0; jx < 3; ++jx) {
        if (jx >= cnt[0]) break;
        const T wX = ew[0][jx], gX = eg[0][jx];
#pragma unroll
        for (int jy = 0; jy < 3; ++jy) {
            if (jy >= cnt[1]) break;
            const T wY = ew[1][jy], gY = eg[1][jy];
            const T wXY = X<T>::mul(wX, wY), gXwY = X<T>::mul(gX, wY), wXgY = X<T>::mul(wX, gY);
            const T* row = vs.v + ((long long)(first[0] + jx - vs.ox) * vs.fy + (first[1] + jy - vs.oy)) * vs.fz +
                               (first[2] - vs.oz);
#pragma unroll
            for (int jz = 0; jz < 3; ++jz) {
                if (jz >= cnt[2]) break;
                const T wZ = ew[2][jz], gZ = eg[2][jz];
                const T weight = X<T>::mul(wXY, wZ);
                const T gw0 = X<T>::mul(gXwY, wZ);
                const T gw1 = X<T>::mul(wXgY, wZ);
                const T gw2 = X<T>::mul(wXY, gZ);
                const T val = row[jz];
                velA = X<T>::add(velA, X<T>::mul(val, weight));
                col[0] = X<T>::add(col[0], X<T>::mul(val, gw0));
                col[1] = X<T>::add(col[1], X<T>::mul(val, gw1));
                col[2] = X<T>::add(col[2], X<T>::mul(val, gw2));
            }
        }
    }
    }
}

// Factored gather (mixed precision) of a particle whose truncated cell ci
// lies in the staged tile, at least one cell away from the grid's faces,
// with a window of +-2 or more (every window node then exists and lies in
// the reference's window).  Per axis the particle has one window for face
// nodes (middle node = the nearest integer coordinate) and one for cell
// centres (middle node = the centre of ci), each three nodes wide; the
// weights of both are formed once and shared by the three components (the
// face window on a component's own axis, the centre window across it).  The
// staged region holds every window node of a particle of the tile, so the
// loads need no test.  The same sums as the factored path of
// g2p_component, up to rounding.
template <class T, int A>
__device__ __forceinline__ void g2p_staged_component(const T wf[3][3], const T gf[3][3], const T wc[3][3],
                                                     const T gc[3][3], const int mf[3], const int ci[3],
                                                     const VSrc<T>& vs, T& velA, T col[3]) {
    const int bx = ((A == 0) ? mf[0] : ci[0]) - 1, by = ((A == 1) ? mf[1] : ci[1]) - 1,
              bz = ((A == 2) ? mf[2] : ci[2]) - 1;
    const T* wx = (A == 0) ? wf[0] : wc[0];
    const T* gx = (A == 0) ? gf[0] : gc[0];
    const T* wy = (A == 1) ? wf[1] : wc[1];
    const T* gy = (A == 1) ? gf[1] : gc[1];
    const T* wz = (A == 2) ? wf[2] : wc[2];
    const T* gz = (A == 2) ? gf[2] : gc[2];
    const T* base = vs.v + ((long long)(bx - vs.ox) * vs.fy + (by - vs.oy)) * vs.fz + (bz - vs.oz);
#pragma unroll
    for (int jx = 0; jx < 3; ++jx) {
        T a = T(0), b = T(0), dd = T(0);
#pragma unroll
        for (int jy = 0; jy < 3; ++jy) {
            const T* row = base + ((long long)jx * vs.fy + jy) * vs.fz;
            T s = T(0), t = T(0);
#pragma unroll
            for (int jz = 0; jz < 3; ++jz) {
                const T val = row[jz];
                s = fma(wz[jz], val, s);
                t = fma(gz[jz], val, t);
            }
            a = fma(wy[jy], s, a);
            b = fma(gy[jy], s, b);
            dd = fma(wy[jy], t, dd);
        }
        velA = fma(wx[jx], a, velA);
        col[0] = fma(gx[jx], a, col[0]);
        col[1] = fma(wx[jx], b, col[1]);
        col[2] = fma(wx[jx], dd, col[2]);
    }
}

template <class T>
__device__ __forceinline__ void g2p_staged_factored(const GridP<T>& g, const int d[3], const T g3[3], const int ci[3],
                                                    const VSrc<T> src[3], T vel[3], T C[9]) {
    T wf[3][3], gf[3][3], wc[3][3], gc[3][3];
    int mf[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T f = g3[i] - T(ci[i]);  // exact: g3 and ci are within one unit
        const int up = f >= T(0.5f);
        mf[i] = ci[i] + up;
        axis_weights(g3[i] - T(mf[i]), wf[i], gf[i]);
        axis_weights(f - T(0.5f), wc[i], gc[i]);
    }
    g2p_staged_component<T, 0>(wf, gf, wc, gc, mf, ci, src[0], vel[0], &C[0]);
    g2p_staged_component<T, 1>(wf, gf, wc, gc, mf, ci, src[1], vel[1], &C[3]);
    g2p_staged_component<T, 2>(wf, gf, wc, gc, mf, ci, src[2], vel[2], &C[6]);
}

// The factored gather of the particles the staged closed-form path does not
// take (near the grid's faces, off the tile, or a window below +-2), kept
// out of line so that its registers do not weigh on the common path.
template <class T>
__device__ __noinline__ void g2p_general_factored(const GridP<T>& g, const int d[3], const T g3[3], const int ci[3],
                                                  const VSrc<T> src[3], T vel[3], T C[9]) {
    g2p_component<T, 0, true>(g, d, g3, ci, src[0], vel[0], &C[0]);
    g2p_component<T, 1, true>(g, d, g3, ci, src[1], vel[1], &C[3]);
    g2p_component<T, 2, true>(g, d, g3, ci, src[2], vel[2], &C[6]);
}

// One particle of LiquidModel<3>::Grid2Particle (LiquidModel.cpp:724-823)
// fused with AdvectParticle (LiquidModel.cpp:913-935) and the next step's
// cell key.  The face velocities come from the sources the caller picks
// for the particle's truncated cell ci (staged in shared memory when ci lies
// in the tile -- pick returns true -- global memory otherwise).
template <class T, bool FACTORED, class PickSrc>
__device__ __forceinline__ void g2p_particle(const GridP<T>& g, T* __restrict__ pd, long long cap, long long i,
                                             const int d[3], int do_g2p, int do_advect, T dt,
                                             const T* __restrict__ sp, uint32_t* __restrict__ keys,
                                             int32_t* __restrict__ vals, PickSrc pick) {
    T q[3] = {pd[i], pd[cap + i], pd[2 * cap + i]};  // (the positions are rows 0-2 of pd also while the sort's
                                                     // permutation waits: pd is then the sorted buffer)
    T vel[3];
    if (do_g2p) {
        T g3[3];
        int ci[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            // the factored sums equal the reference's up to rounding anyway: a multiply for the divide
            g3[k] = FACTORED ? (q[k] - g.mn[k]) * g.idx[k] : X<T>::div(X<T>::sub(q[k], g.mn[k]), g.dx[k]);
            ci[k] = int(g3[k]);
        }
        T C[9];
        vel[0] = vel[1] = vel[2] = T(0);
#pragma unroll
        for (int k = 0; k < 9; ++k) C[k] = T(0);
        VSrc<T> src[3];
        const bool staged = pick(ci, src);
        // the staged closed-form path: ci >= 1 (so g3 >= 0 and ci is the floor) and ci <= n - 2 on every
        // axis with a window of +-2 or more; anything else takes the general path
        const bool full = d[0] >= 2 && d[1] >= 2 && d[2] >= 2 && ci[0] >= 1 && ci[0] <= g.nx - 2 && ci[1] >= 1 &&
                          ci[1] <= g.ny - 2 && ci[2] >= 1 && ci[2] <= g.nz - 2;
        if (FACTORED && staged && full) {
            g2p_staged_factored<T>(g, d, g3, ci, src, vel, C);
        } else if constexpr (FACTORED) {
            g2p_general_factored<T>(g, d, g3, ci, src, vel, C);  // out of line: the rare particles
        } else {
            g2p_component<T, 0, FACTORED>(g, d, g3, ci, src[0], vel[0], &C[0]);
            g2p_component<T, 1, FACTORED>(g, d, g3, ci, src[1], vel[1], &C[3]);
            g2p_component<T, 2, FACTORED>(g, d, g3, ci, src[2], vel[2], &C[6]);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) pd[(3 + k) * cap + i] = vel[k];
#pragma unroll
        for (int k = 0; k < 9; ++k) pd[(6 + k) * cap + i] = C[k];
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) vel[k] = pd[(3 + k) * cap + i];
    }
    if (do_advect) {
#pragma unroll
        for (int k = 0; k < 3; ++k) q[k] = X<T>::add(q[k], X<T>::mul(vel[k], dt));
        T sphi;
        if (FACTORED && in_grid(g, q[0], q[1], q[2]))
            sphi = solid_phi_in<T, false>(g, sp, q[0], q[1], q[2]);
        else
            sphi = solid_phi_at(g, sp, q[0], q[1], q[2]);
        if (sphi < T(0)) {
            T gr[3];
            solid_grad_at(g, sp, q[0], q[1], q[2], gr);
            T s = X<T>::add(sphi, eps8<T>());
#pragma unroll
            for (int k = 0; k < 3; ++k) q[k] = X<T>::sub(q[k], X<T>::mul(s, gr[k]));
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) pd[k * cap + i] = q[k];
        keys[i] = cell_key(g, q[0], q[1], q[2]);
        vals[i] = int32_t(i);
    }
}

template <class T> __device__ __forceinline__ void global_sources(const GridP<T>& g, const T* vx, const T* vy,
                                                                  const T* vz, VSrc<T> src[3]) {
    src[0] = VSrc<T>{vx, 0, 0, 0, g.ny, g.nz};
    src[1] = VSrc<T>{vy, 0, 0, 0, g.ny + 1, g.nz};
    src[2] = VSrc<T>{vz, 0, 0, 0, g.ny, g.nz + 1};
}

// One thread per particle, face velocities from global memory (the
// advection alone, and any particle order).
template <class T, bool FACTORED>
__global__ void __launch_bounds__(256) k_g2p(GridP<T> g, T* __restrict__ pd, long long cap, long long n, int d0,
                                             int d1, int d2, const T* __restrict__ vx, const T* __restrict__ vy,
                                             const T* __restrict__ vz, int do_g2p, int do_advect, T dt,
                                             const T* __restrict__ sp, uint32_t* __restrict__ keys,
                                             int32_t* __restrict__ vals) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int d[3] = {d0, d1, d2};
    g2p_particle<T, FACTORED>(g, pd, cap, i, d, do_g2p, do_advect, dt, sp, keys, vals,
                              [&](const int*, VSrc<T> src[3]) {
                                  global_sources(g, vx, vy, vz, src);
                                  return false;
                              });
}

// G2P + advection over the cell-sorted particles, one CTA per 8^3-cell tile:
// the tile's window region of each face component (the P2G region) is
// staged once in shared memory with coalesced loads, then every particle of
// the tile's 64 rows gathers from it.  The gather arithmetic is that of
// k_g2p (bit-identical in FP32 / FP64, the factored sums in mixed precision).
template <class T, bool FACTORED>
__global__ void __launch_bounds__(256, 3) k_g2p_tile(GridP<T> g, T* __restrict__ pd, long long cap,
                                                  const int32_t* __restrict__ cs, int d0, int d1, int d2,
                                                  const T* __restrict__ vx, const T* __restrict__ vy,
                                                  const T* __restrict__ vz, T dt, const T* __restrict__ sp,
                                                  uint32_t* __restrict__ keys, int32_t* __restrict__ vals,
                                                  const int32_t* __restrict__ pid_src, int32_t* __restrict__ pid_dst) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sv = reinterpret_cast<T*>(smem_raw);
    __shared__ int roff[kTile * kTile + 1];
    __shared__ int rbeg[kTile * kTile];
    const int x0 = blockIdx.z * kTile, y0 = blockIdx.y * kTile, z0 = blockIdx.x * kTile;
    const int zend = min(z0 + kTile, g.nz);
    if (threadIdx.x < kTile * kTile) {
        const int rx = x0 + (threadIdx.x >> 3), ry = y0 + (threadIdx.x & 7);
        int cnt = 0, beg = 0;
        if (rx < g.nx && ry < g.ny) {
            const long long c = ((long long)rx * g.ny + ry) * g.nz + z0;
            beg = cs[c];
            cnt = cs[c + (zend - z0)] - beg;
        }
        rbeg[threadIdx.x] = beg;
        roff[threadIdx.x + 1] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        roff[0] = 0;
        for (int r = 0; r < kTile * kTile; ++r) roff[r + 1] += roff[r];
    }
    __syncthreads();
    const int total = roff[kTile * kTile];
    if (total == 0) return;
    const int R0 = p2g_region(0), R1 = p2g_region(1);
    const T* vsrc[3] = {vx, vy, vz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int ey = kTile + 2 + (a == 1), ez = kTile + 2 + (a == 2);
        const int R = p2g_region(a);
        T* dst = sv + ((a == 1) ? R0 : (a == 2) ? R0 + R1 : 0);
        const int fy = g.ny + (a == 1), fz = g.nz + (a == 2), fx = g.nx + (a == 0);
        for (int e = threadIdx.x; e < R; e += blockDim.x) {
            const int lz = e % ez, ly = (e / ez) % ey, lx = e / (ey * ez);
            const int xi = x0 - 1 + lx, yi = y0 - 1 + ly, zi = z0 - 1 + lz;
            T v = T(0);
            if (xi >= 0 && xi < fx && yi >= 0 && yi < fy && zi >= 0 && zi < fz)
                v = vsrc[a][((long long)xi * fy + yi) * fz + zi];
            dst[e] = v;
        }
    }
    __syncthreads();
    const int d[3] = {d0, d1, d2};
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
        int lo = 0, hi = kTile * kTile;  // the row r with roff[r] <= f < roff[r + 1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (roff[mid] <= f) lo = mid;
            else hi = mid;
        }
        const long long i = rbeg[lo] + (f - roff[lo]);
        // the deferred permutation: vals holds it and gets the identity below
        if (pid_src) pid_dst[i] = pid_src[vals[i]];
        g2p_particle<T, FACTORED>(g, pd, cap, i, d, 1, 1, dt, sp, keys, vals, [&](const int* ci, VSrc<T> src[3]) {
            const bool in = ci[0] >= x0 && ci[0] < x0 + kTile && ci[1] >= y0 && ci[1] < y0 + kTile && ci[2] >= z0 &&
                            ci[2] < zend;
            if (!in) {  // off the grid: sorted into a clamped cell
                global_sources(g, vx, vy, vz, src);
                return false;
            }
            src[0] = VSrc<T>{sv, x0 - 1, y0 - 1, z0 - 1, kTile + 2, kTile + 2};
            src[1] = VSrc<T>{sv + R0, x0 - 1, y0 - 1, z0 - 1, kTile + 3, kTile + 2};
            src[2] = VSrc<T>{sv + R0 + R1, x0 - 1, y0 - 1, z0 - 1, kTile + 2, kTile + 3};
            return true;
        });
    }
}

// ------------------------------------------------------- CorrectVolume
// Uniform number in [0, 1) for the coincident-particle branch of
// CorrectVolume: SplitMix64 (Steele, Lea and Flood, 2014) of the call count,
// both particles' indices, the visit and the axis; the top 24 bits.
__host__ __device__ __forceinline__ float cv_uniform(unsigned long long call, long long i, long long j, int visit,
                                                     int axis) {
    unsigned long long z = call * 0x9E3779B97F4A7C15ull + (unsigned long long)i * 0xBF58476D1CE4E5B9ull +
                           (unsigned long long)j * 0x94D049BB133111EBull + (unsigned long long)(visit * 3 + axis);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return float(z >> 40) * (1.0f / 16777216.0f);
}

// HashNeighborSearch::GetImpactRegion (NeighborSearch.h:87-95): the cells
// within one of the particle's own (unclamped) cell index, clamped to the grid.
template <class T>
__device__ __forceinline__ void cv_region(const GridP<T>& g, const T q[3], int lo[3], int hi[3]) {
    const int n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int c = int(X<T>::div(X<T>::sub(q[i], g.mn[i]), g.dx[i]));
        lo[i] = min(max(c - 1, 0), n[i] - 1);
        hi[i] = min(max(c + 1, 0), n[i] - 1);
    }
}

// LiquidModel<3>::CorrectVolume (LiquidModel.cpp:1086-1124) for the
// particles with caller index = step (mod cycle): the repulsion of every
// other particle within one radius, visited once per cell that the two
// particles' impact regions share (as the hash table lists a particle once
// per cell of its region and the query walks the cells of the particle's
// region), then the move and the solid push-out.  Candidates come from the
// cell-sorted particles of the cells within one of the region; cells in x,
// y, z order, particles in sorted order.  New positions go to out (3 x cap).
template <class T>
__global__ void __launch_bounds__(256)
    k_correct_volume(GridP<T> g, const T* __restrict__ pd, long long cap, const int32_t* __restrict__ pid,
                     const int32_t* __restrict__ cs, long long n, T radius, T wfac, T dt, int cycle, int step,
                     unsigned long long call, const T* __restrict__ sp, T* __restrict__ out) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int id = pid[k];
    if (id % cycle != step) return;
    const T p[3] = {pd[k], pd[cap + k], pd[2 * cap + k]};
    const T r2 = X<T>::mul(radius, radius);
    int lo[3], hi[3];
    cv_region(g, p, lo, hi);
    T rep[3] = {T(0), T(0), T(0)};
    for (int cx = max(lo[0] - 1, 0); cx <= min(hi[0] + 1, g.nx - 1); ++cx)
        for (int cy = max(lo[1] - 1, 0); cy <= min(hi[1] + 1, g.ny - 1); ++cy)
            for (int cz = max(lo[2] - 1, 0); cz <= min(hi[2] + 1, g.nz - 1); ++cz) {
                const long long c = ((long long)cx * g.ny + cy) * g.nz + cz;
                for (int j = cs[c]; j < cs[c + 1]; ++j) {
                    if (j == k) continue;
                    const T q[3] = {pd[j], pd[cap + j], pd[2 * cap + j]};
                    const T dir[3] = {X<T>::sub(p[0], q[0]), X<T>::sub(p[1], q[1]), X<T>::sub(p[2], q[2])};
                    const T d2 = sqnorm3(dir[0], dir[1], dir[2]);
                    if (d2 >= r2) continue;
                    int lj[3], hj[3];
                    cv_region(g, q, lj, hj);
                    int mult = 1;
#pragma unroll
                    for (int i = 0; i < 3; ++i) mult *= max(0, min(hi[i], hj[i]) - max(lo[i], lj[i]) + 1);
                    if (mult == 0) continue;
                    const T dist = X<T>::sqrt(d2);
                    const T w = X<T>::mul(wfac, qweight(X<T>::div(dist, radius)));
                    if (double(dist) > 1e-4 * double(radius)) {
                        const T wr = X<T>::mul(w, radius);
                        const T t[3] = {X<T>::mul(wr, X<T>::div(dir[0], dist)), X<T>::mul(wr, X<T>::div(dir[1], dist)),
                                        X<T>::mul(wr, X<T>::div(dir[2], dist))};
                        for (int v = 0; v < mult; ++v)
#pragma unroll
                            for (int i = 0; i < 3; ++i) rep[i] = X<T>::add(rep[i], t[i]);
                    } else {
                        const T rdt = X<T>::div(radius, dt);
                        for (int v = 0; v < mult; ++v)
#pragma unroll
                            for (int i = 0; i < 3; ++i)
                                rep[i] = X<T>::add(rep[i], X<T>::mul(rdt, T(cv_uniform(call, id, pid[j], v, i))));
                    }
                }
            }
    T np_[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) np_[i] = X<T>::add(p[i], X<T>::mul(rep[i], dt));
    const T sphi = solid_phi_at(g, sp, np_[0], np_[1], np_[2]);
    if (sphi < T(0)) {
        T gr[3];
        solid_grad_at(g, sp, np_[0], np_[1], np_[2], gr);
#pragma unroll
        for (int i = 0; i < 3; ++i) np_[i] = X<T>::sub(np_[i], X<T>::mul(sphi, gr[i]));
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) out[i * cap + k] = np_[i];
}

// SetPosition(pi, GetBuffer(pi)) for the moved particles (LiquidModel.cpp:1126-1129)
template <class T>
__global__ void k_correct_apply(T* __restrict__ pd, long long cap, const int32_t* __restrict__ pid, long long n,
                                int cycle, int step, const T* __restrict__ buf) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || pid[k] % cycle != step) return;
#pragma unroll
    for (int i = 0; i < 3; ++i) pd[i * cap + k] = buf[i * cap + k];
}

// max |v| over particles for GetCFL (LiquidModel.h:49-55)
template <class T>
__global__ void k_vmax(const T* __restrict__ pd, long long cap, long long n, double* __restrict__ partials,
                       unsigned* __restrict__ counter, double* __restrict__ out) {
    double m = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        for (int k = 0; k < 3; ++k) m = fmax(m, fabs(double(pd[(3 + k) * cap + i])));
    m = block_max(m);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = m;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double a = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) a = fmax(a, ((volatile double*)partials)[b]);
    a = block_max(a);
    if (threadIdx.x == 0) {
        *out = a;
        *counter = 0u;
    }
}

// ------------------------------------------------------------- host side
template <class T, class TX> static GridP<T> gridp(const LiquidImpl<T, TX>& s) {
    GridP<T> g;
    g.nx = s.nx_;
    g.ny = s.ny_;
    g.nz = s.nz_;
    for (int i = 0; i < 3; ++i) {
        g.mn[i] = s.min_[i];
        g.mx[i] = s.max_[i];
        g.dx[i] = s.dx_[i];
        g.idx[i] = T(1) / s.dx_[i];
    }
    return g;
}

template <class T> static int window(T r, T dx) { return int(std::ceil(r / dx)); }

template <class T, class TX> void LiquidImpl<T, TX>::alloc_particles(int64_t cap) {
    if (cap <= pcap_) return;
    for (int b = 0; b < 2; ++b) {
        if (pdata_[b]) cudaFree(pdata_[b]);
        if (pid_[b]) cudaFree(pid_[b]);
        if (keys_[b]) cudaFree(keys_[b]);
        if (vals_[b]) cudaFree(vals_[b]);
        LHI_CUDA(cudaMalloc(&pdata_[b], sizeof(T) * 15 * size_t(cap)));
        LHI_CUDA(cudaMalloc(&pid_[b], sizeof(int32_t) * size_t(cap)));
        LHI_CUDA(cudaMalloc(&keys_[b], sizeof(uint32_t) * size_t(cap)));
        LHI_CUDA(cudaMalloc(&vals_[b], sizeof(int32_t) * size_t(cap)));
    }
    pcap_ = cap;
    pcur_ = 0;
    perm_pending_ = false;
}

template <class T, class TX>
void LiquidImpl<T, TX>::set_particles(int64_t n, const void* pos, const void* vel, const void* aff) {
    if (n < 0 || n > (int64_t(1) << 31) - 1) throw std::invalid_argument("particle count out of range");
    if (n > 0 && !pos) throw std::invalid_argument("pos is NULL");
    alloc_particles(std::max<int64_t>(n, 1));
    np_ = n;
    sorted_ = false;
    perm_pending_ = false;
    if (n == 0) return;
    T* stage = pdata_[pcur_ ^ 1];  // AoS staging: pos[3n] vel[3n] aff[9n]
    LHI_CUDA(cudaMemcpyAsync(stage, pos, sizeof(T) * 3 * n, cudaMemcpyHostToDevice, stream_));
    if (vel) LHI_CUDA(cudaMemcpyAsync(stage + 3 * n, vel, sizeof(T) * 3 * n, cudaMemcpyHostToDevice, stream_));
    if (aff) LHI_CUDA(cudaMemcpyAsync(stage + 6 * n, aff, sizeof(T) * 9 * n, cudaMemcpyHostToDevice, stream_));
    k_aos_to_soa<T><<<blocks_for(n, 256), 256, 0, stream_>>>(stage, pdata_[pcur_], pcap_, pid_[pcur_], n,
                                                             vel ? 1 : 0, aff ? 1 : 0);
    LHI_LAUNCH_CHECK();
    keys_fresh_ = false;
}

template <class T, class TX> void LiquidImpl<T, TX>::get_particles(void* pos, void* vel, void* aff) {
    if (np_ == 0) return;
    apply_order();  // its staging buffer is the other one
    T* stage = pdata_[pcur_ ^ 1];
    k_soa_to_aos<T><<<blocks_for(np_, 256), 256, 0, stream_>>>(pdata_[pcur_], pcap_, pid_[pcur_], stage, np_);
    LHI_LAUNCH_CHECK();
    if (pos) LHI_CUDA(cudaMemcpyAsync(pos, stage, sizeof(T) * 3 * np_, cudaMemcpyDeviceToHost, stream_));
    if (vel) LHI_CUDA(cudaMemcpyAsync(vel, stage + 3 * np_, sizeof(T) * 3 * np_, cudaMemcpyDeviceToHost, stream_));
    if (aff) LHI_CUDA(cudaMemcpyAsync(aff, stage + 6 * np_, sizeof(T) * 9 * np_, cudaMemcpyDeviceToHost, stream_));
    LHI_CUDA(cudaStreamSynchronize(stream_));
}

// Stable sort of the particles by cell key, then the per-cell ranges.  The
// keys of the current positions are already in keys_[0]/vals_[0] (written by
// set_particles or by the advection kernel).
template <class T, class TX> void LiquidImpl<T, TX>::sort_particles() {
    apply_order();  // the keys below are those of the physical order
    auto ps_ = scope(LHI_KERNEL_SORT);
    if (np_ > 0) {
        if (!keys_fresh_) {
            k_keys<T><<<blocks_for(np_, 256), 256, 0, stream_>>>(gridp(*this), pdata_[pcur_], pcap_, np_, keys_[0],
                                                                 vals_[0]);
            LHI_LAUNCH_CHECK();
        }
    }
    // counting sort by cell key: per-cell counts, their exclusive scan (the
    // cell ranges), a scatter by atomic ranks, then each cell's indices in
    // input order -- the stable sort, one read of the keys per pass
    LHI_CUDA(cudaMemsetAsync(cell_count_, 0, sizeof(int32_t) * size_t(ncell_ + 1), stream_));
    if (np_ > 0) {
        k_cell_count<<<blocks_for(np_, 256), 256, 0, stream_>>>(keys_[0], np_, cell_count_);
        LHI_LAUNCH_CHECK();
    }
    device_exclusive_scan_i32(cell_count_, cell_start_, ncell_ + 1, scan_tmp_, scan_tmp_bytes_, stream_);
    if (np_ > 0) {
        LHI_CUDA(cudaMemsetAsync(cell_count_, 0, sizeof(int32_t) * size_t(ncell_), stream_));  // rank cursors
        k_rank_scatter<<<blocks_for(np_, 256), 256, 0, stream_>>>(keys_[0], np_, cell_start_, cell_count_, keys_[1],
                                                                 vals_[1]);
        LHI_LAUNCH_CHECK();
        k_cell_order<<<blocks_for(ncell_, 256), 256, 0, stream_>>>(cell_start_, ncell_, pid_[pcur_], vals_[1]);
        LHI_LAUNCH_CHECK();
        // only the positions move now (the liquid SDF walks them); P2G reads
        // the rest through the permutation and G2P writes the sorted state
        k_gather_pos<T><<<blocks_for(np_, 256), 256, 0, stream_>>>(pdata_[pcur_], pdata_[pcur_ ^ 1], pcap_,
                                                                   vals_[1], np_);
        LHI_LAUNCH_CHECK();
        std::swap(keys_[0], keys_[1]);  // the sorted keys in keys_[0]
        std::swap(vals_[0], vals_[1]);  // the permutation in vals_[0]
        perm_pending_ = true;
    }
    LHI_CUDA(cudaMemsetAsync(occ_, 0, size_t(occ_dim_[0]) * occ_dim_[1] * occ_dim_[2], stream_));
    k_occupancy<<<blocks_for(ncell_, 256), 256, 0, stream_>>>(cell_start_, nx_, ny_, nz_, occ_, occ_dim_[0],
                                                              occ_dim_[1], occ_dim_[2]);
    LHI_LAUNCH_CHECK();
    sorted_ = true;
    keys_fresh_ = false;
}

template <class T, class TX> void LiquidImpl<T, TX>::ensure_sorted() {
    if (!sorted_) sort_particles();
}

// Applies a deferred permutation: the whole state (and the ids) in sorted order.
template <class T, class TX> void LiquidImpl<T, TX>::apply_order() {
    if (!perm_pending_) return;
    perm_pending_ = false;
    if (np_ == 0) return;
    auto ps_ = scope(LHI_KERNEL_SORT);
    k_permute<T><<<blocks_for(np_, 256), 256, 0, stream_>>>(pdata_[pcur_], pdata_[pcur_ ^ 1], pcap_, pid_[pcur_],
                                                            pid_[pcur_ ^ 1], vals_[0], np_);
    LHI_LAUNCH_CHECK();
    pcur_ ^= 1;
}

// The window offsets of k_liquid_phi with their distance bounds: a window
// cell at offset (ax, ay, az) holds points no nearer to the cell centre than
// the box distance max(|a| - 1/2, 0) dx per axis; the bound takes 1e-5 off
// that distance and adds 1e-6 to r, far more than the rounding of the
// kernel's |x_c - x_p| - r.  Sorted ascending (stable, own cell first).
template <class T, class TX> void LiquidImpl<T, TX>::build_liquid_phi_table() {
    const int d[3] = {window(radius_, dx_[0]), window(radius_, dx_[1]), window(radius_, dx_[2])};
    if (d[0] > 8 || d[1] > 8 || d[2] > 8) return;  // compute_liquid_phi refuses such a radius
    std::vector<LphiOffset> tab;
    for (int ax = -d[0]; ax <= d[0]; ++ax)
        for (int ay = -d[1]; ay <= d[1]; ++ay)
            for (int az = -d[2]; az <= d[2]; ++az) {
                const T lx = T(std::fmax(double(std::abs(ax)) - 0.5, 0.0)) * dx_[0];
                const T ly = T(std::fmax(double(std::abs(ay)) - 0.5, 0.0)) * dx_[1];
                const T lz = T(std::fmax(double(std::abs(az)) - 0.5, 0.0)) * dx_[2];
                LphiOffset e;
                e.lb = std::sqrt(double(lx) * lx + double(ly) * ly + double(lz) * lz) * (1.0 - 1e-5) -
                       double(radius_) * (1.0 + 1e-6);
                e.off = (ax + 16) | ((ay + 16) << 8) | ((az + 16) << 16);
                e.pad = (ax == 0 && ay == 0 && az == 0) ? 0 : 1;
                tab.push_back(e);
            }
    std::stable_sort(tab.begin(), tab.end(), [](const LphiOffset& a, const LphiOffset& b) {
        return a.pad != b.pad ? a.pad < b.pad : a.lb < b.lb;
    });
    lphi_n_ = int(tab.size());
    LHI_CUDA(cudaMalloc(&lphi_tab_, sizeof(LphiOffset) * tab.size()));
    LHI_CUDA(cudaMemcpy(lphi_tab_, tab.data(), sizeof(LphiOffset) * tab.size(), cudaMemcpyHostToDevice));
}

template <class T, class TX> void LiquidImpl<T, TX>::compute_liquid_phi() {
    if (np_ == 0) return;
    ensure_sorted();
    int d0 = window(radius_, dx_[0]), d1 = window(radius_, dx_[1]), d2 = window(radius_, dx_[2]);
    if (d0 > 8 || d1 > 8 || d2 > 8) throw std::invalid_argument("particle radius above 8 cells is not supported");
    auto ps_ = scope(LHI_KERNEL_LIQUID_PHI);
    k_liquid_phi<T><<<blocks_for(ncell_, 256), 256, 0, stream_>>>(gridp(*this), cell_start_, occ_, occ_dim_[0],
                                                                  occ_dim_[1], occ_dim_[2],
                                                                  pdata_[perm_pending_ ? pcur_ ^ 1 : pcur_], pcap_,
                                                                  radius_, d0, d1, d2, lphi_tab_, lphi_n_,
                                                                  liquid_phi_);
    LHI_LAUNCH_CHECK();
}

template <class T, class TX> void LiquidImpl<T, TX>::p2g_accumulate() {
    ensure_sorted();
    auto ps_ = scope(LHI_KERNEL_P2G);
    int d0 = window(radius_, dx_[0]), d1 = window(radius_, dx_[1]), d2 = window(radius_, dx_[2]);
    P2GOut<T> out;
    for (int a = 0; a < 3; ++a) {
        out.v[a] = v_[a];
        out.w[a] = w_[a];
    }
    // tile accumulators, then one staging buffer per warp (small enough for three CTAs per SM)
    size_t smem = sizeof(T) * (2 * (p2g_region(0) + p2g_region(1) + p2g_region(2)) + kP2GWarps * kP2GStage);
    LHI_CUDA(cudaFuncSetAttribute(k_p2g<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    dim3 grid(unsigned((nz_ + kTile - 1) / kTile), unsigned((ny_ + kTile - 1) / kTile),
              unsigned((nx_ + kTile - 1) / kTile));
    // particles off the grid are listed (in vals_[1], free after the sort) for k_p2g_overflow
    int* ov_count = &sc_->p2g_overflow;
    LHI_CUDA(cudaMemsetAsync(ov_count, 0, sizeof(int), stream_));
    PView<T> pv;
    pv.pos = pdata_[perm_pending_ ? pcur_ ^ 1 : pcur_];
    pv.rest = pdata_[pcur_];
    pv.order = perm_pending_ ? vals_[0] : nullptr;
    pv.cap = pcap_;
    k_p2g<T><<<grid, kP2GWarps * 32, smem, stream_>>>(gridp(*this), cell_start_, pv, d0, d1, d2, out, ov_count,
                                                       vals_[1]);
    LHI_LAUNCH_CHECK();
    k_p2g_overflow<T><<<kSMs, 256, 0, stream_>>>(gridp(*this), pv, d0, d1, d2, out, ov_count, vals_[1]);
    LHI_LAUNCH_CHECK();
}

template <class T, class TX> void LiquidImpl<T, TX>::p2g_normalize(bool with_gravity, T gdt) {
    auto ps_ = scope(LHI_KERNEL_GRID);  // a per-face grid pass (with gravity); P2G times the accumulation alone
    for (int a = 0; a < 3; ++a) {
        int fx = nx_ + (a == 0), fy = ny_ + (a == 1), fz = nz_ + (a == 2);
        k_p2g_normalize<T><<<blocks_for(nface_[a], 256), 256, 0, stream_>>>(
            v_[a], w_[a], fx, fy, fz, (with_gravity && a == 1) ? 1 : 0, gdt, nx_, ny_, nz_);
        LHI_LAUNCH_CHECK();
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::correct_volume(double dt) {
    if (np_ == 0) return;
    ensure_sorted();  // cell lists of the current positions
    apply_order();
    auto ps_ = scope(LHI_KERNEL_G2P);
    // weightFactor = sqrt(dx.x * dx.y * dx.z) (LiquidModel.cpp:1089)
    const T wfac = std::sqrt(dx_[0] * dx_[1] * dx_[2]);
    T* buf = pdata_[pcur_ ^ 1];  // the permutation's other buffer, free between sorts
    k_correct_volume<T><<<blocks_for(np_, 256), 256, 0, stream_>>>(
        gridp(*this), pdata_[pcur_], pcap_, pid_[pcur_], cell_start_, np_, radius_, wfac, T(dt), correct_cycle_,
        correct_step_, correct_calls_, solid_phi_, buf);
    LHI_LAUNCH_CHECK();
    k_correct_apply<T><<<blocks_for(np_, 256), 256, 0, stream_>>>(pdata_[pcur_], pcap_, pid_[pcur_], np_,
                                                                 correct_cycle_, correct_step_, buf);
    LHI_LAUNCH_CHECK();
    correct_step_ = (correct_step_ + 1) % correct_cycle_;
    ++correct_calls_;
    // positions moved: the next sort recomputes the keys
    sorted_ = false;
    keys_fresh_ = false;
}

template <class T, class TX> void LiquidImpl<T, TX>::particle_to_grid() {
    if (np_ == 0) return;
    p2g_accumulate();
    p2g_normalize(false, T(0));
}

template <class T, class TX> void LiquidImpl<T, TX>::g2p(bool do_advect, T dt) {
    if (np_ == 0) return;
    int d0 = window(radius_, dx_[0]), d1 = window(radius_, dx_[1]), d2 = window(radius_, dx_[2]);
    auto ps_ = scope(LHI_KERNEL_G2P);
    // mixed precision takes the factored sums; FP32 and FP64 keep the reference's order bit for bit
    const bool fact = precision_ == LHI_PRECISION_MIXED;
    if (do_advect) {
        // over the cell-sorted particles, tile by tile, with the face velocities staged in shared memory
        ensure_sorted();
        const size_t smem = sizeof(T) * size_t(p2g_region(0) + p2g_region(1) + p2g_region(2));
        dim3 grid(unsigned((nz_ + kTile - 1) / kTile), unsigned((ny_ + kTile - 1) / kTile),
                  unsigned((nx_ + kTile - 1) / kTile));
        auto kern = fact ? k_g2p_tile<T, true> : k_g2p_tile<T, false>;
        // with the sort's permutation deferred the kernel writes the sorted state into the other buffer
        // (whose positions are already sorted) and carries the ids over
        const bool defer = perm_pending_;
        kern<<<grid, 256, smem, stream_>>>(gridp(*this), pdata_[defer ? pcur_ ^ 1 : pcur_], pcap_, cell_start_, d0,
                                           d1, d2, v_[0], v_[1], v_[2], dt, solid_phi_, keys_[0], vals_[0],
                                           defer ? pid_[pcur_] : nullptr, defer ? pid_[pcur_ ^ 1] : nullptr);
        if (defer) {
            pcur_ ^= 1;
            perm_pending_ = false;
        }
    } else {
        apply_order();
        auto kern = fact ? k_g2p<T, true> : k_g2p<T, false>;
        kern<<<blocks_for(np_, 256), 256, 0, stream_>>>(gridp(*this), pdata_[pcur_], pcap_, np_, d0, d1, d2, v_[0],
                                                        v_[1], v_[2], 1, 0, dt, solid_phi_, keys_[0], vals_[0]);
    }
    LHI_LAUNCH_CHECK();
    if (do_advect) {
        sorted_ = false;
        keys_fresh_ = true;
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::grid_to_particle() { g2p(false, T(0)); }

template <class T, class TX> void LiquidImpl<T, TX>::advect(double dt) {
    if (np_ == 0) return;
    apply_order();
    int d0 = window(radius_, dx_[0]), d1 = window(radius_, dx_[1]), d2 = window(radius_, dx_[2]);
    auto ps_ = scope(LHI_KERNEL_G2P);
    k_g2p<T, false><<<blocks_for(np_, 256), 256, 0, stream_>>>(gridp(*this), pdata_[pcur_], pcap_, np_, d0, d1, d2,
                                                               v_[0], v_[1], v_[2], 0, 1, T(dt), solid_phi_, keys_[0],
                                                               vals_[0]);
    LHI_LAUNCH_CHECK();
    sorted_ = false;
    keys_fresh_ = true;
}

template <class T, class TX> double LiquidImpl<T, TX>::cfl() {
    double vmax = 0.0;
    if (np_ > 0) {
        k_vmax<T><<<std::min<unsigned>(blocks_for(np_, 256), 4 * kSMs), 256, 0, stream_>>>(
            pdata_[pcur_], pcap_, np_, partials_, counter_, &sc_->vmax);
        LHI_LAUNCH_CHECK();
        vmax = read_scalar(&sc_->vmax);
    }
    // MathUtils::Clamp(dx.x / maxVel, 0.001, 0.1) in Scalar
    T mv = T(vmax);
    T r = dx_[0] / mv;
    T lo = T(0.001), hi = T(0.1);
    T t = (lo > r) ? lo : r;
    return double((hi < t) ? hi : t);
}

template class LiquidImpl<float, float>;
template class LiquidImpl<float, double>;
template class LiquidImpl<double, double>;

}  // namespace lhi
