// net.cuh -- the learned preconditioner: a small multilevel 3D convolutional
// network M(r, masks) -> search direction, used inside flexible PCG.
//
// Network (3 levels, 3x3x3 convolutions, zero padding, no biases, ~140k
// weights):
//   a0 = r/s x [1, next to air, next to solid, 0]   4 channels (stored as 16)  N
//   h0 = act(conv0(a0))                        16                         N
//   h1 = act(conv1(avgpool(h0)))               32                         N/2
//   h2 = act(conv2(avgpool(h1)))               64                         N/4
//   u1 = act(conv3(upsample(h2)) + h1)         32                         N/2
//   u0 = act(conv4(upsample(u1)) + h0)         16                         N
// act is the identity by default (a linear multilevel operator: a fixed
// preconditioner for a given geometry, which flexible CG needs to keep its
// conjugate directions) or ReLU (lhi_net_set_relu).
//   z  = s * conv5(u0)  on fluid cells          1                         N
// s = RMS of r over fluid cells.  The fluid / air / solid masks enter
// multiplied by r and nothing is added, so M(a r) = a M(r) for a > 0 and
// M(0) = 0: a constant offset in z would stall the conjugate directions.
// The packed layout keeps a bias vector per layer; it is ignored.  Activations are BF16
// channels-last (voxel-major, channels contiguous, padded to 16); every
// convolution accumulates in FP32.  Parameters are FP32 master copies with
// BF16 working copies for the tensor cores.
#pragma once

#include <cstring>
#include <vector>

#include "common.cuh"

namespace lhi {

constexpr int kNetLayers = 6;
constexpr int kNetCin[kNetLayers] = {4, 16, 32, 64, 32, 16};   // real input channels
constexpr int kNetCout[kNetLayers] = {16, 32, 64, 32, 16, 1};  // real output channels
constexpr int kNetTaps = 27;

__host__ __device__ constexpr int pad16(int c) { return (c + 15) / 16 * 16; }

// Parameter packing (the C-ABI order): per layer, W[27][cout][cin] then
// b[cout]; tap = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1).
inline long long net_param_count() {
    long long n = 0;
    for (int l = 0; l < kNetLayers; ++l) n += (long long)kNetTaps * kNetCout[l] * kNetCin[l] + kNetCout[l];
    return n;
}
inline long long net_param_offset(int layer) {
    long long n = 0;
    for (int l = 0; l < layer; ++l) n += (long long)kNetTaps * kNetCout[l] * kNetCin[l] + kNetCout[l];
    return n;
}

// BF16 round-to-nearest-even from the FP32 bit pattern (quiet NaN kept).
__host__ __device__ __forceinline__ uint16_t bf16_bits(float f) {
    uint32_t u;
#ifdef __CUDA_ARCH__
    u = __float_as_uint(f);
#else
    std::memcpy(&u, &f, 4);
#endif
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return uint16_t((u >> 16) | 0x40u);
    u += 0x7fffu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
}
__host__ __device__ __forceinline__ float bf16_float(uint16_t b) {
    uint32_t u = uint32_t(b) << 16;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}

struct NetStatus {
    int timeout;  // a bounded wait on the tensor-core pipeline gave up
    int pad[7];
};

// Device buffers of one network applied at one grid size (level dims n0,
// n1 = n0 / 2, n2 = n1 / 2 per axis).
struct NetBuffers {
    int dims[3][3] = {};
    long long vox[3] = {0, 0, 0};
    long long cap_vox0 = 0;  // allocation size (voxels of level 0)
    // activations (BF16 channels-last)
    uint16_t* a0 = nullptr;  // 16 ch, L0
    uint16_t* h0 = nullptr;  // 16, L0
    uint16_t* p0 = nullptr;  // 16, L1
    uint16_t* h1 = nullptr;  // 32, L1
    uint16_t* p1 = nullptr;  // 32, L2
    uint16_t* h2 = nullptr;  // 64, L2
    uint16_t* q1 = nullptr;  // 64, L1
    uint16_t* u1 = nullptr;  // 32, L1
    uint16_t* q0 = nullptr;  // 32, L0
    uint16_t* u0 = nullptr;  // 16, L0
    float* y = nullptr;      // 1, L0
    // gradients
    uint16_t* g[kNetLayers] = {};  // BF16 gradient at each layer's pre-activation (g5 = dy, 16 ch)
    float* dx = nullptr;           // FP32 scratch: conv input gradients (max 64 ch at L1 or 32 ch at L0)
    float* acc = nullptr;          // FP32 scratch: summed gradients (max 32 ch at L0)
};

class LearnedNet {
public:
    explicit LearnedNet(uint64_t seed);
    ~LearnedNet();
    long long num_params() const { return net_param_count(); }
    void set_params(const float* host);
    void get_params(float* host);
    // z = M(r) on a grid of dims n (device pointers, float), fluid = type == 2
    // cells, solid from the cell-centre solid flag, stream s.
    // sparse: evaluate each convolution only on the output tiles the cells
    // with type != 0 depend on (the plan of plan_sparse for this type array;
    // dense when there is none): the same values there, bit for bit.
    void forward(const int dims[3], const float* r, const uint8_t* type, const uint8_t* solid, float* z,
                 double scale_fixed, cudaStream_t s, bool sparse = false);
    // Tile lists of the six convolutions for the output cells type != 0 of
    // this grid (device type array; rebuilt whenever the cells change).
    void plan_sparse(const int dims[3], const uint8_t* type, cudaStream_t s);
    // d(loss)/d(params) += backward of the last forward given dL/dz (device, float); returns in grad_
    void backward(const float* dz, cudaStream_t s);
    void zero_grad(cudaStream_t s);
    void adam_step(double lr, double beta1, double beta2, double eps, cudaStream_t s);
    void get_grads(float* host, cudaStream_t s);
    int check_status(cudaStream_t s);  // 0 or LHI_E_TIMEOUT (once: the status is cleared after a timeout)

    // parameters
    float* w32_ = nullptr;      // master FP32 parameters (packed order)
    float* grad_ = nullptr;     // FP32 gradients (packed order)
    float* adam_m_ = nullptr;
    float* adam_v_ = nullptr;
    long long adam_t_ = 0;
    uint16_t* wfwd_ = nullptr;  // per layer, per tap: B tiles [cout_pad][cin_pad] in UMMA K-major layout
    uint16_t* wbwd_ = nullptr;  // per layer, per tap: B tiles [cin_pad][cout_pad], taps mirrored
    long long wfwd_off_[kNetLayers] = {};
    long long wbwd_off_[kNetLayers] = {};
    bool wfmt_stale_ = true;
    bool relu_ = false;         // activation between layers: ReLU, or none (a linear network)
    NetBuffers b_;
    const uint8_t* last_type_ = nullptr;  // cell types of the last forward (device)
    NetStatus* status_ = nullptr;
    int last_timeout_[3] = {0, 0, 0};  // kernel (1 conv, 2 weight grad), tap / chunk, block of the last timeout
    float* scale_ = nullptr;    // device: s of the last forward
    double* red_ = nullptr;     // device reduction scratch
    unsigned* counter_ = nullptr;

    void ensure(const int dims[3]);
    void format_weights(cudaStream_t s);

    // sparse evaluation (plan_sparse): voxel masks (level 0: two, level 1:
    // two, level 2: two, and the dilations' intermediate), tile flags per
    // level, tile list and count per layer's output and per elementwise
    // stage (kPlanInput .. kPlanUp0: the input channels, the two poolings,
    // the two upsamplings)
    static constexpr int kPlanInput = kNetLayers, kPlanPool0 = kNetLayers + 1, kPlanPool1 = kNetLayers + 2,
                         kPlanUp1 = kNetLayers + 3, kPlanUp0 = kNetLayers + 4, kPlanLists = kNetLayers + 5;
    bool sparse_enabled_ = true;
    const uint8_t* plan_type_ = nullptr;
    int plan_dims_[3] = {0, 0, 0};
    uint8_t* mask_[7] = {};
    uint8_t* tflag_[3] = {};
    int32_t* tlist_[kPlanLists] = {};
    int* tcount_ = nullptr;  // [kPlanLists] on the device
    long long plan_cap_vox0_ = 0;
    void free_plan();
};

// Limit of the brick convolution's pipeline waits on the current device.
void set_net_wait_limit_ns(unsigned long long ns);

// One-CTA tcgen05 GEMM check: D = A B^T, A 128 x K, B N x K (BF16 bits,
// row-major), D 128 x N; *stage reports how far the kernel got.
int umma_selftest(const uint16_t* a_host, const uint16_t* b_host, int N, int K, float* d_host, int* stage);

}  // namespace lhi
