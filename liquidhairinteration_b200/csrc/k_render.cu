// k_render.cu -- headless particle render: the reference's point drawing
// (LiquidModel<3>::Render, LiquidModel.cpp:1138-1159, with the vertex shader
// Shader/Scene3D_vertex.glsl and the fragment shader Scene3D_fragment.glsl)
// as CUDA kernels writing an RGBA image in device memory.  No graphics API.
//
// Per particle (the vertex shader): point = (pos - minCoord) / (maxCoord -
// minCoord) * 2 - 1, in float, the attribute type of the reference's vertex
// buffer (GL_FLOAT).  Then fixed-function GL, restated: a point whose
// normalised device coordinates leave [-1, 1] on any axis is clipped; the
// viewport maps x to xw = (x + 1) * (width / 2) (same for y); the point is a
// square of side pointSize centred at (xw, yw) that covers the pixels whose
// centres (i + 0.5, j + 0.5) satisfy xw - s/2 <= i + 0.5 < xw + s/2 (same
// for y).  Every covered pixel takes the point colour (the fragment shader
// writes one uniform colour and the reference enables no depth test or
// blending), every other pixel keeps the clear colour.  Row 0 of the image
// is the bottom row, as in GL window coordinates.
#include "impl.cuh"

namespace lhi {

namespace {

// the vertex shader, float arithmetic without contraction
__device__ __forceinline__ float ndc_axis(float p, float mn, float mx) {
    const float a = __fsub_rn(p, mn);
    const float b = __fsub_rn(mx, mn);
    return __fsub_rn(__fmul_rn(__fdiv_rn(a, b), 2.0f), 1.0f);
}

// covered pixel range [lo, hi] of one axis, clamped to the image
__device__ __forceinline__ void cover(float ndc, int extent, float size, int& lo, int& hi) {
    const float xw = __fmul_rn(__fadd_rn(ndc, 1.0f), __fmul_rn(0.5f, float(extent)));
    const float h = __fmul_rn(size, 0.5f);
    lo = int(ceilf(__fsub_rn(__fsub_rn(xw, h), 0.5f)));
    hi = int(ceilf(__fsub_rn(__fadd_rn(xw, h), 0.5f))) - 1;
    lo = max(lo, 0);
    hi = min(hi, extent - 1);
}

__global__ void k_clear_image(uchar4* __restrict__ img, long long n, uchar4 bg) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) img[i] = bg;
}

template <class T>
__global__ void k_splat(const T* __restrict__ pd, long long cap, const int32_t* __restrict__ pid, long long n,
                        float3 mn, float3 mx, int width, int height, float size, uchar4 color,
                        uchar4* __restrict__ img, float* __restrict__ ndc_out) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float x = ndc_axis(float(pd[k]), mn.x, mx.x);
    const float y = ndc_axis(float(pd[cap + k]), mn.y, mx.y);
    const float z = ndc_axis(float(pd[2 * cap + k]), mn.z, mx.z);
    if (ndc_out) {
        const long long i = pid[k];  // the caller's particle order
        ndc_out[3 * i + 0] = x;
        ndc_out[3 * i + 1] = y;
        ndc_out[3 * i + 2] = z;
    }
    if (!img) return;
    // clipping (a NaN coordinate fails every comparison and is clipped too)
    if (!(x >= -1.f && x <= 1.f && y >= -1.f && y <= 1.f && z >= -1.f && z <= 1.f)) return;
    int x0, x1, y0, y1;
    cover(x, width, size, x0, x1);
    cover(y, height, size, y0, y1);
    // every writer stores the same colour, so overlapping points need no ordering
    for (int j = y0; j <= y1; ++j)
        for (int i = x0; i <= x1; ++i) img[(long long)j * width + i] = color;
}

}  // namespace

template <class T, class TX>
void LiquidImpl<T, TX>::render(const lhi_render_params& rp, float* ndc_host, uint8_t* rgba_host) {
    if (rp.width < 1 || rp.height < 1 || (long long)rp.width * rp.height > (1LL << 28))
        throw std::invalid_argument("render: image size out of range");
    if (!(rp.point_size >= 0.f) || rp.point_size > 1024.f) throw std::invalid_argument("render: bad point size");
    const long long npix = (long long)rp.width * rp.height;
    if (rgba_host && npix > image_cap_) {
        if (image_) cudaFree(image_);
        image_ = nullptr;
        image_cap_ = 0;
        LHI_CUDA(cudaMalloc(&image_, sizeof(uchar4) * npix));
        image_cap_ = npix;
    }
    if (ndc_host && np_ > ndc_cap_) {
        if (ndc_) cudaFree(ndc_);
        ndc_ = nullptr;
        ndc_cap_ = 0;
        LHI_CUDA(cudaMalloc(&ndc_, sizeof(float) * 3 * np_));
        ndc_cap_ = np_;
    }
    uchar4* img = rgba_host ? reinterpret_cast<uchar4*>(image_) : nullptr;
    float* ndc = ndc_host ? ndc_ : nullptr;
    if (img) {
        const uchar4 bg = make_uchar4(rp.background[0], rp.background[1], rp.background[2], rp.background[3]);
        k_clear_image<<<blocks_for(npix, 256), 256, 0, stream_>>>(img, npix, bg);
        LHI_LAUNCH_CHECK();
    }
    if (np_ > 0 && (img || ndc)) {
        const float3 mn = make_float3(float(min_[0]), float(min_[1]), float(min_[2]));
        const float3 mx = make_float3(float(max_[0]), float(max_[1]), float(max_[2]));
        const uchar4 col = make_uchar4(rp.color[0], rp.color[1], rp.color[2], rp.color[3]);
        k_splat<T><<<blocks_for(np_, 256), 256, 0, stream_>>>(pdata_[pcur_], pcap_, pid_[pcur_], np_, mn, mx,
                                                             rp.width, rp.height, rp.point_size, col, img, ndc);
        LHI_LAUNCH_CHECK();
    }
    if (img) LHI_CUDA(cudaMemcpyAsync(rgba_host, img, sizeof(uchar4) * npix, cudaMemcpyDeviceToHost, stream_));
    if (ndc && np_ > 0) LHI_CUDA(cudaMemcpyAsync(ndc_host, ndc, sizeof(float) * 3 * np_, cudaMemcpyDeviceToHost, stream_));
    LHI_CUDA(cudaStreamSynchronize(stream_));
}

template class LiquidImpl<float, float>;
template class LiquidImpl<float, double>;
template class LiquidImpl<double, double>;

}  // namespace lhi
