// TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// Runs the reference's own GPU algorithm for general block sizes (the cuFFT
// backend of vs-dfttest2: cuda_source/kernels.cu compiled unchanged from the
// reference tree by oracle/Makefile, plus cuFFT) on one plane, as a second
// checker for block sizes 8 and 32, which dfttest2_cpu does not support.
//
// cuda_source/source.cpp drives those kernels through VapourSynth and the
// CUDA driver API; this file restates that per-plane sequence with the
// runtime API and without VapourSynth:
//   reflection padding of the 2r+1 frames    cuda_source/source.cpp:250-312, 498-510
//   table conversion (window, sigma scalar   cuda_source/source.cpp:790-850
//     or array, window_freq)
//   cuFFT plans: rank 3 {2r+1, B, B}, rank 2  cuda_source/source.cpp:899-923
//     when r = 0, batch = blocks per plane
//   im2col -> R2C -> filter -> C2R -> col2im  cuda_source/source.cpp:515-618
//     (out-of-place: spatial buffer with rows of B samples)
//   slice r of the padded buffer -> output    cuda_source/source.cpp:619-662
// Launch shapes as the reference: 4 warps per CTA, im2col and filter grids of
// SMs x occupancy, col2im on 32 x 4 thread blocks.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "kernels.cu"

namespace {

int pad_size_h(int n, int B, int S) { return n + ((n % B) ? B - n % B : 0) + std::max(B - S, S) * 2; }
int pad_num_h(int n, int B, int S) { return (pad_size_h(n, B, S) - B) / S + 1; }

template <typename T>
void reflect(T* dst, const T* src, int width, int height, int stride, int B, int S) {
    const int pw = pad_size_h(width, B, S), ph = pad_size_h(height, B, S);
    const int oy = (ph - height) / 2, ox = (pw - width) / 2;
    for (int y = 0; y < height; ++y) std::memcpy(&dst[(oy + y) * pw + ox], &src[y * stride], width * sizeof(T));
    for (int y = oy; y < oy + height; ++y) {
        T* line = &dst[y * pw];
        for (int x = 0; x < ox; ++x) line[x] = line[ox * 2 - x];
        for (int x = ox + width; x < pw; ++x) line[x] = line[2 * (ox + width) - 2 - x];
    }
    for (int y = 0; y < oy; ++y) std::memcpy(&dst[y * pw], &dst[(oy * 2 - y) * pw], pw * sizeof(T));
    for (int y = oy + height; y < ph; ++y)
        std::memcpy(&dst[y * pw], &dst[(2 * (oy + height) - 2 - y) * pw], pw * sizeof(T));
}

struct Buffers {
    void* padded = nullptr;
    float* spatial = nullptr;
    cufftComplex* freq = nullptr;
    float* window = nullptr;
    float* sigma = nullptr;
    float* wf = nullptr;
    cufftHandle r2c = 0, c2r = 0;
    bool plans = false;
    ~Buffers() {
        cudaFree(padded);
        cudaFree(spatial);
        cudaFree(freq);
        cudaFree(window);
        cudaFree(sigma);
        cudaFree(wf);
        if (plans) {
            cufftDestroy(r2c);
            cufftDestroy(c2r);
        }
    }
};

}  // namespace

extern "C" {

// src: 2r+1 planes (time clamp applied by the caller), element strides.
// sample_type 0 = integer (bits 8..16), 1 = float.  window: (2r+1)*B*B,
// sigma: 1 (flat, as python/dfttest2.py passes it to the GPU backends) or
// (2r+1)*B*(B/2+1) values, window_freq: (2r+1)*B*(B/2+1)*2 interleaved; all
// FP64 as the plugin receives them.  Returns 0 on success, else a CUDA or
// cuFFT error code (negative for cuFFT).
int ref_cufft_plane(const void* const* src, int width, int height, int src_stride, int sample_type, int bits,
                    void* dst, int dst_stride, const double* window, const double* sigma, int sigma_len,
                    double sigma2, double pmin, double pmax, int filter_type, int zero_mean,
                    const double* window_freq, int radius, int block_size, int block_step) {
    const int B = block_size, S = block_step, T = 2 * radius + 1, X = B / 2 + 1;
    const int bps = sample_type == 1 ? 4 : (bits <= 8 ? 1 : 2);
    const int pw = pad_size_h(width, B, S), ph = pad_size_h(height, B, S);
    const int nx = pad_num_h(width, B, S), ny = pad_num_h(height, B, S), nblocks = nx * ny;
    const size_t plane_elems = (size_t)pw * ph;

    std::vector<uint8_t> h_padded(plane_elems * T * bps);
    for (int t = 0; t < T; ++t) {
        uint8_t* d = h_padded.data() + plane_elems * t * bps;
        if (bps == 1) reflect((uint8_t*)d, (const uint8_t*)src[t], width, height, src_stride, B, S);
        else if (bps == 2) reflect((uint16_t*)d, (const uint16_t*)src[t], width, height, src_stride, B, S);
        else reflect((float*)d, (const float*)src[t], width, height, src_stride, B, S);
    }
    std::vector<float> win(T * B * B), sig(std::max(sigma_len, 1)), wf(T * B * X * 2, 0.0f);
    for (int i = 0; i < T * B * B; ++i) win[i] = (float)window[i];
    for (int i = 0; i < sigma_len; ++i) sig[i] = (float)sigma[i];
    if (zero_mean)
        for (int i = 0; i < T * B * X * 2; ++i) wf[i] = (float)window_freq[i];
    const float sigma_scalar = sigma_len == 1 ? sig[0] : 0.0f;
    const int sigma_is_scalar = sigma_len == 1 ? 1 : 0;
    const float scale = sample_type == 1 ? 255.0f : (float)(1.0 / (1 << (bits - 8)));
    const float peak = (float)((1 << bits) - 1);

    Buffers b;
#define TRY(expr)                               \
    do {                                        \
        cudaError_t e_ = (expr);                \
        if (e_ != cudaSuccess) return (int)e_;  \
    } while (0)
#define TRYF(expr)                               \
    do {                                         \
        cufftResult r_ = (expr);                 \
        if (r_ != CUFFT_SUCCESS) return -(int)r_ - 1; \
    } while (0)
    TRY(cudaMalloc(&b.padded, h_padded.size()));
    TRY(cudaMalloc((void**)&b.spatial, sizeof(float) * (size_t)nblocks * T * B * B));
    TRY(cudaMalloc((void**)&b.freq, sizeof(cufftComplex) * (size_t)nblocks * T * B * X));
    TRY(cudaMalloc((void**)&b.window, sizeof(float) * win.size()));
    TRY(cudaMalloc((void**)&b.sigma, sizeof(float) * sig.size()));
    TRY(cudaMalloc((void**)&b.wf, sizeof(float) * wf.size()));
    TRY(cudaMemcpy(b.padded, h_padded.data(), h_padded.size(), cudaMemcpyHostToDevice));
    TRY(cudaMemcpy(b.window, win.data(), sizeof(float) * win.size(), cudaMemcpyHostToDevice));
    TRY(cudaMemcpy(b.sigma, sig.data(), sizeof(float) * sig.size(), cudaMemcpyHostToDevice));
    TRY(cudaMemcpy(b.wf, wf.data(), sizeof(float) * wf.size(), cudaMemcpyHostToDevice));

    int fft_size[3] = {T, B, B};
    const int spatial_only = radius == 0;
    TRYF(cufftPlanMany(&b.r2c, 3 - spatial_only, &fft_size[spatial_only], nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C,
                       nblocks));
    TRYF(cufftPlanMany(&b.c2r, 3 - spatial_only, &fft_size[spatial_only], nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R,
                       nblocks));
    b.plans = true;

    int dev = 0, sms = 0, occ = 0;
    TRY(cudaGetDevice(&dev));
    TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int threads = 128;
    const int padded_block_size = B;
    if (bps == 1) {
        TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, im2col_u8, threads, 0));
        im2col_u8<<<sms * std::max(occ, 1), threads>>>(b.spatial, (const uint8_t*)b.padded, b.window, scale, radius,
                                                       B, S, padded_block_size, width, height);
    } else if (bps == 2) {
        TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, im2col_u16, threads, 0));
        im2col_u16<<<sms * std::max(occ, 1), threads>>>(b.spatial, (const uint16_t*)b.padded, b.window, scale, radius,
                                                        B, S, padded_block_size, width, height);
    } else {
        TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, im2col_f32, threads, 0));
        im2col_f32<<<sms * std::max(occ, 1), threads>>>(b.spatial, (const float*)b.padded, b.window, scale, radius,
                                                        B, S, padded_block_size, width, height);
    }
    TRY(cudaGetLastError());
    TRYF(cufftExecR2C(b.r2c, b.spatial, b.freq));
    auto filter = zero_mean ? frequency_filtering_zm1 : frequency_filtering_zm0;
    TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)filter, threads, 0));
    filter<<<sms * std::max(occ, 1), threads>>>((float2*)b.freq, nblocks, radius, B, b.wf, b.sigma, sigma_scalar,
                                                 sigma_is_scalar, (float)sigma2, (float)pmin, (float)pmax,
                                                 filter_type);
    TRY(cudaGetLastError());
    TRYF(cufftExecC2R(b.c2r, b.freq, b.spatial));
    dim3 grid((pw + 31) / 32, (ph + 3) / 4), block(32, 4);
    if (bps == 1)
        col2im_u8<<<grid, block>>>((uint8_t*)b.padded, b.spatial, b.window, scale, peak, radius, B, S,
                                   padded_block_size, width, height);
    else if (bps == 2)
        col2im_u16<<<grid, block>>>((uint16_t*)b.padded, b.spatial, b.window, scale, peak, radius, B, S,
                                    padded_block_size, width, height);
    else
        col2im_f32<<<grid, block>>>((float*)b.padded, b.spatial, b.window, scale, peak, radius, B, S,
                                    padded_block_size, width, height);
    TRY(cudaGetLastError());
    TRY(cudaMemcpy(h_padded.data(), b.padded, h_padded.size(), cudaMemcpyDeviceToHost));
    const int oy = (ph - height) / 2, ox = (pw - width) / 2;
    const uint8_t* slice = h_padded.data() + plane_elems * radius * bps;
    for (int y = 0; y < height; ++y)
        std::memcpy((uint8_t*)dst + (size_t)y * dst_stride * bps, slice + ((size_t)(oy + y) * pw + ox) * bps,
                    (size_t)width * bps);
    return 0;
#undef TRY
#undef TRYF
}

}  // extern "C"
