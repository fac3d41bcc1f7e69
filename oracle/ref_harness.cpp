// TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// Harness that runs the reference's own CPU math (vs-dfttest2
// gcc_source/kernel.hpp, compiled unchanged from the reference tree by
// oracle/Makefile into oracle/_ref/libdfttest_ref.so) on one plane.
//
// kernel.hpp holds the FFT codelets, frequency_filtering and fused() that
// dfttest2_cpu uses (cpu_source/kernel.hpp:16-1983; the GCC twin differs only
// in its SIMD wrapper).  The per-frame driver around it lives in
// cpu_source/getframe_impl.cpp and needs the VapourSynth SDK, which is not
// available, so this file restates it without VapourSynth:
//   calc_pad_size / calc_pad_num   getframe_impl.cpp:11-20
//   reflection padding             getframe_impl.cpp:22-65
//   load_block                     getframe_impl.cpp:105-156
//   store_block                    getframe_impl.cpp:158-175  (synthesis
//                                  window slice 2*radius, as the CPU backend)
//   store_frame                    getframe_impl.cpp:177-221
//   block loop / table conversion  getframe_impl.cpp:311-403,
//                                  cpu_source/source.cpp:146-203
// FTZ/DAZ is enabled around the call as dfttest2_cpu does
// (getframe_impl.cpp:251-252).
#include <xmmintrin.h>
#include <pmmintrin.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "kernel.hpp"

namespace {

int pad_size(int size, int B, int S) { return size + ((size % B) ? B - size % B : 0) + std::max(B - S, S) * 2; }
int pad_num(int size, int B, int S) { return (pad_size(size, B, S) - B) / S + 1; }

template <typename T>
void reflect(T* dst, const T* src, int width, int height, int stride, int B, int S) {
    const int pw = pad_size(width, B, S), ph = pad_size(height, B, S);
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

}  // namespace

extern "C" {

// src: 2r+1 planes (time clamp applied by the caller), element strides.
// sample_type 0 = integer (bits 8..16), 1 = float.  window: (2r+1)*256,
// sigma: (2r+1)*16*9 (a flat sigma is expanded by the caller, as
// python/dfttest2.py:364 does for this backend), window_freq:
// (2r+1)*16*9*2 interleaved, all FP64 as the plugin receives them.
// Returns 0 on success.
int ref_dfttest_plane(const void* const* src, int width, int height, int src_stride, int sample_type, int bits,
                           void* dst, int dst_stride, const double* window, const double* sigma, double sigma2,
                           double pmin, double pmax, int filter_type, int zero_mean, const double* window_freq,
                           int radius, int block_step) {
    constexpr int B = 16;
    const int S = block_step;
    const int T = 2 * radius + 1;
    if (radius < 0 || radius > 3 || S < 1 || S > B) return -1;
    const int bps = sample_type == 1 ? 4 : (bits <= 8 ? 1 : 2);

    // tables as DFTTestCreate builds them (cpu_source/source.cpp:146-203)
    Vec16f* win = static_cast<Vec16f*>(std::aligned_alloc(64, T * 16 * sizeof(Vec16f)));
    Vec16f* sig = static_cast<Vec16f*>(std::aligned_alloc(64, T * 16 * sizeof(Vec16f)));
    Vec16f* wf = static_cast<Vec16f*>(std::aligned_alloc(64, T * 32 * sizeof(Vec16f)));
    for (int i = 0; i < T * 16; ++i)
        for (int j = 0; j < 16; ++j) win[i][j] = static_cast<float>(window[i * 16 + j]);
    for (int i = 0; i < T * 16; ++i) {
        for (int j = 0; j < 16; ++j) sig[i][j] = j < 9 ? static_cast<float>(sigma[i * 9 + j]) : 0.0f;
    }
    for (int i = 0; i < T * 32; ++i)
        for (int j = 0; j < 16; ++j) wf[i][j] = 0.0f;
    if (zero_mean) {
        for (int i = 0; i < T * 16; ++i) {
            for (int j = 0; j < 9; ++j) {
                wf[i * 2][j] = static_cast<float>(window_freq[(i * 9 + j) * 2]);
                wf[i * 2 + 1][j] = static_cast<float>(window_freq[(i * 9 + j) * 2 + 1]);
            }
        }
    }

    const unsigned int mxcsr = _mm_getcsr();
    _mm_setcsr(mxcsr | 0x8040);  // FTZ | DAZ

    const int pw = pad_size(width, B, S), ph = pad_size(height, B, S);
    std::vector<uint8_t> padded((size_t)T * pw * ph * bps);
    std::vector<float> acc((size_t)pw * ph, 0.0f);
    for (int t = 0; t < T; ++t) {
        uint8_t* d = &padded[(size_t)t * pw * ph * bps];
        if (bps == 1)
            reflect((uint8_t*)d, (const uint8_t*)src[t], width, height, src_stride, B, S);
        else if (bps == 2)
            reflect((uint16_t*)d, (const uint16_t*)src[t], width, height, src_stride, B, S);
        else
            reflect((uint32_t*)d, (const uint32_t*)src[t], width, height, src_stride, B, S);
    }
    float scale = 1.0f / (1 << (bits - 8));
    if (sample_type == 1) scale = 255.0f;

    alignas(64) Vec16f block[7 * 16 * 2];
    for (int i = 0; i < pad_num(height, B, S); ++i) {
        for (int j = 0; j < pad_num(width, B, S); ++j) {
            const size_t off = (size_t)(i * pw + j) * S;
            // load_block
            for (int t = 0; t < T; ++t) {
                for (int y = 0; y < 16; ++y) {
                    const size_t base = (size_t)(t * ph + y) * pw + off;
                    Vec16f v;
                    for (int x = 0; x < 16; ++x) {
                        if (bps == 1) v[x] = (float)padded[base + x];
                        else if (bps == 2) v[x] = (float)((const uint16_t*)padded.data())[base + x];
                        else v[x] = ((const float*)padded.data())[base + x];
                    }
                    block[t * 32 + y] = scale * win[t * 16 + y] * v;
                }
            }
            fused(block, sig, (float)sigma2, (float)pmin, (float)pmax, filter_type, zero_mean != 0, wf, radius);
            // store_block with the CPU backend's synthesis slice (radius*512 floats = slice 2r)
            const Vec16f* sw = &win[2 * radius * 16];
            for (int y = 0; y < 16; ++y) {
                float* a = &acc[off + (size_t)y * pw];
                Vec16f o = block[radius * 32 + y];
                for (int x = 0; x < 16; ++x) a[x] = o[x] * sw[y][x] + a[x];
            }
        }
    }
    // store_frame
    const int oy = (ph - height) / 2, ox = (pw - width) / 2;
    const int peak = (1 << bits) - 1;
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            const float v = acc[(size_t)(oy + y) * pw + ox + x];
            if (bps == 4) {
                ((float*)dst)[(size_t)y * dst_stride + x] = v / scale;
            } else {
                const int q = std::clamp(static_cast<int>(v / scale + 0.5f), 0, peak);
                if (bps == 1) ((uint8_t*)dst)[(size_t)y * dst_stride + x] = (uint8_t)q;
                else ((uint16_t*)dst)[(size_t)y * dst_stride + x] = (uint16_t)q;
            }
        }
    }
    _mm_setcsr(mxcsr);
    std::free(win);
    std::free(sig);
    std::free(wf);
    return 0;
}

}  // extern "C"
