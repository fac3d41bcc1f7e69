// Host-side pieces shared by the translation units of the library: error
// reporting, and the factories of the kernel variants.  The kernels are
// compiled in separate units (one per block size for the unit kernel, one for
// the adjoint, one for the tensor-core form) so that they build in parallel;
// dfttest_capi.cu holds the host logic and reaches them only through the
// function pointers and launchers declared here.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "dfttest2_b200.h"
#include "dfttest_adjoint.cuh"
#include "dfttest_kernel.cuh"
#include "dfttest_tc.cuh"

namespace dft2h {

// records the message of a failing call for dfttest2_b200_last_error (per thread)
int fail(int code, const std::string& msg);

// Raises the kernel's dynamic shared-memory limit to `smem` (once per
// device, kernel and size) and, when per_sm is given, returns its resident
// CTAs per SM for `threads` threads (cached: the runtime queries cost more
// than a small launch).
int prepare_kernel(const void* kern, size_t smem, int threads, int* per_sm);

#define CUDA_TRY(expr)                                                                                   \
    do {                                                                                                 \
        cudaError_t e_ = (expr);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            return ::dft2h::fail(DFTTEST2_B200_ECUDA, std::string("[") + std::to_string(__LINE__) +      \
                                                          "] '" #expr "' failed: " + cudaGetErrorString(e_)); \
        }                                                                                                \
    } while (0)

using KernelFn = void (*)(const dft2::KernelArgs);

// one compiled shape of the unit kernel
struct Variant {
    KernelFn main = nullptr;      // Wiener fast path
    KernelFn generic = nullptr;   // every filter type, asymmetric sigma
    KernelFn fixup = nullptr;
    int nw = 0;      // warps per CTA
    int bpw = 0;     // blocks per warp
    int minb = 1;    // CTAs per SM the register budget is sized for
    size_t (*smem)(int pitch) = nullptr;
};

// The unit-kernel shape (B, T, warps per CTA, CTAs per SM), or an empty
// Variant when that shape is not compiled (inst_unit_b8/16/32.cu).
Variant unit_variant(int B, int T, int NW, int MINB);
Variant unit_variant_b8(int T, int NW, int MINB);
Variant unit_variant_b16(int T, int NW, int MINB);
Variant unit_variant_b32(int T, int NW, int MINB);

// adjoint kernel and the sigma-table kernel of the differentiable path (inst_adjoint.cu)
int adjoint_tile_dims(int B, int T, int& tbx, int& tby);
int launch_adjoint(int B, int T, const dft2::AdjointArgs& a, int num_sms, cudaStream_t st);
int launch_sigma_tables(const float* sigma, const int* idx, const int* idx2, float* tab, float* tab2, int n,
                        cudaStream_t st);

// tensor-core form (inst_tc.cu)
using TcKernelFn = void (*)(const dft2::TcArgs);
struct TcVariant {
    TcKernelFn wiener = nullptr, generic = nullptr;
    size_t (*smem)(int patch_w) = nullptr;
    int gbytes = 0;
    int tb = 0;  // blocks per tile
    void (*build)(std::vector<char>&) = nullptr;
};
TcVariant select_tc(int B, int T, int mode);
int launch_tc_finalize(const dft2::TcArgs& a, dim3 grid, cudaStream_t st);

// tensor-core strip form (inst_tc2.cu): 16x16 blocks, radius 0 or 1, block
// steps 1, 2, 4, separable windows; runs in the unit framework (same plans,
// band records, seams and fix-up kernel as the FP32 unit kernel)
struct Tc2Input {
    int T, S, radius, syn;
    const double* window;  // [T][16][16]
    const double* wfreq;   // [T][16][9][2] window spectrum, null without zero-mean
    const float* sigma;    // [T][16][9]
    int fmt;               // kTc2FmtFp16 / kTc2FmtBf16
};
constexpr int kTc2FmtFp16 = 0, kTc2FmtBf16 = 1;  // dft2::kTc2Fp16 / kTc2Bf16 of dfttest_tc2.cuh
struct Tc2Shape {
    int nbx = 0;       // blocks per strip
    int xg = 0;        // 8-column groups of a strip footprint the kernel reads
    size_t smem = 0;   // dynamic shared memory per CTA
};
// Builds the constant image; non-zero (with the reason) when the arguments
// are outside the form.
int tc2_build(const Tc2Input& in, std::vector<char>& img, Tc2Shape& shape, std::string& why);
Variant tc2_variant(int T, int fmt, int S);

}  // namespace dft2h
