// Tensor-core form: constant operand images, kernel shapes and the
// accumulator conversion kernel (one translation unit).
#include <cmath>
#include <cstring>

#include "dfttest_host.h"

namespace dft2 {

// accumulator planes -> output samples (store_frame, cpu_source/getframe_impl.cpp:177-221)
__global__ void __launch_bounds__(256) dfttest_tc_finalize(const __grid_constant__ TcArgs a) {
    const int j = blockIdx.y;
    const TcJob& job = a.jobs[j];
    const long long n = (long long)job.width * job.height;
    const float inv_scale = 1.0f / a.p.scale;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / job.width), x = (int)(i - (long long)y * job.width);
        store_sample(job.dst, (long long)y * job.dst_stride + x, job.acc[i], a.p.kind, a.p.scale, a.p.peak,
                     a.p.kind == kF32 ? 0.0f : inv_scale);
    }
}

}  // namespace dft2

namespace dft2h {

// the constant operands (N x K, K-major canonical layout) of the four products
template <int B, int T, int MODE>
void build_gmat(std::vector<char>& img) {
    using L = dft2::TcLayout<B, T, MODE>;
    constexpr int ESZ = L::ESZ;
    img.assign(L::GBYTES, 0);
    const double pi = 3.14159265358979323846;
    auto put = [&](int off, int n, int k, int KT, double v) {
        const int idx = off + dft2::op_index<ESZ>(n, k, KT);
        if (MODE == dft2::kTcTf32) {
            // round to the 10-bit tf32 mantissa, nearest even (the tensor cores would truncate)
            const float f = (float)v;
            uint32_t u;
            std::memcpy(&u, &f, 4);
            u = (u + 0x0FFFu + ((u >> 13) & 1u)) & ~0x1FFFu;
            std::memcpy(&img[(size_t)idx * 4], &u, 4);
        } else {
            const __nv_bfloat16 h = __float2bfloat16_rn((float)v);
            std::memcpy(&img[(size_t)idx * 2], &h, 2);
            if (MODE == dft2::kTcBf16x3) {
                const __nv_bfloat16 l = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
                std::memcpy(&img[(size_t)(L::GELEM + idx) * 2], &l, 2);
            }
        }
    };
    // G1: packed r2c of a row, [j][x]
    for (int j = 0; j < B; ++j)
        for (int x = 0; x < B; ++x) {
            const int k = j < 2 ? (j == 0 ? 0 : B / 2) : j / 2;
            const double ang = 2.0 * pi * k * x / B;
            put(L::g1, j, x, B, j < 2 ? std::cos(ang) : ((j & 1) ? -std::sin(ang) : std::cos(ang)));
        }
    // G2: forward complex DFT over y in real form, [(c', ky)][(c, y)]
    for (int cp = 0; cp < 2; ++cp)
        for (int ky = 0; ky < B; ++ky)
            for (int c = 0; c < 2; ++c)
                for (int y = 0; y < B; ++y) {
                    const double th = 2.0 * pi * (double)(ky * y % B) / B;
                    const double v = cp == c ? std::cos(th) : (c == 1 ? std::sin(th) : -std::sin(th));
                    put(L::g2, cp * B + ky, c * B + y, 2 * B, v);
                }
    // G4: inverse complex DFT over y, [(c', y)][(c, ky)]
    for (int cp = 0; cp < 2; ++cp)
        for (int y = 0; y < B; ++y)
            for (int c = 0; c < 2; ++c)
                for (int ky = 0; ky < B; ++ky) {
                    const double ph = 2.0 * pi * (double)(ky * y % B) / B;
                    const double v = cp == c ? std::cos(ph) : (c == 1 ? -std::sin(ph) : std::sin(ph));
                    put(L::g4, cp * B + y, c * B + ky, 2 * B, v);
                }
    // G5: c2r of a packed row, [x][j]
    for (int x = 0; x < B; ++x)
        for (int j = 0; j < B; ++j) {
            const int k = j < 2 ? (j == 0 ? 0 : B / 2) : j / 2;
            const double ang = 2.0 * pi * (double)(k * x % B) / B;
            put(L::g5, x, j, B, j < 2 ? std::cos(ang) : ((j & 1) ? -2.0 * std::sin(ang) : 2.0 * std::cos(ang)));
        }
}

template <int B, int T, int MODE>
TcVariant make_tc() {
    TcVariant v;
    v.wiener = dft2::dfttest_tc_kernel<B, T, MODE, dft2::kFilterWiener>;
    v.generic = dft2::dfttest_tc_kernel<B, T, MODE, dft2::kFilterGeneric>;
    v.smem = [](int pw) { return dft2::TcLayout<B, T, MODE>::bytes(pw); };
    v.gbytes = dft2::TcLayout<B, T, MODE>::GBYTES;
    v.tb = dft2::TcLayout<B, T, MODE>::TB;
    v.build = build_gmat<B, T, MODE>;
    return v;
}

template <int B, int T>
TcVariant select_tc_mode(int mode) {
    switch (mode) {
    case dft2::kTcBf16x3: return make_tc<B, T, dft2::kTcBf16x3>();
    case dft2::kTcTf32: return make_tc<B, T, dft2::kTcTf32>();
    case dft2::kTcBf16: return make_tc<B, T, dft2::kTcBf16>();
    }
    return TcVariant{};
}

TcVariant select_tc(int B, int T, int mode) {
    if (B == 16 && T == 1) return select_tc_mode<16, 1>(mode);
    if (B == 16 && T == 3) return select_tc_mode<16, 3>(mode);
    if (B == 32 && T == 1) return select_tc_mode<32, 1>(mode);
    return TcVariant{};
}

int launch_tc_finalize(const dft2::TcArgs& a, dim3 grid, cudaStream_t st) {
    dft2::dfttest_tc_finalize<<<grid, 256, 0, st>>>(a);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace dft2h
