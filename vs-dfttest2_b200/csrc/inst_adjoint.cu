// Adjoint kernel of the differentiable path and the kernel that rebuilds the
// gain-slot sigma tables from a device sigma array (one translation unit).
#include <algorithm>

#include "dfttest_host.h"

namespace dft2 {

// builds the gain-slot sigma tables of the forward kernel from a device sigma array
__global__ void __launch_bounds__(256) sigma_tables_kernel(const float* __restrict__ sigma, const int* __restrict__ idx,
                                                           const int* __restrict__ idx2, float* __restrict__ tab,
                                                           float* __restrict__ tab2, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        tab[i] = sigma[idx[i]];
        tab2[i] = sigma[idx2[i]];
    }
}

}  // namespace dft2

namespace dft2h {

template <int B, int T>
int launch_adjoint_t(dft2::AdjointArgs a, int num_sms, cudaStream_t st) {
    using L = dft2::AdjTile<B, T>;
    a.patch_h = B + (L::TBY - 1) * a.block_step;
    a.patch_w = B + (L::TBX - 1) * a.block_step;
    const size_t smem = L::smem_bytes(a.patch_h, a.patch_w);
    auto kern = dft2::dfttest_adjoint_kernel<B, T>;
    int per_sm = 0;
    if (int rc = prepare_kernel((const void*)kern, smem, L::NTH, &per_sm)) return rc;
    if (per_sm < 1) return fail(DFTTEST2_B200_ECUDA, "adjoint kernel does not fit on an SM");
    const int grid = std::max(1, std::min(a.ntiles, num_sms * per_sm));
    kern<<<grid, L::NTH, smem, st>>>(a);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

template <int B, int T>
void adjoint_tile_dims_t(int& tbx, int& tby) {
    tbx = dft2::AdjTile<B, T>::TBX;
    tby = dft2::AdjTile<B, T>::TBY;
}

#define DFT2_FOR_ADJ_VARIANTS(M) M(16, 1) M(16, 3) M(16, 5) M(16, 7)
#define DFT2_FOR_ADJ_MORE(M) M(8, 1) M(8, 3) M(8, 5) M(8, 7) M(32, 1) M(32, 3) M(32, 5) M(32, 7)

int adjoint_tile_dims(int B, int T, int& tbx, int& tby) {
#define DFT2_ADJ(b, t) \
    if (B == b && T == t) return adjoint_tile_dims_t<b, t>(tbx, tby), 0;
    DFT2_FOR_ADJ_VARIANTS(DFT2_ADJ) DFT2_FOR_ADJ_MORE(DFT2_ADJ)
#undef DFT2_ADJ
    return fail(DFTTEST2_B200_EINVAL, "unsupported block_size / radius");
}

int launch_adjoint(int B, int T, const dft2::AdjointArgs& a, int num_sms, cudaStream_t st) {
#define DFT2_ADJ(b, t) \
    if (B == b && T == t) return launch_adjoint_t<b, t>(a, num_sms, st);
    DFT2_FOR_ADJ_VARIANTS(DFT2_ADJ) DFT2_FOR_ADJ_MORE(DFT2_ADJ)
#undef DFT2_ADJ
    return fail(DFTTEST2_B200_EINVAL, "unsupported block_size / radius");
}

int launch_sigma_tables(const float* sigma, const int* idx, const int* idx2, float* tab, float* tab2, int n,
                        cudaStream_t st) {
    dft2::sigma_tables_kernel<<<(n + 255) / 256, 256, 0, st>>>(sigma, idx, idx2, tab, tab2, n);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace dft2h
