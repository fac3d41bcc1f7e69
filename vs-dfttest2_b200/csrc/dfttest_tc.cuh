// Tensor-core form of the DFTTest per-block pipeline: the transforms of
// cpu_source/kernel.hpp:1899-1983 (fused) as dense products on the sm_100a
// 5th-generation tensor cores (tcgen05.mma, operands in shared memory,
// accumulators in tensor memory), with the elementwise work (operand
// re-layout, hi/lo split, zero-mean, gain, temporal inverse of the centre
// frame, synthesis window, overlap-add) on the CUDA cores.
//
// A tile is TB = 128 / B neighbouring blocks of one block row.  Per tile:
//   G1  row r2c          rows (blk, y)   K = B (x)        N = B (packed bins j)   one product per frame t
//   G2  column DFT       rows (blk, kx)  K = (c, y) 2B    N = (c, ky) 2B          one product per frame t
//       (kx padded to B rows, rows kx > B/2 unused; the operand is MN-major so
//       that each thread writes whole 16-byte chunks of the row spectra it holds)
//   --  temporal DFT, zero-mean, gain, inverse over t of the centre frame
//       (CUDA cores; the T products of a bin sit in one tensor-memory lane)
//   G4  inverse col DFT  rows (blk, kx)  K = (c, ky) 2B   N = (c, y) 2B
//   G5  c2r              rows (blk, y)   K = B (packed j) N = B (x)   (A MN-major)
// Packed bins j of a real row: j = 0 -> Re X0, 1 -> Re X_{B/2}, 2k -> Re Xk,
// 2k + 1 -> Im Xk (k = 1 .. B/2 - 1); c2r ignores Im X0 and Im X_{B/2}.
//
// Precision modes: BF16X3 splits every operand into bf16 hi + lo and sums
// hi*hi + hi*lo + lo*hi in FP32 (three MMAs per K step); BF16 and TF32 use
// one MMA per K step.  Accumulation is FP32 in tensor memory.
//
// The overlap-add of a tile is summed in shared memory and added to a float
// accumulator plane in global memory (atomic adds); a second kernel converts
// the accumulators to the output format.
#pragma once

#include <cuda_bf16.h>

#include "dfttest_kernel.cuh"
#include "dfttest_adjoint.cuh"  // cdft_n

namespace dft2 {

enum TcMode { kTcOff = 0, kTcBf16x3 = 1, kTcTf32 = 2, kTcBf16 = 3 };

struct TcJob {
    const void* src[7];
    void* dst;
    float* acc;             // accumulator plane, width x height floats (zeroed before the launch)
    long long src_stride, dst_stride;  // elements
    int width, height;
    int tile_base;          // first global tile id
    int ntx;                // tiles per block row
};

struct TcArgs {
    const TcJob* jobs;
    int njobs;
    int ntiles;
    int block_step;
    FilterParams p;
    const float* sigma;     // [T][B][X]
    const float* wf;        // [T][B][X][2]
    const void* gmat;       // the four constant operands, shared-memory image
    int gmat_bytes;
    int* error_flag;
    int wait_limit;         // iteration limit of the in-loop waits for the tensor cores
};

// ---- PTX wrappers (tcgen05) ------------------------------------------------
// shared-memory matrix descriptor: K-major, no swizzle (8-row x 16-byte core
// matrices; lbo = byte step between core matrices along K, sbo = along M/N)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, swizzle none
}

// instruction descriptor of kind::f16 / kind::tf32: D f32, A and B K-major
__host__ __device__ constexpr uint32_t idesc(int ab_format, int M, int N, bool a_mn_major = false) {
    return (1u << 4)                       // D format f32
           | ((uint32_t)ab_format << 7)    // A format (1 = bf16, 2 = tf32)
           | ((uint32_t)ab_format << 10)   // B format
           | ((a_mn_major ? 1u : 0u) << 15)  // A major: 0 = K, 1 = MN
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

template <bool TF32>
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    const uint32_t z = 0;
    if constexpr (TF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
            :: "r"(d_tmem), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(z));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
            :: "r"(d_tmem), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(z));
    }
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 8 consecutive 32-bit columns of this thread's lane
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld1(uint32_t taddr, float& v) {
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
    v = __uint_as_float(r);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- operand layouts -------------------------------------------------------
// element (m, k) of a K-major operand with KT columns, in elements of ESZ bytes
template <int ESZ>
__host__ __device__ constexpr int op_index(int m, int k, int KT) {
    constexpr int PER = 16 / ESZ;  // elements per 16-byte core-matrix row
    return (((m >> 3) * (KT / PER) + k / PER) * 8 + (m & 7)) * PER + (k % PER);
}

// element (m, k) of an MN-major operand with MT rows: 8 k-rows of 16 bytes (16/ESZ
// consecutive m) per core matrix; m-groups 128 bytes apart, k-groups MT/(16/ESZ) * 128 bytes
template <int ESZ>
__host__ __device__ constexpr int op_index_mn(int m, int k, int MT) {
    constexpr int PER = 16 / ESZ;
    return ((k / 8) * (MT / PER) + m / PER) * (8 * PER) + (k % 8) * PER + (m % PER);
}

// operand store of one value: bf16 hi (+ lo) or tf32 (fp32 bits)
template <int MODE>
struct Operand {
    static constexpr bool TF = MODE == kTcTf32;
    static constexpr int ESZ = TF ? 4 : 2;
    static constexpr bool SPLIT = MODE == kTcBf16x3;
};

// fp32 -> tf32, rounded to nearest (the tensor cores would truncate the low mantissa bits)
__device__ __forceinline__ float to_tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return __uint_as_float(r);
}

// operand buffers hold a hi plane and (BF16X3) a lo plane `lo_off` bytes later
template <int MODE>
__device__ __forceinline__ void put(char* base, int lo_off, int idx, float v) {
    if constexpr (MODE == kTcTf32) {
        reinterpret_cast<float*>(base)[idx] = to_tf32(v);
    } else {
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        reinterpret_cast<__nv_bfloat16*>(base)[idx] = h;
        if constexpr (MODE == kTcBf16x3)
            reinterpret_cast<__nv_bfloat16*>(base + lo_off)[idx] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

// 8 consecutive K values of one row (one 16-byte core-matrix row for bf16)
template <int MODE>
__device__ __forceinline__ void put8(char* base, int lo_off, int idx, const float (&v)[8]) {
    if constexpr (MODE == kTcTf32) {
        float4* p = reinterpret_cast<float4*>(reinterpret_cast<float*>(base) + idx);
        // idx is a multiple of 4; the two halves lie in consecutive core matrices along K
        p[0] = make_float4(to_tf32(v[0]), to_tf32(v[1]), to_tf32(v[2]), to_tf32(v[3]));
        reinterpret_cast<float4*>(reinterpret_cast<float*>(base) + idx + 32)[0] =
            make_float4(to_tf32(v[4]), to_tf32(v[5]), to_tf32(v[6]), to_tf32(v[7]));
    } else {
        __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            h[i] = __float2bfloat16_rn(v[i]);
            l[i] = __float2bfloat16_rn(v[i] - __bfloat162float(h[i]));
        }
        *reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(base) + idx) = *reinterpret_cast<const uint4*>(h);
        if constexpr (MODE == kTcBf16x3)
            *reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(base + lo_off) + idx) =
                *reinterpret_cast<const uint4*>(l);
    }
}

// 8 consecutive M values (m0 a multiple of 8) of one K column of a 128-row MN-major
// operand (16-bit types: the tensor cores read MN-major operands of bf16, not tf32)
template <int MODE>
__device__ __forceinline__ void put8_mn(char* base, int lo_off, int m0, int k, const float (&v)[8]) {
    static_assert(MODE != kTcTf32, "tf32 operands are K-major");
    put8<MODE>(base, lo_off, op_index_mn<2>(m0, k, 128), v);
}

// shared-memory plan of the tensor-core kernel (bytes)
template <int B, int T, int MODE>
struct TcLayout {
    static constexpr int ESZ = Operand<MODE>::ESZ;
    static constexpr int NPLANE = Operand<MODE>::SPLIT ? 2 : 1;
    static constexpr int X = B / 2 + 1;
    static constexpr int TB = 128 / B;       // blocks per tile
    // constant operands (N x K each, K-major), hi planes then lo planes
    static constexpr int G1 = B * B, G2 = 4 * B * B, G4 = 4 * B * B, G5 = B * B;
    static constexpr int GELEM = G1 + G2 + G4 + G5;
    static constexpr int g1 = 0, g2 = G1, g4 = G1 + G2, g5 = G1 + G2 + G4;  // element offsets in a plane
    static constexpr int GBYTES = GELEM * ESZ * NPLANE;
    // A operand region: the largest stage (A1, A2 have T planes)
    static constexpr int A1 = T * 128 * B, A2 = T * 128 * 2 * B, A4 = 128 * 2 * B, A5 = 128 * B;
    static constexpr int AELEM = A1 > A2 ? (A1 > A4 ? A1 : A4) : (A2 > A4 ? A2 : A4);
    static constexpr int ABYTES = AELEM * ESZ * NPLANE;
    static constexpr int o_g = 0;
    static constexpr int o_a = (o_g + GBYTES + 127) & ~127;
    static constexpr int o_tab = (o_a + ABYTES + 127) & ~127;  // floats from here
    // float tables: scale * window [T][B][B], wsyn [B][B], sigma and WF as [kx][kt][ky]
    static constexpr int F_WIN = 0, F_WSYN = T * B * B, F_SIG = F_WSYN + B * B, F_WF = F_SIG + X * T * B;
    static constexpr int F_END = F_WF + 2 * X * T * B;
    static constexpr int o_patch = o_tab + 4 * F_END;  // input rows [T][B][patch_w], then the overlap-add tile [B][patch_w]
    static size_t bytes(int patch_w) { return (size_t)o_patch + 4 * (size_t)(T + 1) * B * patch_w + 64; }
};

template <int B, int T, int MODE, int FC>
__global__ void __launch_bounds__(256, 2) dfttest_tc_kernel(const __grid_constant__ TcArgs a) {
    using L = TcLayout<B, T, MODE>;
    constexpr bool TF = MODE == kTcTf32;
    constexpr int ESZ = L::ESZ;
    constexpr int X = L::X, TB = L::TB;
    constexpr int NT = 256;
    constexpr int KSTEP = TF ? 8 : 16;  // K per MMA
    extern __shared__ __align__(128) char tc_smem[];
    char* smem = tc_smem;
    __shared__ uint64_t s_bar;
    __shared__ uint32_t s_tmem;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int row = ((warp & 3) << 5) | (tid & 31);  // tensor-memory lane of this thread
    const int half = warp >> 2;                       // which half of the columns this thread handles
    const int S = a.block_step;
    const FilterParams& P = a.p;

    char* g_hi = smem + L::o_g;
    char* a_hi = smem + L::o_a;
    constexpr int G_LO = L::GELEM * ESZ;  // lo plane offsets (BF16X3)
    constexpr int A_LO = L::AELEM * ESZ;
    float* tab = reinterpret_cast<float*>(smem + L::o_tab);
    float* s_win = tab + L::F_WIN;
    float* s_wsyn = tab + L::F_WSYN;
    float* s_sig = tab + L::F_SIG;
    float* s_wf = tab + L::F_WF;
    const int PWID = B + (TB - 1) * S;                // patch width
    float* s_patch = reinterpret_cast<float*>(smem + L::o_patch);
    float* s_ola = s_patch + T * B * PWID;

    // ---- one-time set-up: constants, tables, barrier, tensor memory
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.gmat);
        uint4* dst = reinterpret_cast<uint4*>(g_hi);
        for (int i = tid; i < a.gmat_bytes / 16; i += NT) dst[i] = src[i];
    }
    for (int i = tid; i < T * B * B; i += NT) s_win[i] = P.scale * P.win[i];
    for (int i = tid; i < B * B; i += NT) s_wsyn[i] = P.wsyn[i];
    for (int i = tid; i < X * T * B; i += NT) {
        const int kx = i / (T * B), rem = i - kx * T * B;  // rem = kt * B + ky
        const int src = rem * X + kx;                        // [kt][ky][kx]
        s_sig[i] = a.sigma[src];
        s_wf[2 * i] = P.g_div != 0.0f ? a.wf[2 * src] : 0.0f;
        s_wf[2 * i + 1] = P.g_div != 0.0f ? a.wf[2 * src + 1] : 0.0f;
    }
    for (int i = tid; i < B * PWID; i += NT) s_ola[i] = 0.0f;
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&s_tmem)), "r"(256) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    constexpr uint32_t C_D1 = 0, C_D2 = 128, C_D4 = 0, C_D5 = 64;  // tensor-memory columns of the stages
    uint32_t phase = 0;
    bool s_fail_any = false;

    // issue `nk` K steps of D(128 x N) = A(128 x K) * G(N x K)^T for `count` operand slices
    // (slice i: A at a_off + i * a_step elements, D at d_col + i * d_step columns), one commit;
    // thread 0 waits for the tensor cores, the others at the barrier.  Returns false on a timeout.
    // A is K-major, or MN-major (a_mn) with 128 rows; G is K-major.
    auto gemm = [&](uint32_t d_col, int a_off, int a_kt, bool a_mn, int g_off, int n, int nk, int count = 1,
                    int a_step = 0, int d_step = 0) -> bool {
        bool ok = true;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t id = idesc(TF ? 2 : 1, 128, n, a_mn);
            const uint32_t g0 = smem_addr(g_hi) + g_off * ESZ;
            const uint32_t g_sbo = (a_kt * ESZ / 16) * 128;               // K-major: 8-row group stride
            const uint32_t a_lbo = a_mn ? (128 * ESZ / 16) * 128 : 128;   // K-direction core-matrix stride
            const uint32_t a_sbo = a_mn ? 128 : g_sbo;                    // M-direction core-matrix stride
            const uint32_t a_kstep = a_mn ? (KSTEP / 8) * a_lbo : 256;     // bytes per MMA K step
            for (int sl = 0; sl < count; ++sl) {
                const uint32_t a0 = smem_addr(a_hi) + (a_off + sl * a_step) * ESZ;
                const uint32_t d = tmem + d_col + sl * d_step;
                for (int s = 0; s < nk; ++s) {
                    const uint32_t gs = s * 256;  // two core matrices along K per MMA
                    const uint64_t ad = sdesc(a0 + s * a_kstep, a_lbo, a_sbo), gd = sdesc(g0 + gs, 128, g_sbo);
                    mma<TF>(d, ad, gd, id, s > 0 ? 1u : 0u);
                    if constexpr (MODE == kTcBf16x3) {
                        mma<TF>(d, ad, sdesc(g0 + G_LO + gs, 128, g_sbo), id, 1u);
                        mma<TF>(d, sdesc(a0 + A_LO + s * a_kstep, a_lbo, a_sbo), gd, id, 1u);
                    }
                }
            }
            mma_commit(&s_bar);
            ok = mbar_wait(&s_bar, phase, a.wait_limit);
            if (!ok) atomicExch(a.error_flag, 2);
        }
        phase ^= 1;
        const bool fail = __syncthreads_or(!ok);
        tc_fence_after();
        return !fail;
    };
    // all threads: operand writes visible to the tensor cores, tensor-memory reads done
    auto handoff = [&]() {
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
    };

    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        int lo = 0, hi = a.njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.jobs[mid].tile_base <= tile) lo = mid; else hi = mid - 1;
        }
        const TcJob& job = a.jobs[lo];
        const int W = job.width, Hh = job.height;
        const int pw = pad_size(W, B, S), ph = pad_size(Hh, B, S);
        const int pnx = (pw - B) / S + 1;
        const int ox = (pw - W) / 2, oy = (ph - Hh) / 2;
        const int lt = tile - job.tile_base;
        const int by = lt / job.ntx, tx = lt - by * job.ntx;
        const int bx0 = tx * TB;
        const int nb = min(TB, pnx - bx0);  // blocks of this tile
        const int py0 = by * S, px0 = bx0 * S;

        // ---- stage the input rows of the tile: [t][y][0, PWID), one warp per row
        for (int r = warp; r < T * B; r += NT / 32) {
            const int t = r / B, y = r - t * B;
            const long long rowoff = (long long)mirror(py0 + y - oy, Hh) * job.src_stride;
            for (int c = tid & 31; c < PWID; c += 32) {
                const int px = min(px0 + c, pw - 1);
                s_patch[r * PWID + c] = load_sample(job.src[t], rowoff + mirror(px - ox, W), P.kind);
            }
        }
        __syncthreads();
        // ---- A1: windowed rows, [t][row = blk * B + y][x]
        {
            const int blk = row / B, y = row % B;
#pragma unroll
            for (int t = 0; t < T; ++t) {
#pragma unroll
                for (int x8 = 0; x8 < B / 16; ++x8) {
                    const int xb = half * (B / 2) + x8 * 8;
                    float v[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        v[i] = s_win[(t * B + y) * B + xb + i] * s_patch[(t * B + y) * PWID + blk * S + xb + i];
                    put8<MODE>(a_hi, A_LO, t * 128 * B + op_index<ESZ>(row, xb, B), v);
                }
            }
        }
        handoff();
        bool ok = gemm(C_D1, 0, B, false, L::g1, B, B / KSTEP, T, 128 * B, B);  // D1[t] = rows of slice t
        if (!ok) {
            s_fail_any = true;
            break;
        }

        // ---- A2[t][(blk, kx)][(c, y)] (MN-major) from the packed row spectra: thread (blk, y)
        //      writes the real (half 0) or imaginary (half 1) parts of its row, kx = 0 .. B-1
        {
            const int blk = row / B, y = row % B;
#pragma unroll
            for (int t = 0; t < T; ++t) {
                float v[B];
#pragma unroll
                for (int j8 = 0; j8 < B / 8; ++j8) {
                    float w8[8];
                    tmem_ld8(tmem + lane_base + C_D1 + t * B + j8 * 8, w8);
#pragma unroll
                    for (int i = 0; i < 8; ++i) v[j8 * 8 + i] = w8[i];
                }
                tmem_wait_ld();
                char* base = a_hi + (size_t)t * 128 * 2 * B * ESZ;
#pragma unroll
                for (int q = 0; q < B / 8; ++q) {  // kx = 8q .. 8q+7
                    float c8[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int kx = 8 * q + i;
                        float re = 0.0f, im = 0.0f;
                        if (kx == 0) re = v[0];
                        else if (kx == B / 2) re = v[1];
                        else if (kx < B / 2) { re = v[2 * kx]; im = v[2 * kx + 1]; }
                        c8[i] = half ? im : re;
                    }
                    if constexpr (TF) {  // tf32 operands stay K-major (MN-major is for 16-bit types)
#pragma unroll
                        for (int i = 0; i < 8; ++i)
                            put<MODE>(base, A_LO, op_index<ESZ>(blk * B + 8 * q + i, half * B + y, 2 * B), c8[i]);
                    } else {
                        put8_mn<MODE>(base, A_LO, blk * B + 8 * q, half * B + y, c8);
                    }
                }
            }
        }
        handoff();
        ok = gemm(C_D2, 0, 2 * B, !TF, L::g2, 2 * B, 2 * B / KSTEP, T, 128 * 2 * B, 2 * B);
        if (!ok) {
            s_fail_any = true;
            break;
        }

        // ---- temporal DFT, zero-mean, gain, temporal inverse of the centre frame -> A4[(blk, kx)][(c, ky)]
        {
            const int blk = row / B, kx = row % B;
            // Re Z(kt 0, ky 0) of this row = sum over t of the column products at (c 0, ky 0)
            float z00 = 0.0f;
#pragma unroll
            for (int t = 0; t < T; ++t) {
                float z;
                tmem_ld1(tmem + lane_base + C_D2 + t * 2 * B, z);
                tmem_wait_ld();
                z00 += z;
            }
            const float dc = __shfl_sync(0xffffffffu, z00, (tid & 31) & ~(B - 1) & 31);
            const float g = P.g_div != 0.0f ? __fdiv_rn(dc, P.g_div) : 0.0f;
            // tensor-memory loads are warp-wide: every lane loads, rows kx > B/2 and blocks past the tile end discard
            const bool active = kx <= B / 2 && blk < nb;
            const int kxc = kx <= B / 2 ? kx : B / 2;
#pragma unroll
            for (int k8 = 0; k8 < B / 16; ++k8) {
                const int kb = half * (B / 2) + k8 * 8;
                float pr[T][8], pi[T][8];
#pragma unroll
                for (int t = 0; t < T; ++t) {
                    tmem_ld8(tmem + lane_base + C_D2 + t * 2 * B + kb, pr[t]);
                    tmem_ld8(tmem + lane_base + C_D2 + t * 2 * B + B + kb, pi[t]);
                }
                tmem_wait_ld();
                float yr[8], yi[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    float re[T], im[T];
#pragma unroll
                    for (int t = 0; t < T; ++t) {
                        re[t] = pr[t][i];
                        im[t] = pi[t][i];
                    }
                    if constexpr (T > 1) cdft_n<T>(re, im, false);
                    float sr = 0.0f, si = 0.0f;
#pragma unroll
                    for (int kt = 0; kt < T; ++kt) {
                        const int tb = (kxc * T + kt) * B + kb + i;
                        const float wr = s_wf[2 * tb], wi = s_wf[2 * tb + 1];
                        const float dre = fmaf(-g, wr, re[kt]), dim = fmaf(-g, wi, im[kt]);
                        const float psd = fmaf(dim, dim, dre * dre);
                        const float s = s_sig[tb];
                        const float m = FC == kFilterWiener ? gain<0>(psd, s, P) : gain_rt(P.filter_type, psd, s, P);
                        const float ur = fmaf(m, dre, g * wr), ui = fmaf(m, dim, g * wi);
                        // e^{+2 pi i kt r / T}
                        const float cs = CentreTwiddle<T>::re(kt), sn = CentreTwiddle<T>::im(kt);
                        sr += ur * cs - ui * sn;
                        si += ur * sn + ui * cs;
                    }
                    yr[i] = sr;
                    yi[i] = si;
                }
                if (active) {
                    put8<MODE>(a_hi, A_LO, op_index<ESZ>(row, kb, 2 * B), yr);
                    put8<MODE>(a_hi, A_LO, op_index<ESZ>(row, B + kb, 2 * B), yi);
                }
            }
        }
        handoff();
        ok = gemm(C_D4, 0, 2 * B, false, L::g4, 2 * B, 2 * B / KSTEP);
        if (!ok) {
            s_fail_any = true;
            break;
        }

        // ---- A5[(blk, y)][j] (MN-major): thread (blk, kx) writes its y-half of columns j(kx, re / im)
        {
            const int blk = row / B, kx = row % B;
#pragma unroll
            for (int y8 = 0; y8 < B / 16; ++y8) {
                const int yb = half * (B / 2) + y8 * 8;
                float vr[8], vi[8];
                tmem_ld8(tmem + lane_base + C_D4 + yb, vr);
                tmem_ld8(tmem + lane_base + C_D4 + B + yb, vi);
                tmem_wait_ld();
                if (kx <= B / 2) {
                    const int jr = kx == 0 ? 0 : (kx == B / 2 ? 1 : 2 * kx);
                    const bool pair = kx != 0 && kx != B / 2;
                    if constexpr (TF) {
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            put<MODE>(a_hi, A_LO, op_index<ESZ>(blk * B + yb + i, jr, B), vr[i]);
                            if (pair) put<MODE>(a_hi, A_LO, op_index<ESZ>(blk * B + yb + i, jr + 1, B), vi[i]);
                        }
                    } else {
                        put8_mn<MODE>(a_hi, A_LO, blk * B + yb, jr, vr);
                        if (pair) put8_mn<MODE>(a_hi, A_LO, blk * B + yb, jr + 1, vi);
                    }
                }
            }
        }
        handoff();
        ok = gemm(C_D5, 0, B, !TF, L::g5, B, B / KSTEP);
        if (!ok) {
            s_fail_any = true;
            break;
        }

        // ---- synthesis window and overlap-add of the tile
        {
            const int blk = row / B, y = row % B;
#pragma unroll
            for (int x8 = 0; x8 < B / 16; ++x8) {
                const int xb = half * (B / 2) + x8 * 8;
                float v[8];
                tmem_ld8(tmem + lane_base + C_D5 + xb, v);
                tmem_wait_ld();
                if (blk < nb) {
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        atomicAdd(&s_ola[y * PWID + blk * S + xb + i], v[i] * s_wsyn[y * B + xb + i]);
                }
            }
        }
        tc_fence_before();
        __syncthreads();
        for (int y = warp; y < B; y += NT / 32) {
            const int py = py0 + y;
            const bool rin = py >= oy && py < oy + Hh;
            float* accrow = job.acc + (long long)(py - oy) * W - ox;
            for (int c = tid & 31; c < PWID; c += 32) {
                const int px = px0 + c;
                const float v = s_ola[y * PWID + c];
                s_ola[y * PWID + c] = 0.0f;
                if (rin && c < (nb - 1) * S + B && px >= ox && px < ox + W) atomicAdd(accrow + px, v);
            }
        }
        // the next tile's first barrier orders these reads before the patch and tile reuse
    }
    // After a wait that ran out, the products of that commit may still be in
    // flight: wait (with the full limit) for the phase that was being waited
    // on before freeing the tensor memory they write.  `phase` was already
    // flipped past it, so that phase's parity is phase ^ 1.
    if (s_fail_any) mbar_wait(&s_bar, phase ^ 1u);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(256) : "memory");
}

}  // namespace dft2
