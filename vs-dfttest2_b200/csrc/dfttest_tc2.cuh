// Tensor-core form of the 16x16 block pipeline, organised around the tensor
// cores rather than around one block at a time ("strip" form).  Same
// semantics as dfttest_unit_kernel (cpu_source/kernel.hpp:1899-1983 fused,
// cpu_source/getframe_impl.cpp:105-221 gather / overlap-add / store) for
// 16x16 blocks, 1 or 3 frames, block steps dividing 16, a separable window
// and a gain table symmetric under k -> -k on the x-bins 0 and B/2 (the
// plugin front end always produces both).
//
// The 3D DFT is separable and linear, so it is reordered to make every
// product a dense tensor-core GEMM whose operands are written in their
// natural order:
//   temporal  : the T frames of each input pixel are combined into T real
//               "P planes" once per pixel (P0 = sum c_t x_t, and for T = 3
//               the cosine and sine parts of temporal bin 1; bin 2 is the
//               conjugate combination), with the temporal window, the
//               sample scale and the centre-first time origin folded in;
//   y (rows)  : MMA_Y   D[x][(p, j)] = P_p[x][y] * Wy[y][j]   (j = packed
//               real-DFT bins of y, y-window folded in).  The P planes sit in
//               a 16-row ring indexed by y mod 16; instead of sliding the
//               operand, the constant is rotated (16/S copies of Wy);
//   x (cols)  : MMA_X   D_c[(blk, kx)][(p, j)] = Wx_c[(blk, kx)][x] * Y[x][(p, j)]
//               for c = cos, sin: a Toeplitz product over a strip of 8
//               blocks at once (the x-window folded in).  One "tall"
//               constant serves every K step: K step s is the same matrix
//               moved up by 16/S blocks;
//   gain      : per (blk, kx) lane, all (kt, ky) bins of the block in one
//               thread: complex bins from the cos/sin products, temporal
//               bins from the P planes, zero-mean, gain, and the inverse
//               over t of the centre frame (a sum, centre-first order);
//   inverse x : 16-point complex IDFT per (blk, ky) on the CUDA cores
//               (register codelet); the x synthesis window scales the output rows;
//   inverse y : MMA_IY  D[(blk, x)][row mod 16] += Y'[(blk, x)][j] * Wiy_rot[j][row mod 16]
//               (c2r over y, y synthesis window folded in): the overlap-add
//               in y happens in the tensor-memory accumulator, whose column
//               of an output row is the row's index mod 16 (the constant's
//               columns are rotated instead of moving the accumulator);
//   overlap-add in x of the rows no later block row reaches (S rows a
//   step): the columns are read, restarted from zero, and the blocks
//   covering each 4-pixel segment summed; final pixels go to the output
//   (or the unit's band record) as in the unit kernel.
// Our bins are (ky 0..8, kx 0..15), the reference's (ky 0..15, kx 0..8):
// a bin with kx > 8 is the conjugate of the reference bin (-kt, -ky, 16-kx),
// whose sigma and window spectrum the gain table holds.
//
// Every operand is split into 16-bit hi + lo parts (fp16: about 22
// significant bits; bf16: about 16) and each product is hi*hi + hi*lo +
// lo*hi, accumulated in FP32 in tensor memory (tcgen05.mma kind::f16,
// cta_group::1, M = 128, operands in shared memory, no swizzle).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "dfttest_kernel.cuh"
#include "dfttest_tc.cuh"

namespace dft2 {

constexpr int kTc2Fp16 = 0, kTc2Bf16 = 1;

// Host-built constants of a filter in the strip form (one image in device
// memory: this header, then the sections, each 128-byte aligned).
struct Tc2Head {
    int S;          // block step (divides 16)
    int nrot;       // rotations of Wy: 16 / S
    int nks;        // K steps (16 columns each) of an 8-block x product
    int nvb;        // virtual blocks of the tall x constants
    int voff;       // virtual block of strip block 0 in K step 0
    int nbx;        // blocks per strip (at most 16: two 8-block tiles)
    int xg;         // 8-column groups of a strip footprint held in the rings
    int np;         // P planes (= T)
    int wmask;      // bit kt: temporal bin kt of the window spectrum is not identically zero
    float q[3][3];  // P-plane coefficients [plane][frame]
    float sx[16];   // synthesis window, x factor
    int off_wy, off_wx, off_wi, off_tab, total;  // byte offsets in the image; total bytes
};
constexpr int kTc2HeadBytes = 256;
constexpr int kTc2ZPitch = 18;       // float2 per (block, y-bin) row of the gain output (bank spread)
static_assert(sizeof(Tc2Head) <= kTc2HeadBytes, "Tc2Head");

// shared-memory plan (bytes from the 128-aligned dynamic base)
struct Tc2Smem {
    int consts;  // image bytes from off_wy (sections in image order)
    int ring, ring_hl;  // P ring: [hl][p][xg][16 rows x 16 B], + slack for the M rows past xg
    int yb, yb_hl;      // Y operand [hl][n-group][xg][8 rows x 16 B]; the gain output aliases it
    int ai, ai_tile;    // inverse-y operand [tile][hl][16 m-groups][2 x 128 B]
    int total;
    __host__ __device__ static Tc2Smem make(int consts_bytes, int np, int xg) {
        Tc2Smem s;
        s.consts = consts_bytes;
        s.ring = (consts_bytes + 127) & ~127;
        s.ring_hl = np * xg * 256;
        const int ring_bytes = 2 * s.ring_hl + (16 - xg) * 256;
        s.yb = s.ring + ((ring_bytes + 127) & ~127);
        s.yb_hl = 2 * np * xg * 128;
        const int zbytes = 16 * 9 * kTc2ZPitch * 8;
        const int yb_bytes = 2 * s.yb_hl > zbytes ? 2 * s.yb_hl : zbytes;
        s.ai = s.yb + ((yb_bytes + 127) & ~127);
        s.ai_tile = 2 * 16 * 256;
        s.total = s.ai + 2 * s.ai_tile;  // the final-row buffer (16 x 16 x 16 floats) aliases it
        return s;
    }
};

// instruction descriptor of kind::f16: D f32, A/B fp16 (fmt 0) or bf16 (1), K- or MN-major
__host__ __device__ constexpr uint32_t idesc2(int fmt, int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((a_mn ? 1u : 0u) << 15) |
           ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// hi + lo 16-bit parts of two values, packed in two 32-bit words
template <int FMT>
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    if constexpr (FMT == kTc2Fp16) {
        const __half2 h = __floats2half2_rn(a, b);
        const float2 hf = __half22float2(h);
        const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
        hi = *reinterpret_cast<const uint32_t*>(&h);
        lo = *reinterpret_cast<const uint32_t*>(&l);
    } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        const float2 hf = __bfloat1622float2(h);
        const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
        hi = *reinterpret_cast<const uint32_t*>(&h);
        lo = *reinterpret_cast<const uint32_t*>(&l);
    }
}

// 8 values -> one 16-byte hi row and one 16-byte lo row
template <int FMT>
__device__ __forceinline__ void put_row8(char* hi_dst, char* lo_dst, const float (&v)[8]) {
    uint4 h, l;
    split2<FMT>(v[0], v[1], h.x, l.x);
    split2<FMT>(v[2], v[3], h.y, l.y);
    split2<FMT>(v[4], v[5], h.z, l.z);
    split2<FMT>(v[6], v[7], h.w, l.w);
    *reinterpret_cast<uint4*>(hi_dst) = h;
    *reinterpret_cast<uint4*>(lo_dst) = l;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// N (1, 2 or 4) consecutive 32-bit columns of this thread's lane: load, store
template <int N> __device__ __forceinline__ void tmem_ld_n(uint32_t taddr, float (&v)[N]) {
    uint32_t r[4];
    if constexpr (N == 1) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r[0]) : "r"(taddr));
    } else if constexpr (N == 2) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(taddr));
    } else {
        static_assert(N == 4, "1, 2 or 4 columns");
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                     : "r"(taddr));
    }
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __uint_as_float(r[i]);
}
template <int N> __device__ __forceinline__ void tmem_st_n(uint32_t taddr, const uint32_t (&v)[N]) {
    if constexpr (N == 1) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(v[0]) : "memory");
    } else if constexpr (N == 2) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(v[0]), "r"(v[1])
                     : "memory");
    } else {
        static_assert(N == 4, "1, 2 or 4 columns");
        asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(v[0]),
                     "r"(v[1]), "r"(v[2]), "r"(v[3])
                     : "memory");
    }
}

// packed real-DFT bin index of y-bin ky: j 0 = Re 0, (1, 2) = (Re, Im) 1, (3, 4) = 2, (5, 6) = 3,
// 7 = Re 8, (8, 9) = (Re, Im) 4, ..., (14, 15) = 7: y-bins 0, 1, 2, 3, 8 in j 0..7, 4..7 in j 8..15
__host__ __device__ constexpr int tc2_jre(int ky) { return ky == 0 ? 0 : (ky == 8 ? 7 : (ky <= 3 ? 2 * ky - 1 : 2 * ky)); }
__host__ __device__ constexpr int tc2_jim(int ky) { return ky <= 3 ? 2 * ky : 2 * ky + 1; }

template <int T, int FC, int FMT, int SS>
__global__ void __launch_bounds__(256, 2) dfttest_tc2_kernel(const __grid_constant__ KernelArgs a) {
    constexpr int NT = 256;
    constexpr int NP = T;          // P planes
    constexpr int NJ = 16 * NP;    // columns of the y products
    extern __shared__ __align__(128) char tc2_smem[];
    __shared__ uint64_t s_bars[3];  // product batches: y, x, inverse y
    __shared__ uint32_t s_tmem;
    __shared__ PlaneJob s_job;
    __shared__ FilterParams s_par;
    __shared__ Tc2Head s_head;
    __shared__ int s_next;
    __shared__ uint64_t s_sbar[2];  // TMA staging slots

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quarter = warp & 3, hf = warp >> 2;

    // ---- once per CTA: header, constants, barrier, tensor memory
    const Tc2Head* gh = reinterpret_cast<const Tc2Head*>(a.tc_consts);
    if (tid < (int)(sizeof(Tc2Head) / 4))
        reinterpret_cast<int*>(&s_head)[tid] = reinterpret_cast<const int*>(gh)[tid];
    __syncthreads();
    const Tc2Head& hd = s_head;
    constexpr int S = SS, O = 16 - S;  // block step (the host built the constants for it)
    const int XG = hd.xg;
    const Tc2Smem L = Tc2Smem::make(hd.total - hd.off_wy, NP, XG);
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.tc_consts + hd.off_wy);
        uint4* dst = reinterpret_cast<uint4*>(tc2_smem);
        for (int i = tid; i < L.consts / 16; i += NT) dst[i] = __ldg(src + i);
    }
    char* c_wy = tc2_smem;
    char* c_wx = tc2_smem + (hd.off_wx - hd.off_wy);
    char* c_wi = tc2_smem + (hd.off_wi - hd.off_wy);
    const float4* __restrict__ c_tab = reinterpret_cast<const float4*>(tc2_smem + (hd.off_tab - hd.off_wy));
    char* s_ring = tc2_smem + L.ring;
    char* s_yb = tc2_smem + L.yb;
    float2* s_z = reinterpret_cast<float2*>(tc2_smem + L.yb);  // gain output, aliases the Y operand
    char* s_ai = tc2_smem + L.ai;
    // final output rows [row][block][x] (16 x 16 x 16 floats), after the inverse-y products
    float* s_fin = reinterpret_cast<float*>(tc2_smem + L.ai);
    // the ring's slack rows are read (as M rows past the footprint) before any write: keep them finite
    for (int i = tid; i < (L.yb - L.ring) / 16; i += NT) reinterpret_cast<uint4*>(s_ring)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        // arrivals per batch: one commit per issuing thread (planes, x-product regions, tiles)
        mbar_init(&s_bars[0], NP);
        mbar_init(&s_bars[1], 4);
        mbar_init(&s_bars[2], 2);
        mbar_init(&s_sbar[0], 1);
        mbar_init(&s_sbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // staging slots: the first 128-byte boundary at or after stage_off (the host adds 128 bytes)
    unsigned char* s_stg = reinterpret_cast<unsigned char*>(tc2_smem) + a.stage_off;
    s_stg += (128u - (smem_addr(s_stg) & 127u)) & 127u;
    // TMA batches this CTA has issued and waited for: batch n uses slot n & 1 and is that slot's
    // (n >> 1)-th phase; every batch is waited for in the unit that issued it
    uint32_t tma_issued = 0, tma_waited = 0;
    constexpr uint32_t kCols = T == 1 ? 128 : 256;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
    // tensor-memory columns: D_X tile h, part c at (2h + c) NJ; D_Y in the columns of tile 1 part sin
    // (written after the gain has read them); D_out, the overlap-add accumulator of the inverse-y
    // products (16 output rows, indexed by padded row mod 16, per tile), after D_X
    constexpr uint32_t C_X = 0, C_Y = 3 * NJ, C_OUT = 4 * NJ;
    // one barrier per product batch; bit k of `ph` is the phase batch k waits for next
    constexpr int BY = 0, BX = 1, BIY = 2;
    uint32_t ph = 0;
    // thread 0: barriers with a committed batch not yet waited for, and that batch's phase parity
    uint32_t pend = 0, ppar = 0;
    auto commit = [&](int k) {
        mma_commit(&s_bars[k]);
        pend |= 1u << k;
        ppar = (ppar & ~(1u << k)) | (((ph >> k) & 1u) << k);
    };
    bool failed = false;

    // the three products hi*hi + hi*lo + lo*hi of one K step
    // part 0: the two correction products hi*lo + lo*hi of one K step; part 1: hi*hi.  Callers
    // issue the correction products of every K step first and the hi*hi products last: the
    // accumulation in tensor memory loses low bits relative to the running sum, so the small terms
    // are summed while the sum is still small.
    // (a_desc / b_desc: descriptor bits other than the start address, sdesc(0, lbo, sbo))
    auto mma3 = [&](int part, uint32_t d, uint32_t a_hi, uint32_t a_lo, uint64_t a_desc, uint32_t b_hi,
                    uint32_t b_lo, uint64_t b_desc, uint32_t id, bool accumulate) {
        const uint64_t ah = a_desc | (a_hi >> 4), bh = b_desc | (b_hi >> 4);
        if (part == 0) {
            mma<false>(d, ah, b_desc | (b_lo >> 4), id, accumulate ? 1u : 0u);
            mma<false>(d, a_desc | (a_lo >> 4), bh, id, 1u);
        } else {
            mma<false>(d, ah, bh, id, 1u);
        }
    };
    // the issuing threads: lane 0 of warps 0..3
    const bool issuer = lane == 0 && warp < 4;
    // wait (thread 0, bounded) for the batch committed to barrier k; every thread learns the outcome
    auto wait_batch = [&](int k) -> bool {
        bool ok = true;
        if (tid == 0) {
            ok = mbar_wait(&s_bars[k], (ph >> k) & 1u, a.wait_limit);
            if (ok) pend &= ~(1u << k);
            else atomicExch(a.error_flag, 2);
        }
        ph ^= 1u << k;
        const bool fail = __syncthreads_or(!ok);
        tc_fence_after();
        return !fail;
    };
    // operand writes of every thread visible to the tensor cores before thread 0 issues products
    auto to_tensor_cores = [&]() {
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    };
    const uint32_t a_ring = smem_addr(s_ring), a_yb = smem_addr(s_yb), a_ai = smem_addr(s_ai);
    const uint32_t a_wy = smem_addr(c_wy), a_wx = smem_addr(c_wx), a_wi = smem_addr(c_wi);
    constexpr int WY_BYTES = 512;                    // one 16 x 16 16-bit matrix
    const int WX_PART = hd.nvb * 16 * 16 * 2;        // one tall matrix (cos or sin, hi or lo)

    for (int uid = blockIdx.x; uid < a.nunits;) {
        int lo = 0, hi = a.njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.jobs[mid].unit_base <= uid) lo = mid; else hi = mid - 1;
        }
        constexpr int NJI = sizeof(PlaneJob) / sizeof(int), NPI = sizeof(FilterParams) / sizeof(int);
        if (tid < NJI) reinterpret_cast<int*>(&s_job)[tid] = reinterpret_cast<const int*>(&a.jobs[lo])[tid];
        if (tid >= 64 && tid < 64 + NPI) {
            const FilterParams* src = a.params ? a.params + a.jobs[lo].param : &a.p;
            reinterpret_cast<int*>(&s_par)[tid - 64] = reinterpret_cast<const int*>(src)[tid - 64];
        }
        __syncthreads();
        const PlaneJob& job = s_job;
        const FilterParams& P = s_par;
        const int W = job.width, Hh = job.height;
        const int pw = pad_size(W, 16, S), ph_ = pad_size(Hh, 16, S);
        const int pnx = (pw - 16) / S + 1, pny = (ph_ - 16) / S + 1;
        const int ox = (pw - W) / 2, oy = (ph_ - Hh) / 2;
        const int lid = uid - job.unit_base;
        const int sx = lid % job.nsx, sy = lid / job.nsx;
        const UnitGeom u = unit_geom(sx, sy, job.nsx, job.nsy, pnx, pny, 16, S);
        const int nbx = u.bx1 - u.bx0;
        if (nbx > hd.nbx || u.fw > XG * 8) {  // uniform: the planner's strips must fit the rings
            if (tid == 0) atomicExch(a.error_flag, 1);
            break;
        }
        const int ntile = nbx > 8 ? 2 : 1;
        float* rec = a.scratch + (size_t)uid * a.rec_stride;
        const bool is_float = (P.kind == kF32);
        const float inv_scale = 1.0f / P.scale;
        const int x0 = u.bx0 * S;
        const int excl_y0 = u.by0 * S + O, excl_y1 = u.by1 * S;
        const int excl_x0 = x0 + O, excl_x1 = u.bx1 * S;
        // P-plane coefficients with the sample scale (scale * window, cpu_source/getframe_impl.cpp:137)
        float qs[NP][T];
#pragma unroll
        for (int p = 0; p < NP; ++p)
#pragma unroll
            for (int t = 0; t < T; ++t) qs[p][t] = hd.q[p][t] * P.scale;
        // TMA staging of the input rows (as the unit kernel): box of stage_bw samples from xa, the
        // footprint's first source column rounded down to 16 bytes; every source column the
        // footprint reads, mirrored ones included, must lie in the box
        const int esz = P.kind == kF32 ? 4 : (P.kind == kU16 ? 2 : 1);
        const int xa = (x0 - ox) >= 0 ? ((x0 - ox) / (16 / esz)) * (16 / esz)
                                      : -(((ox - x0) + (16 / esz) - 1) / (16 / esz)) * (16 / esz);
        bool use_tma = a.tmaps != nullptr && job.tmap[0] >= 0;
        {
            const int c_lo = x0 - ox, c_hi = x0 - ox + 8 * XG - 1;
            int need_lo = max(c_lo, 0), need_hi = min(c_hi, W - 1);
            if (c_lo < 0) need_hi = max(need_hi, -c_lo);
            if (c_hi >= W) need_lo = min(need_lo, 2 * (W - 1) - c_hi);
            use_tma = use_tma && need_lo >= xa && need_hi < xa + a.stage_bw && need_lo >= 0 && need_hi < W;
        }
        const int srb = stage_row_bytes(a.stage_bw, esz);
        const FinishGeom fg{job.dst, job.dst_stride, P.kind, P.scale, P.peak, is_float ? 0.0f : inv_scale,
                            x0, ox, oy, W, Hh, excl_x0, excl_x1, excl_y0, excl_y1, rec, u.fw, u.fh, u.by0 * S, O,
                            a.rec_stride, a.error_flag};
        const int nseg = (u.fw + 3) >> 2;
        const float inv_nseg = 1.0f / (float)nseg;
        // one P-plane item: 4 pixels of padded row r_lo + r (item = r * 2 XG + 4-pixel group), the
        // T frames combined into the NP planes, hi and lo parts into the ring (staged rows from TMA
        // slot `slot`, or plain loads)
        const int ng4 = 2 * XG;
        const float inv_S = 1.0f / (float)S;
        auto pconv_item = [&](int item, int r_lo, int nr, float inv_nr, bool staged, int slot) {
            const int g4 = div_small(item, inv_nr), r = item - g4 * nr;  // rows fastest (spreads the stores)
            const int py = r_lo + r;
            int sc[4];  // source columns (mirror padding)
#pragma unroll
            for (int i = 0; i < 4; ++i) sc[i] = mirror(min(x0 + g4 * 4 + i, pw - 1) - ox, W);
            const bool fast4 = sc[3] == sc[0] + 3 && ((sc[0] - xa) & 3) == 0;
            float pv[NP][4];
#pragma unroll
            for (int p = 0; p < NP; ++p)
#pragma unroll
                for (int i = 0; i < 4; ++i) pv[p][i] = 0.0f;
            const long long rowoff = (long long)mirror(py - oy, Hh) * job.src_stride;
#pragma unroll
            for (int t = 0; t < T; ++t) {
                float xv[4];
                if (staged) {
                    const unsigned char* srow = s_stg + ((slot * T + t) * S + r) * srb;
                    if (fast4) {  // four in-plane samples, aligned in the staged row: one vector load
                        const float4 q4 = stage_load4(srow, sc[0] - xa, P.kind);
                        xv[0] = q4.x;
                        xv[1] = q4.y;
                        xv[2] = q4.z;
                        xv[3] = q4.w;
                    } else {
#pragma unroll
                        for (int i = 0; i < 4; ++i) xv[i] = stage_load1(srow, sc[i] - xa, P.kind);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 4; ++i) xv[i] = load_sample(job.src[t], rowoff + sc[i], P.kind);
                }
#pragma unroll
                for (int p = 0; p < NP; ++p)
#pragma unroll
                    for (int i = 0; i < 4; ++i) pv[p][i] = fmaf(qs[p][t], xv[i], pv[p][i]);
            }
            const int ro = (py & 15) * 16 + (g4 & 1) * 8;
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                char* base = s_ring + (p * XG + (g4 >> 1)) * 256 + ro;
                uint2 h, l;
                split2<FMT>(pv[p][0], pv[p][1], h.x, l.x);
                split2<FMT>(pv[p][2], pv[p][3], h.y, l.y);
                *reinterpret_cast<uint2*>(base) = h;
                *reinterpret_cast<uint2*>(base + L.ring_hl) = l;
            }
        };

        // Software pipeline over the unit's block rows: iteration it runs the front of block row it
        // (P planes, y products, Y operand, x products) and the back of block row it - 1 (gain,
        // inverse x, inverse-y products, overlap-add), so that each batch of products overlaps
        // CUDA-core work of the other block row.
        for (int it = u.by0; it <= u.by1 && !failed; ++it) {
            const bool front = it < u.by1, back = it > u.by0;
            const int bb = it - 1;  // block row of the back half
            if (front) {
                // ---- 0. the next block row's S new input rows of every frame: TMA copies (one box per
                //      row, the row index through the mirror map) into the free staging slot
                if (use_tma && it + 1 < u.by1) {
                    const int slot = tma_issued & 1;
                    ++tma_issued;
                    const int n_lo = (it + 1) * S + O;
                    if (warp == 7) {
                        if (lane == 0) {
                            fence_proxy_async_smem();
                            mbar_arrive_expect_tx(&s_sbar[slot], (uint32_t)(T * S * a.stage_bw * esz));
                        }
                        __syncwarp();
                        for (int k = lane; k < T * S; k += 32) {
                            const int t = k / S, rr = k - t * S;
                            const unsigned char* map =
                                reinterpret_cast<const unsigned char*>(a.tmaps) + (size_t)job.tmap[t] * kTmapBytes;
                            tma_load_2d(s_stg + ((slot * T + t) * S + rr) * srb, map, xa, mirror(n_lo + rr - oy, Hh),
                                        &s_sbar[slot]);
                        }
                    }
                }
                // ---- 1. P planes of the unit's first block row (all 16 rows, plain loads); later block
                //      rows get theirs at the end of the previous iteration, with its overlap-add
                if (it == u.by0)
                    for (int item = tid; item < 16 * ng4; item += NT) pconv_item(item, it * S, 16, 1.0f / 16.0f, false, 0);
            }
            if (back) {
                // ---- 5. gain of block row bb: lane (blk, kx) of tile hf, every (kt, ky) bin of its block
                if (!wait_batch(BX)) {
                    failed = true;
                    break;
                }
                {
                    const int l = quarter * 32 + lane;
                    const int blk = l >> 4, kx = l & 15;
                    const int b = hf * 8 + blk;
                    const bool active = hf < ntile && b < nbx;
                    const uint32_t dc = tmem + lane_base + C_X + (2 * hf) * NJ;
                    const uint32_t ds = dc + NJ;
                    float g = 0.0f;
                    const int zm_mask = P.g_div != 0.0f ? hd.wmask : 0;  // temporal bins with zero-mean terms
#pragma unroll
                    for (int pass = 0; pass < 2; ++pass) {
                        float vc[NP][8], vs[NP][8];
#pragma unroll
                        for (int p = 0; p < NP; ++p) {  // warp-wide loads, inactive lanes included
                            tmem_ld8(dc + 16 * p + 8 * pass, vc[p]);
                            tmem_ld8(ds + 16 * p + 8 * pass, vs[p]);
                        }
                        tmem_wait_ld();
                        if (pass == 0) {
                            // zero-mean: g = Re Z(0,0,0) / Re W(0,0,0), Z(0,0,0) held by lane kx = 0 of the block
                            const float dc0 = __shfl_sync(0xffffffffu, vc[0][0], lane & 16);
                            g = P.g_div != 0.0f ? __fdiv_rn(dc0, P.g_div) : 0.0f;
                        }
                        // y-bins of this pass (their packed bins j lie in its 8 columns): pass 0 -> 0, 1, 2, 3, 8;
                        // pass 1 -> 4, 5, 6, 7; outputs are stored after the pass, so that no store sits
                        // between the table loads of the bins
                        float2 outv[5];
#pragma unroll
                        for (int kk = 0; kk < 5; ++kk) {
                            if (pass == 1 && kk == 4) continue;
                            const int ky = pass == 0 ? (kk == 4 ? 8 : kk) : 4 + kk;
                            float zr[NP], zi[NP];
#pragma unroll
                            for (int p = 0; p < NP; ++p) {
                                if (ky == 0 || ky == 8) {  // real in y: no imaginary column
                                    const int jr = tc2_jre(ky) - 8 * pass;
                                    zr[p] = vc[p][jr];
                                    zi[p] = -vs[p][jr];
                                } else {
                                    const int jr = tc2_jre(ky) - 8 * pass, ji = tc2_jim(ky) - 8 * pass;
                                    zr[p] = vc[p][jr] + vs[p][ji];
                                    zi[p] = vc[p][ji] - vs[p][jr];
                                }
                            }
                            float kr[T], ki[T];
                            kr[0] = zr[0];
                            ki[0] = zi[0];
                            if constexpr (T == 3) {
                                kr[1] = zr[1] - zi[2];
                                ki[1] = zi[1] + zr[2];
                                kr[2] = zr[1] + zi[2];
                                ki[2] = zi[1] - zr[2];
                            }
                            // per temporal bin: U = Z - g W, m = gain(|U|^2, sigma), sum of m U over the bins,
                            // plus g times the sum of W (the add-back of the zero-mean terms, summed once);
                            // bins whose window spectrum is zero skip the subtraction
                            float sr = 0.0f, si = 0.0f;
                            float4 tb0;
#pragma unroll
                            for (int kt = 0; kt < T; ++kt) {
                                const float4 tb = c_tab[(kt * 9 + ky) * 16 + kx];
                                if (kt == 0) tb0 = tb;
                                float dre = kr[kt], dim = ki[kt];
                                if (zm_mask & (1 << kt)) {
                                    dre = fmaf(-g, tb.y, dre);
                                    dim = fmaf(-g, tb.z, dim);
                                }
                                const float psd = fmaf(dim, dim, dre * dre);
                                const float m =
                                    FC == kFilterWiener ? gain<0>(psd, tb.x, P) : gain_rt(P.filter_type, psd, tb.x, P);
                                sr = fmaf(m, dre, sr);
                                si = fmaf(m, dim, si);
                            }
                            if (zm_mask) {
                                // sum over the bins of W: in the w slots of bins 0 and 1 (T = 3), W itself (T = 1)
                                const float swr = T == 1 ? tb0.y : tb0.w;
                                const float swi = T == 1 ? tb0.z : c_tab[(9 + ky) * 16 + kx].w;
                                sr = fmaf(g, swr, sr);
                                si = fmaf(g, swi, si);
                            }
                            outv[kk] = make_float2(sr, si);
                        }
                        if (active) {
#pragma unroll
                            for (int kk = 0; kk < 5; ++kk) {
                                if (pass == 1 && kk == 4) continue;
                                s_z[(b * 9 + (pass == 0 ? (kk == 4 ? 8 : kk) : 4 + kk)) * kTc2ZPitch + kx] = outv[kk];
                            }
                        }
                    }
                }
            }
            // ---- 2. MMA_Y of block row it: D_Y[x][(p, j)] = ring_p[x][ring row] * Wy_rot[ring row][j], into the
            //      columns of D_X tile 1 part sin, which the gain above has read (the barrier orders it)
            to_tensor_cores();
            if (front && issuer && warp < NP) {  // plane p = warp
                const int rot = ((it * S) & 15) / S;
                const uint32_t id = idesc2(FMT, 128, 16, true, false);
                const uint32_t wy = a_wy + rot * 2 * WY_BYTES;
                const uint32_t ap = a_ring + warp * XG * 256;
                const uint64_t da = sdesc(0, 128, 256);
#pragma unroll
                for (int part = 0; part < 2; ++part)
                    mma3(part, tmem + C_Y + 16 * warp, ap, ap + L.ring_hl, da, wy, wy + WY_BYTES, da, id, false);
                commit(BY);
            }
            if (back) {
                // ---- 6. inverse x per (block, y-bin): 16-point complex IDFT, x synthesis window -> inverse-y operand
                if (tid < 16 * 9) {
                    const int b = tid / 9, ky = tid - b * 9;
                    if (b < nbx) {
                        float re[16], im[16];
                        const float4* zp = reinterpret_cast<const float4*>(s_z + (b * 9 + ky) * kTc2ZPitch);
#pragma unroll
                        for (int k2 = 0; k2 < 8; ++k2) {
                            const float4 v = zp[k2];
                            re[2 * k2] = v.x;
                            im[2 * k2] = v.y;
                            re[2 * k2 + 1] = v.z;
                            im[2 * k2 + 1] = v.w;
                        }
                        cdft_16_inv(re, im);
                        const int h = b >> 3, blk = b & 7;
                        char* tb = s_ai + h * L.ai_tile;
                        // element (m = blk*16 + x, j): m-group (blk*2 + x/8) at 256 B, j-group at 128 B, row (j % 8)
                        auto put_j = [&](int j, const float (&v)[16]) {
#pragma unroll
                            for (int xh = 0; xh < 2; ++xh) {
                                float w8[8];
#pragma unroll
                                for (int i = 0; i < 8; ++i) w8[i] = v[8 * xh + i];
                                char* dst = tb + (blk * 2 + xh) * 256 + (j >> 3) * 128 + (j & 7) * 16;
                                put_row8<FMT>(dst, dst + 16 * 256, w8);
                            }
                        };
                        put_j(tc2_jre(ky), re);
                        if (ky >= 1 && ky <= 7) put_j(tc2_jim(ky), im);
                    }
                }
            }
            // ---- 4. inverse-y products of block row bb (accumulated into D_out), issued as soon as the
            //      inverse x of every thread is in shared memory: the barrier of the y-product wait (an
            //      explicit hand-off when no front half runs) orders them, and they run while the Y
            //      operand below is written (the tensor cores then run them before the x products)
            if (back) async_proxy_fence();
            if (front) {
                if (!wait_batch(BY)) {
                    failed = true;
                    break;
                }
            } else {
                to_tensor_cores();
            }
            if (back && issuer && warp < 2) {  // tile h = warp (an empty commit when the strip has one tile)
                const int h = warp;
                if (h < ntile) {
                    // output row (bb S + y) of the block lands in accumulator column (bb S + y) mod 16:
                    // the constant's columns are rotated; the unit's first block row starts the sums
                    const uint32_t id = idesc2(FMT, 128, 16, true, false);
                    const uint32_t ah = a_ai + h * L.ai_tile;
                    const uint32_t wi = a_wi + (((bb * S) & 15) / S) * 2 * WY_BYTES;
                    const uint64_t da = sdesc(0, 128, 256);
#pragma unroll
                    for (int part = 0; part < 2; ++part)
                        mma3(part, tmem + C_OUT + 16 * h, ah, ah + 16 * 256, da, wi, wi + WY_BYTES, da, id,
                             bb > u.by0);
                }
                commit(BIY);
            }
            if (front) {
                // ---- 3. Y operand: lane x writes its (p, j) columns as 16-byte rows (the Y operand
                //      aliases the gain output, which the inverse x above has consumed)
                const int x = quarter * 32 + lane;
                constexpr int CPH = NJ / 2;  // columns per half
                float v[CPH / 8][8];  // every load issued before one wait
#pragma unroll
                for (int c8 = 0; c8 < CPH / 8; ++c8) tmem_ld8(tmem + lane_base + C_Y + hf * CPH + c8 * 8, v[c8]);
                tmem_wait_ld();
                if (x < XG * 8) {
#pragma unroll
                    for (int c8 = 0; c8 < CPH / 8; ++c8) {
                        const int n0 = hf * CPH + c8 * 8;
                        char* dst = s_yb + (n0 / 8) * (XG * 128) + (x >> 3) * 128 + (x & 7) * 16;
                        put_row8<FMT>(dst, dst + L.yb_hl, v[c8]);
                    }
                }
                // ---- 7. x products of block row it (D_X, the Y products read above included)
                to_tensor_cores();
                if (issuer) {  // region (tile h, part c) = (warp / 2, warp % 2)
                    const int h = warp >> 1, c = warp & 1;
                    if (h < ntile) {
                        const uint32_t id = idesc2(FMT, 128, NJ, false, true);
                        const uint32_t d = tmem + C_X + (2 * h + c) * NJ;
                        const uint64_t da = sdesc(0, 128, 256), db = sdesc(0, 128, XG * 128);
                        for (int part = 0; part < 2; ++part)
                            for (int s = 0; s < hd.nks; ++s) {
                                const int vb0 = hd.voff - s * (16 / S);
                                const uint32_t ah = a_wx + (2 * c) * WX_PART + vb0 * 512;
                                const uint32_t bh = a_yb + ((8 * h * S + 16 * s) >> 3) * 128;
                                mma3(part, d, ah, ah + WX_PART, da, bh, bh + L.yb_hl, db, id, s > 0);
                            }
                    }
                    commit(BX);
                }
            }
            if (back) {
                // ---- 8. final rows of block row bb: the accumulator columns of the output rows that no
                //      later block row reaches (S rows; all 16 at the unit's last block row), x synthesis
                //      window, per block into the row buffer (aliases the inverse-y operand, which the
                //      products have read); those columns restart from zero for the next block row
                if (!wait_batch(BIY)) {
                    failed = true;
                    break;
                }
                {
                    const bool last = (bb + 1 == u.by1);
                    const int c0 = (bb * S) & 15;  // accumulator column of output row bb * S
                    const int l = quarter * 32 + lane;
                    const int blk = l >> 4, x = l & 15;
                    const int b = hf * 8 + blk;
                    const uint32_t col = tmem + lane_base + C_OUT + 16 * hf;
                    const bool mine = hf < ntile && b < nbx;
                    const float w = hd.sx[x];
                    if (last) {
                        float v[16];
                        tmem_ld16(col, v);
                        tmem_wait_ld();
                        if (mine) {
#pragma unroll
                            for (int y = 0; y < 16; ++y)  // column y holds output row bb S + ((y - c0) mod 16)
                                s_fin[((((y - c0) & 15)) * 16 + b) * 16 + x] = v[y] * w;
                        }
                    } else {
                        // the S columns c0 .. c0 + S - 1 (c0 + S <= 16): read, then restart from zero
                        float v[S];
                        uint32_t z[S];
                        tmem_ld_n<S>(col + c0, v);
                        tmem_wait_ld();
#pragma unroll
                        for (int r = 0; r < S; ++r) z[r] = 0u;
                        tmem_st_n<S>(col + c0, z);
                        if (mine) {
#pragma unroll
                            for (int r = 0; r < S; ++r) s_fin[(r * 16 + b) * 16 + x] = v[r] * w;
                        }
                        tmem_wait_st();
                    }
                }
                tc_fence_before();
                __syncthreads();
            }
            // ---- 9. output of block row bb's final rows (item (row r, 4-pixel segment q): the covering
            //      blocks in ascending order), and the P planes of block row it + 1 (its S new rows,
            //      staged or plain loads), in one loop: the ring rows they overwrite were read by MMA_Y(it)
            {
                const bool last = (bb + 1 == u.by1);
                const int nfin = last ? 16 : S;
                const int n_out = back ? nfin * nseg : 0;
                const bool next = it + 1 < u.by1;
                const int n_pc = next ? S * 2 * XG : 0;
                const bool staged = use_tma && next;
                int slot = 0;
                if (staged) {  // the batch issued at the top of this iteration
                    slot = tma_waited & 1;
                    const uint32_t parity = (tma_waited >> 1) & 1;
                    ++tma_waited;
                    if (!mbar_wait(&s_sbar[slot], parity, a.wait_limit)) {
                        // record it, and let the copies land before this shared memory is reused
                        atomicExch(a.error_flag, 4);
                        mbar_wait(&s_sbar[slot], parity, 16 * kDefaultWaitLimit);
                    }
                }
                for (int item = tid; item < n_out + n_pc; item += NT) {
                    if (item >= n_out) {
                        pconv_item(item - n_out, (it + 1) * S + O, S, inv_S, staged, slot);
                        continue;
                    }
                    const int r = div_small(item, inv_nseg), q = item - r * nseg;
                    const int py = bb * S + r;
                    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
                    float* av = reinterpret_cast<float*>(&acc);
                    const float* row = s_fin + r * 256;
                    if constexpr ((S & 3) == 0) {
                        // the segment lies inside or outside each block
                        const int px = 4 * q;
                        const int b_lo = px + 4 <= 16 ? 0 : (px + 4 - 16 + S - 1) / S;
                        const int b_hi = min(px / S, nbx - 1);
                        constexpr int NK = 16 / S;  // covering blocks at most: loads issued together
                        float4 w4[NK];
#pragma unroll
                        for (int k = 0; k < NK; ++k)
                            w4[k] = b_lo + k <= b_hi
                                        ? *reinterpret_cast<const float4*>(row + (b_lo + k) * 16 + (px - (b_lo + k) * S))
                                        : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                        for (int k = 0; k < NK; ++k) {  // ascending block order
                            acc.x += w4[k].x;
                            acc.y += w4[k].y;
                            acc.z += w4[k].z;
                            acc.w += w4[k].w;
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int px = 4 * q + i;
                            const int b_lo = px <= 15 ? 0 : (px - 15 + S - 1) / S;
                            const int b_hi = min(px / S, nbx - 1);
                            for (int b = b_lo; b <= b_hi; ++b) av[i] += row[b * 16 + (px - b * S)];
                        }
                    }
                    const int gx = x0 + 4 * q;
                    if (4 * q + 4 <= u.fw && gx >= excl_x0 && gx + 4 <= excl_x1 && gx >= ox && gx + 4 <= ox + W &&
                        py >= excl_y0 && py < excl_y1 && py >= oy && py < oy + Hh) {
                        store4(job.dst, (long long)(py - oy) * job.dst_stride + (gx - ox), acc, P.kind, P.peak,
                               inv_scale);
                    } else {
                        // a segment of the unit's band (shared with a neighbour): one vector store into the
                        // band record when its 4 pixels are in the plane and contiguous there, else per pixel
                        bool done = false;
                        if (4 * q + 4 <= u.fw && gx >= ox && gx + 4 <= ox + W && py >= oy && py < oy + Hh &&
                            !(py >= excl_y0 && py < excl_y1 && gx + 3 >= excl_x0 && gx < excl_x1)) {
                            const int ly = py - u.by0 * S;
                            const int i0 = band_index(4 * q, ly, u.fw, u.fh, O);
                            const int i3 = band_index(4 * q + 3, ly, u.fw, u.fh, O);
                            float* dst = rec + i0;
                            if (i3 == i0 + 3 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0 &&
                                DFT_IN_RANGE(i3, a.rec_stride, a.error_flag)) {
                                *reinterpret_cast<float4*>(dst) = acc;
                                done = true;
                            }
                        }
                        if (!done) {
#pragma unroll
                            for (int i = 0; i < 4; ++i)
                                if (4 * q + i < u.fw) finish_px(fg, py, 4 * q + i, av[i]);
                        }
                    }
                }
            }
            // the next iteration's first barrier orders these ring and row-buffer accesses before reuse
        }
        if (failed) break;

        // ---- seams shared with the neighbouring full-height strips
        if (a.seam_count != nullptr)
            sum_seams<16>(a, job, P, sx, pnx, pny, ox, oy, W, Hh, is_float ? 0.0f : inv_scale, tid, NT);

        // ---- the next unit (persistent grid)
        if (a.unit_counter == nullptr) break;
        __syncthreads();
        if (tid == 0) s_next = (int)gridDim.x + atomicAdd(a.unit_counter, 1);
        __syncthreads();
        uid = s_next;
    }
    // After a wait that ran out, products may still be in flight: wait (with the full limit) for
    // every batch committed and not yet waited for before freeing the tensor memory they write,
    // and for row copies issued and not yet waited for before the shared memory is released.
    if (failed && tid == 0) {
        for (int k = 0; k < 3; ++k)
            if ((pend >> k) & 1u) mbar_wait(&s_bars[k], (ppar >> k) & 1u);
        for (; tma_waited < tma_issued; ++tma_waited)
            mbar_wait(&s_sbar[tma_waited & 1], (tma_waited >> 1) & 1, 16 * kDefaultWaitLimit);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

}  // namespace dft2
