// DFTTest per-plane hot path for sm_100a: block gather + analysis window,
// forward 3D real DFT, frequency-domain gain (optionally zero-mean), inverse
// DFT of the centre frame, synthesis window and overlap-add, all on chip.
//
// Reference semantics: cpu_source/getframe_impl.cpp:11-221 (geometry,
// mirror padding, load_block, store_block, store_frame) and
// cpu_source/kernel.hpp:1819-1983 (remove_mean, frequency_filtering,
// add_mean, fused); general block sizes follow cuda_source/kernels.cu:84-246.
//
// Work decomposition
// ------------------
// A plane is padded (mirror, no edge repeat) to pw x ph and covered by
// pnx x pny blocks of B x B at stride S.  The blocks are split into
// rectangular *units* (nsx strips x nsy segments); one CTA owns one unit and
// walks down its block rows.  Per block row ("step"):
//   1. the S new input rows of every temporal frame enter a ring in shared
//      memory (mirror padding done by index math, samples kept unscaled);
//   2. each warp transforms BPW = 64/B blocks entirely in registers and a
//      private shared buffer:
//        row phase    lane = (block, y), 2 tasks: T real rows -> r2c_B,
//                     then the temporal DFT over the T frames per x-bin;
//        column phase lane = (block, c), c < B/2 packs x-bins c (and, for
//                     c = 0, the Nyquist bin B/2): y-DFT per temporal plane,
//                     gain, accumulation of the centre-frame inverse, y-IDFT;
//        inverse rows lane = (block, y), 2 tasks: c2r_B, synthesis window;
//   3. the CTA sums the windowed block outputs into an overlap-add ring;
//   4. the S rows that no later block touches are final: interior pixels
//      are converted and stored, pixels within B-S of the unit edge go to
//      a per-unit scratch record and are summed by the fix-up kernel.
//
// x-bins 0 and B/2 are real in (t, y) and travel as one complex column
// ("packed" lane): the temporal DFT of the two real sequences is split in
// the row phase, the y-DFT of plane 0 is untangled into the two Hermitian
// spectra before the gain and the centre-frame sum is re-packed after it.
// This is exact: the reference's c2r ignores the imaginary parts of those
// bins, i.e. it uses the Hermitian part of each column, which is what the
// re-packing reconstructs.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "codelets.cuh"

namespace dft2 {

enum SampleKind : int { kU8 = 0, kU16 = 1, kF32 = 2 };

// one output plane of one frame
struct PlaneJob {
    const void* src[7];   // 2r+1 source planes on the device (time clamp already applied)
    void* dst;            // output plane on the device
    long long src_stride; // elements
    long long dst_stride; // elements
    int width, height;
    int nsx, nsy;         // unit split of the block grid
    int unit_base;        // first global unit id of this job
    int fix_base;         // first global fix-up pixel id of this job
};

struct KernelArgs {
    const PlaneJob* jobs;
    int njobs;
    int nunits;
    int nfix;
    int kind;          // SampleKind
    float scale;       // 2^-(bits-8) for integers, 255 for float
    float peak;        // 2^bits - 1
    int block_step;    // S
    int filter_type;   // 0..6
    float sigma2, pmin, pmax;
    float g_div;       // Re(window_freq[0,0,0]); 0 disables zero-mean
    const float* win;  // [T][B][B] analysis window * scale
    const float* wsyn; // [B][B] synthesis window
    const float* sig;  // [T][B+2][B/2] sigma per gain slot
    const float* sig2; // [T][B+2][B/2] partner sigma (packed lane, asymmetric sigma), may be null
    const float* wfe;  // [T][B+2][B/2][2] window spectrum per gain slot (zero-mean)
    float* scratch;    // per-unit band records
    int rec_stride;    // floats per unit record
    int ring_pitch;    // floats per ring row
    int* error_flag;   // set to a non-zero code on an internal consistency failure
};

__host__ __device__ inline int pad_size(int n, int B, int S) {
    return n + ((n % B) ? B - n % B : 0) + 2 * (B - S > S ? B - S : S);
}
__host__ __device__ inline int pad_num(int n, int B, int S) { return (pad_size(n, B, S) - B) / S + 1; }

// first block of strip s when n blocks are split into ns near-equal strips
__host__ __device__ inline int split_lo(int s, int n, int ns) { return (int)(((long long)s * n) / ns); }

struct UnitGeom {
    int bx0, bx1, by0, by1; // block range
    int fw, fh;             // footprint size
};

__host__ __device__ inline UnitGeom unit_geom(int sx, int sy, int nsx, int nsy, int pnx, int pny, int B, int S) {
    UnitGeom u;
    u.bx0 = split_lo(sx, pnx, nsx);
    u.bx1 = split_lo(sx + 1, pnx, nsx);
    u.by0 = split_lo(sy, pny, nsy);
    u.by1 = split_lo(sy + 1, pny, nsy);
    u.fw = (u.bx1 - u.bx0) * S + (B - S);
    u.fh = (u.by1 - u.by0) * S + (B - S);
    return u;
}

// offset of footprint pixel (lx, ly) inside the unit's band record; the band
// is every footprint pixel within O = B-S of the footprint edge.
__host__ __device__ inline int band_index(int lx, int ly, int fw, int fh, int O) {
    if (ly < O) return ly * fw + lx;
    if (ly >= fh - O) return (O + ly - (fh - O)) * fw + lx;
    const int r = ly - O;
    const int base = 2 * O * fw;
    if (lx < O) return base + r * O + lx;
    return base + (fh - 2 * O) * O + r * O + (lx - (fw - O));
}

__host__ __device__ inline int band_record_size(int fw, int fh, int O) { return 2 * O * fw + 2 * (fh - 2 * O) * O; }

__device__ __forceinline__ int mirror(int i, int n) {
    // reflection without edge repeat (cpu_source/getframe_impl.cpp:44-62)
    i = i < 0 ? -i : i;
    return i >= n ? 2 * (n - 1) - i : i;
}

__device__ __forceinline__ float load_sample(const void* base, long long idx, int kind) {
    if (kind == kU8) return (float)__ldg(reinterpret_cast<const uint8_t*>(base) + idx);
    if (kind == kU16) return (float)__ldg(reinterpret_cast<const uint16_t*>(base) + idx);
    return __ldg(reinterpret_cast<const float*>(base) + idx);
}

__device__ __forceinline__ void store_sample(void* base, long long idx, float acc, int kind, float scale, float peak,
                                             float inv_scale = 0.0f) {
    // cpu_source/getframe_impl.cpp:177-221: v = acc / scale, integers rounded
    // by truncation of v + 0.5 and clamped to [0, peak]; for the power-of-two
    // integer scales the division is an exact multiplication (inv_scale)
    const float v = inv_scale != 0.0f ? acc * inv_scale : __fdiv_rn(acc, scale);
    if (kind == kF32) {
        reinterpret_cast<float*>(base)[idx] = v;
        return;
    }
    int q = __float2int_rz(__fadd_rn(v, 0.5f));
    q = q < 0 ? 0 : q;
    const int pk = (int)peak;
    q = q > pk ? pk : q;
    if (kind == kU8)
        reinterpret_cast<uint8_t*>(base)[idx] = (uint8_t)q;
    else
        reinterpret_cast<uint16_t*>(base)[idx] = (uint16_t)q;
}

// reciprocal from the MUFU unit (PTX rcp.approx.ftz.f32, < 1 ulp)
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// multiplier of frequency_filtering (cpu_source/kernel.hpp:1826-1890).
// FT 0 is the Wiener gain max((psd - s) / (psd + 1e-15), 0), evaluated as
// max(1 - s * rcp(psd + 1e-15), 0); the other types keep IEEE division.
template <int FT>
__device__ __forceinline__ float gain(float psd, float s, const KernelArgs& a) {
    if constexpr (FT == 0) {
        return fmaxf(fmaf(-s, rcp_approx(psd + 1e-15f), 1.0f), 0.0f);
    } else if constexpr (FT == 1) {
        return psd < s ? 0.0f : 1.0f;
    } else if constexpr (FT == 2) {
        return s;
    } else if constexpr (FT == 3) {
        return (psd >= a.pmin && psd <= a.pmax) ? s : a.sigma2;
    } else if constexpr (FT == 4) {
        return s * sqrtf(psd * __fdiv_rn(a.pmax, (psd + a.pmin) * (psd + a.pmax) + 1e-15f));
    } else if constexpr (FT == 5) {
        return powf(fmaxf(__fdiv_rn(psd - s, psd + 1e-15f), 0.0f), a.pmin);
    } else {
        return sqrtf(fmaxf(__fdiv_rn(psd - s, psd + 1e-15f), 0.0f));
    }
}

__device__ __forceinline__ float gain_rt(int ft, float psd, float s, const KernelArgs& a) {
    switch (ft) {
    case 0: return fmaxf(__fdiv_rn(psd - s, psd + 1e-15f), 0.0f);
    case 1: return gain<1>(psd, s, a);
    case 2: return gain<2>(psd, s, a);
    case 3: return gain<3>(psd, s, a);
    case 4: return gain<4>(psd, s, a);
    case 5: return gain<5>(psd, s, a);
    default: return gain<6>(psd, s, a);
    }
}

// kernel filter classes: the Wiener fast path, or every type with a runtime
// switch (also handles asymmetric sigma on the packed columns)
constexpr int kFilterWiener = 0;
constexpr int kFilterGeneric = 7;

// Y = m(|U - gW|^2) * (U - gW) + gW   (remove_mean / filter / add_mean,
// cpu_source/kernel.hpp:1943-1952)
template <int FC>
__device__ __forceinline__ void apply_bin(float& re, float& im, float s, float s2, bool dual, float2 w, float g,
                                          const KernelArgs& a) {
    const float dre = fmaf(-g, w.x, re);
    const float dim = fmaf(-g, w.y, im);
    const float psd = fmaf(dim, dim, dre * dre);
    float m;
    if constexpr (FC == kFilterWiener) {
        m = gain<0>(psd, s, a);
    } else {
        m = gain_rt(a.filter_type, psd, s, a);
        if (dual) m = 0.5f * (m + gain_rt(a.filter_type, psd, s2, a));
    }
    re = fmaf(m, dre, re - dre);
    im = fmaf(m, dim, im - dim);
}

template <int B> struct Tile {
    static constexpr int H = B / 2;          // packed x-bins per block (lanes per block)
    static constexpr int BPW = 64 / B;       // blocks per warp
    static constexpr int WP = B + 4;         // padded window row pitch (floats)
    static constexpr int RPL = 32 / B;       // rows per 128-byte line in the warp buffer
    static constexpr int NCH = B / 4;        // 16-byte chunks per buffer row
    __device__ static __forceinline__ int swz(int y) { return (y / RPL) & (NCH - 1); }
    // float offset of (y, x) inside one B x B plane of the warp buffer
    __device__ static __forceinline__ int off(int y, int x) { return y * B + ((((x >> 2) ^ swz(y)) << 2) | (x & 3)); }
};

template <int B, int T, int NW>
struct Layout {
    static constexpr int H = B / 2;
    static constexpr int BPW = 64 / B;
    static constexpr int WP = B + 4;
    static constexpr int NSLOT = B + 2;
    static constexpr int BSTR = T * B * B + B;  // warp-buffer floats per block
    // offsets in floats (ring sizes depend on the runtime pitch)
    static constexpr int o_win = 0;
    static constexpr int o_wsyn = o_win + T * B * WP;
    static constexpr int o_sig = o_wsyn + B * WP;
    static constexpr int o_sig2 = o_sig + T * NSLOT * H;
    static constexpr int o_wfe = o_sig2 + T * NSLOT * H;
    static constexpr int o_g = o_wfe + 2 * T * NSLOT * H;
    static constexpr int o_wbuf = o_g + ((NW * BPW + 3) & ~3);
    static constexpr int o_ring = o_wbuf + NW * BPW * BSTR;
    __host__ __device__ static int in_ring_floats(int pitch) { return T * B * pitch; }
    __host__ __device__ static int ola_floats(int pitch) { return B * pitch; }
    __host__ __device__ static size_t smem_bytes(int pitch) {
        return sizeof(float) * (size_t)(o_ring + in_ring_floats(pitch) + ola_floats(pitch));
    }
};

// i / n and i % n for small non-negative i, n through a float reciprocal
// (exact while i * n < 2^22, which the shared-memory extents guarantee)
__device__ __forceinline__ int div_small(int i, float inv_n) { return __float2int_rz(((float)i + 0.5f) * inv_n); }

// ---------------------------------------------------------------------------
// row phase: T rows of one block at one y -> packed spectra per temporal plane;
// returns this row's contribution to the block's 3D DC (zero-mean)
// ---------------------------------------------------------------------------
template <int B, int T>
__device__ __forceinline__ float row_task(float* __restrict__ wb, const float* __restrict__ ring, int pitch, int slot_y,
                                          int xoff, const float* __restrict__ win, int y, bool vec, bool store) {
    using TL = Tile<B>;
    constexpr int H = B / 2;
    constexpr int R = (T - 1) / 2;
    float X[T][B];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        const float* src = ring + (t * B + slot_y) * pitch + xoff;
        const float* w = win + (t * B + y) * TL::WP;
        float v[B];
        if (vec) {
#pragma unroll
            for (int q = 0; q < B / 4; ++q) {
                const float4 s4 = *reinterpret_cast<const float4*>(src + 4 * q);
                const float4 w4 = *reinterpret_cast<const float4*>(w + 4 * q);
                v[4 * q + 0] = s4.x * w4.x;
                v[4 * q + 1] = s4.y * w4.y;
                v[4 * q + 2] = s4.z * w4.z;
                v[4 * q + 3] = s4.w * w4.w;
            }
        } else {
#pragma unroll
            for (int x = 0; x < B; ++x) v[x] = src[x] * w[x];
        }
        if constexpr (B == 8) r2c_8(v, X[t]);
        if constexpr (B == 16) r2c_16(v, X[t]);
        if constexpr (B == 32) r2c_32(v, X[t]);
    }
    // temporal DFT over the T frames (plane p = temporal bin)
    if constexpr (T > 1) {
        // x-bins 0 and B/2: two real sequences
        float a_re[R + 1], a_im[R + 1], b_re[R + 1], b_im[R + 1];
        {
            float xa[T], xb[T];
#pragma unroll
            for (int t = 0; t < T; ++t) {
                xa[t] = X[t][0];
                xb[t] = X[t][1];
            }
            if constexpr (T == 3) { rdftT_3(xa, a_re, a_im); rdftT_3(xb, b_re, b_im); }
            if constexpr (T == 5) { rdftT_5(xa, a_re, a_im); rdftT_5(xb, b_re, b_im); }
            if constexpr (T == 7) { rdftT_7(xa, a_re, a_im); rdftT_7(xb, b_re, b_im); }
        }
        X[0][0] = a_re[0];
        X[0][1] = b_re[0];
#pragma unroll
        for (int p = 1; p <= R; ++p) {
            X[p][0] = a_re[p];
            X[p][1] = a_im[p];
            X[T - p][0] = b_re[p];
            X[T - p][1] = b_im[p];
        }
#pragma unroll
        for (int c = 1; c < H; ++c) {
            float re[T], im[T];
#pragma unroll
            for (int t = 0; t < T; ++t) {
                re[t] = X[t][2 * c];
                im[t] = X[t][2 * c + 1];
            }
            if constexpr (T == 3) cdft_3_fwd(re, im);
            if constexpr (T == 5) cdft_5_fwd(re, im);
            if constexpr (T == 7) cdft_7_fwd(re, im);
#pragma unroll
            for (int t = 0; t < T; ++t) {
                X[t][2 * c] = re[t];
                X[t][2 * c + 1] = im[t];
            }
        }
    }
    if (store) {
#pragma unroll
        for (int p = 0; p < T; ++p) {
            float* dst = wb + p * B * B;
#pragma unroll
            for (int q = 0; q < B / 4; ++q) {
                *reinterpret_cast<float4*>(dst + TL::off(y, 4 * q)) =
                    make_float4(X[p][4 * q], X[p][4 * q + 1], X[p][4 * q + 2], X[p][4 * q + 3]);
            }
        }
    }
    return X[0][0];
}

// sum over the B lanes (rows) of one block; lanes of a block are contiguous
template <int B> __device__ __forceinline__ float block_row_sum(float v) {
#pragma unroll
    for (int o = (B < 32 ? B : 32) / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// column phase helpers
// ---------------------------------------------------------------------------
template <int B> __device__ __forceinline__ void ydft_fwd(float (&re)[B], float (&im)[B]) {
    if constexpr (B == 8) cdft_8_fwd(re, im);
    if constexpr (B == 16) cdft_16_fwd(re, im);
    if constexpr (B == 32) cdft_32_fwd(re, im);
}
template <int B> __device__ __forceinline__ void ydft_inv(float (&re)[B], float (&im)[B]) {
    if constexpr (B == 8) cdft_8_inv(re, im);
    if constexpr (B == 16) cdft_16_inv(re, im);
    if constexpr (B == 32) cdft_32_inv(re, im);
}

// register index of gain slot j in plane 0 (pairs (k, B-k), then 0 and B/2)
template <int B> __host__ __device__ constexpr int slot0_reg(int j) {
    return j == 0 ? 0 : (j == 1 ? B / 2 : ((j & 1) ? B - (j >> 1) : (j >> 1)));
}

// gain of every bin of one plane held in (re, im); slot tables are [B+2][H]
template <int B, int FC, bool PLANE0>
__device__ __forceinline__ void gain_plane(float (&re)[B], float (&im)[B], const float* __restrict__ sig,
                                           const float* __restrict__ sig2, const float* __restrict__ wfe, int c,
                                           float g, bool dual, const KernelArgs& a) {
    constexpr int H = B / 2;
#pragma unroll
    for (int j = 0; j < B; ++j) {
        const int r = PLANE0 ? slot0_reg<B>(j) : j;
        const float s = sig[j * H + c];
        const float s2 = (FC != kFilterWiener && dual) ? sig2[j * H + c] : s;
        const float2 w = reinterpret_cast<const float2*>(wfe)[j * H + c];
        apply_bin<FC>(re[r], im[r], s, s2, dual, w, g, a);
    }
}

// one column task: lane (block, c) of a warp buffer block `wb`.
//
// Every temporal plane p is transformed along y, filtered, weighted by its
// centre-frame twiddle w^(p r) and summed into S.  The packed lane (c = 0)
// holds, for p <= r, the spectrum A_p of x-bin 0 and, for p > r, the
// spectrum B_q (q = T - p) of x-bin B/2; each plane enters S through its
// Hermitian part, the B planes multiplied by i, so that after plane 0 the
// packed lane holds S_A + i S_B and one inverse y-DFT yields both columns.
template <int B, int T, int FC>
__device__ __forceinline__ void column_task(float* __restrict__ wb, float g, const float* __restrict__ sm_sig,
                                            const float* __restrict__ sm_sig2, const float* __restrict__ sm_wfe, int c,
                                            bool dual_tables, const KernelArgs& a) {
    using TL = Tile<B>;
    constexpr int H = B / 2;
    constexpr int R = (T - 1) / 2;
    constexpr int NSLOT = B + 2;
    const bool packed = (c == 0);
    const bool dual = dual_tables && packed;

    float sr[B], si[B];
#pragma unroll
    for (int k = 0; k < B; ++k) sr[k] = si[k] = 0.0f;
    float qr[B], qi[B];

#pragma unroll
    for (int p = 1; p < T; ++p) {
        const float* src = wb + p * B * B;
#pragma unroll
        for (int y = 0; y < B; ++y) {
            const float2 v = *reinterpret_cast<const float2*>(src + TL::off(y, 2 * c));
            qr[y] = v.x;
            qi[y] = v.y;
        }
        ydft_fwd<B>(qr, qi);
        gain_plane<B, FC, false>(qr, qi, sm_sig + p * NSLOT * H, sm_sig2 + p * NSLOT * H, sm_wfe + 2 * p * NSLOT * H,
                                 c, g, dual, a);
        // twiddle: w^(p r) = (tc, ts); packed lane on a B plane uses i * conj(w^(p r))
        const float tc = CentreTwiddle<T>::re(p), ts = CentreTwiddle<T>::im(p);
        const bool swap = packed && (p > R);
        const float twr = swap ? ts : tc;
        const float twi = swap ? tc : ts;
#pragma unroll
        for (int k = 0; k < B; ++k) {
            const float vr = fmaf(qr[k], twr, -qi[k] * twi);
            const float vi = fmaf(qr[k], twi, qi[k] * twr);
            qr[k] = vr;
            qi[k] = vi;
        }
        if (packed) {
            // Hermitian part (A planes) or anti-Hermitian part (i * B planes)
            const float sg = (p <= R) ? 1.0f : -1.0f;
            qr[0] = qr[0] + sg * qr[0];
            qi[0] = qi[0] - sg * qi[0];
            qr[H] = qr[H] + sg * qr[H];
            qi[H] = qi[H] - sg * qi[H];
#pragma unroll
            for (int k = 1; k < H; ++k) {
                const float ar = qr[k], ai = qi[k], br = qr[B - k], bi = qi[B - k];
                qr[k] = fmaf(sg, br, ar);
                qi[k] = fmaf(-sg, bi, ai);
                qr[B - k] = fmaf(sg, ar, br);
                qi[B - k] = fmaf(-sg, ai, bi);
            }
        }
#pragma unroll
        for (int k = 0; k < B; ++k) {
            sr[k] += qr[k];
            si[k] += qi[k];
        }
    }

    // plane 0 last
#pragma unroll
    for (int y = 0; y < B; ++y) {
        const float2 v = *reinterpret_cast<const float2*>(wb + TL::off(y, 2 * c));
        qr[y] = v.x;
        qi[y] = v.y;
    }
    ydft_fwd<B>(qr, qi);
    float e1r = 0.0f, e1i = 0.0f, e2r = 0.0f, e2i = 0.0f;
    if (packed) {
        // untangle Q = A + iB (A, B Hermitian): A -> reg k, B -> reg B-k
#pragma unroll
        for (int k = 1; k < H; ++k) {
            const float ar = qr[k], ai = qi[k], br = qr[B - k], bi = qi[B - k];
            qr[k] = 0.5f * (ar + br);
            qi[k] = 0.5f * (ai - bi);
            qr[B - k] = 0.5f * (ai + bi);
            qi[B - k] = 0.5f * (br - ar);
        }
        e1r = qr[H];
        e2r = qi[H];
        qr[H] = qi[0];
        qi[H] = 0.0f;
        qi[0] = 0.0f;
    }
    gain_plane<B, FC, true>(qr, qi, sm_sig, sm_sig2, sm_wfe, c, g, dual, a);
    if (packed) {
        const float2 w1 = reinterpret_cast<const float2*>(sm_wfe)[B * H + c];
        const float2 w2 = reinterpret_cast<const float2*>(sm_wfe)[(B + 1) * H + c];
        apply_bin<FC>(e1r, e1i, sm_sig[B * H + c], dual ? sm_sig2[B * H + c] : 0.0f, dual, w1, g, a);
        apply_bin<FC>(e2r, e2i, sm_sig[(B + 1) * H + c], dual ? sm_sig2[(B + 1) * H + c] : 0.0f, dual, w2, g, a);
        // add Y_A0 + i Y_B0, both Hermitian in y
        sr[0] += qr[0];
        si[0] += qr[H];
        sr[H] += e1r;
        si[H] += e2r;
#pragma unroll
        for (int k = 1; k < H; ++k) {
            const float ar = qr[k], ai = qi[k], br = qr[B - k], bi = qi[B - k];
            sr[k] += ar - bi;
            si[k] += ai + br;
            sr[B - k] += ar + bi;
            si[B - k] += br - ai;
        }
    } else {
#pragma unroll
        for (int k = 0; k < B; ++k) {
            sr[k] += qr[k];
            si[k] += qi[k];
        }
    }
    ydft_inv<B>(sr, si);
#pragma unroll
    for (int y = 0; y < B; ++y) *reinterpret_cast<float2*>(wb + TL::off(y, 2 * c)) = make_float2(sr[y], si[y]);
}

// inverse rows: packed row -> real, synthesis window, in place
template <int B>
__device__ __forceinline__ void inverse_row_task(float* __restrict__ wb, const float* __restrict__ wsyn, int y) {
    using TL = Tile<B>;
    float v[B], o[B];
#pragma unroll
    for (int q = 0; q < B / 4; ++q) {
        const float4 s4 = *reinterpret_cast<const float4*>(wb + TL::off(y, 4 * q));
        v[4 * q] = s4.x;
        v[4 * q + 1] = s4.y;
        v[4 * q + 2] = s4.z;
        v[4 * q + 3] = s4.w;
    }
    if constexpr (B == 8) c2r_8(v, o);
    if constexpr (B == 16) c2r_16(v, o);
    if constexpr (B == 32) c2r_32(v, o);
    const float* w = wsyn + y * TL::WP;
#pragma unroll
    for (int q = 0; q < B / 4; ++q) {
        const float4 w4 = *reinterpret_cast<const float4*>(w + 4 * q);
        *reinterpret_cast<float4*>(wb + TL::off(y, 4 * q)) =
            make_float4(o[4 * q] * w4.x, o[4 * q + 1] * w4.y, o[4 * q + 2] * w4.z, o[4 * q + 3] * w4.w);
    }
}

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// ---------------------------------------------------------------------------
// main kernel
// ---------------------------------------------------------------------------
template <int B, int T, int NW, int FC>
__global__ void __launch_bounds__(NW * 32, NW <= 4 ? 2 : 1) dfttest_unit_kernel(const __grid_constant__ KernelArgs a) {
    using L = Layout<B, T, NW>;
    using TL = Tile<B>;
    constexpr int H = B / 2;
    constexpr int BPW = 64 / B;
    constexpr int BPS = NW * BPW;  // blocks per step
    constexpr int NT = NW * 32;
    extern __shared__ __align__(16) float sm[];

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int S = a.block_step;
    const int O = B - S;
    const int pitch = a.ring_pitch;

    // --- locate the unit ---------------------------------------------------
    const int uid = blockIdx.x;
    int lo = 0, hi = a.njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.jobs[mid].unit_base <= uid) lo = mid; else hi = mid - 1;
    }
    const PlaneJob& job = a.jobs[lo];
    const int W = job.width, Hh = job.height;
    const int pw = pad_size(W, B, S), ph = pad_size(Hh, B, S);
    const int pnx = (pw - B) / S + 1, pny = (ph - B) / S + 1;
    const int ox = (pw - W) / 2, oy = (ph - Hh) / 2;
    const int lid = uid - job.unit_base;
    const int sx = lid % job.nsx, sy = lid / job.nsx;
    const UnitGeom u = unit_geom(sx, sy, job.nsx, job.nsy, pnx, pny, B, S);
    const int nbx = u.bx1 - u.bx0;
    if (nbx > BPS) {
        if (tid == 0) atomicExch(a.error_flag, 1);
        return;
    }
    float* rec = a.scratch + (size_t)uid * a.rec_stride;
    const bool is_float = (a.kind == kF32);
    const float inv_scale = 1.0f / a.scale;  // exact for the power-of-two integer scales

    // --- constants into shared memory -----------------------------------
    float* s_win = sm + L::o_win;
    float* s_wsyn = sm + L::o_wsyn;
    float* s_sig = sm + L::o_sig;
    float* s_sig2 = sm + L::o_sig2;
    float* s_wfe = sm + L::o_wfe;
    float* s_g = sm + L::o_g;
    float* s_wbuf = sm + L::o_wbuf;
    float* s_in = sm + L::o_ring;
    float* s_ola = s_in + L::in_ring_floats(pitch);
    // scale * window, rounded once as in load_block (cpu_source/getframe_impl.cpp:137)
    for (int i = tid; i < T * B * B; i += NT) s_win[(i / B) * TL::WP + (i % B)] = a.scale * a.win[i];
    for (int i = tid; i < B * B; i += NT) s_wsyn[(i / B) * TL::WP + (i % B)] = a.wsyn[i];
    const bool dual_tables = (FC != kFilterWiener) && a.sig2 != nullptr;
    for (int i = tid; i < T * L::NSLOT * H; i += NT) {
        s_sig[i] = a.sig[i];
        if (dual_tables) s_sig2[i] = a.sig2[i];
    }
    for (int i = tid; i < 2 * T * L::NSLOT * H; i += NT) s_wfe[i] = a.wfe[i];
    for (int i = tid; i < L::ola_floats(pitch); i += NT) s_ola[i] = 0.0f;

    const int fw = u.fw;
    const int x0 = u.bx0 * S;  // footprint origin (padded coordinates)
    const bool vec = ((S & 3) == 0);
    const float inv_fw = 1.0f / (float)fw;

    for (int by = u.by0; by <= u.by1; ++by) {
        // ---- finalize rows of the previous step + stage input rows of this one
        if (by > u.by0) {
            const int pb = by - 1;
            const bool last = (pb == u.by1 - 1);
            const int nrows = last ? B : S;
            const int excl_y0 = u.by0 * S + O, excl_y1 = u.by1 * S;
            const int excl_x0 = x0 + O, excl_x1 = u.bx1 * S;
            for (int i = tid; i < nrows * fw; i += NT) {
                const int r = div_small(i, inv_fw);
                const int lx = i - r * fw;
                const int py = pb * S + r;
                float* cell = s_ola + (py % B) * pitch + lx;
                const float v = *cell;
                *cell = 0.0f;
                const int px = x0 + lx;
                if (px < ox || px >= ox + W || py < oy || py >= oy + Hh) continue;
                const bool excl = (px >= excl_x0) && (px < excl_x1) && (py >= excl_y0) && (py < excl_y1);
                if (excl) {
                    store_sample(job.dst, (long long)(py - oy) * job.dst_stride + (px - ox), v, a.kind, a.scale,
                                 a.peak, is_float ? 0.0f : inv_scale);
                } else {
                    rec[band_index(lx, py - u.by0 * S, fw, u.fh, O)] = v;
                }
            }
        }
        if (by == u.by1) break;
        {
            const int r_lo = (by == u.by0) ? by * S : by * S + B - S;
            const int r_hi = by * S + B;
            const int nr = r_hi - r_lo;
            const int rowlen = nbx * S + O;  // footprint width of this step
            for (int row = warp; row < T * nr; row += NW) {
                const int t = row / nr;
                const int py = r_lo + (row - t * nr);
                const long long sy_ = mirror(py - oy, Hh);
                const void* base = job.src[t];
                for (int lx = lane; lx < rowlen; lx += 32) {
                    const int sx_ = mirror(x0 + lx - ox, W);
                    s_in[(t * B + (py % B)) * pitch + lx] = load_sample(base, sy_ * job.src_stride + sx_, a.kind);
                }
            }
            // warm L2 with the rows of the next step (one request per 128 B)
            if (by + 1 < u.by1) {
                const int npy = r_hi;  // first new row of the next step
                const int esz = a.kind == kF32 ? 4 : (a.kind == kU16 ? 2 : 1);
                const int sx_lo = max(x0 - ox, 0), sx_hi = max(min(x0 + rowlen - ox, W) - 1, sx_lo);
                const int nline = (int)(((long long)(sx_hi - sx_lo) * esz) / 128) + 2;
                for (int i = tid; i < T * S * nline; i += NT) {
                    const int t = i / (S * nline);
                    const int rem = i - t * S * nline;
                    const int r = rem / nline, li = rem - r * nline;
                    const int py = npy + r;
                    if (py >= ph) continue;
                    const long long sy_ = mirror(py - oy, Hh);
                    const int sxp = min(sx_lo + li * (128 / esz), sx_hi);
                    prefetch_l2(reinterpret_cast<const char*>(job.src[t]) + (sy_ * job.src_stride + sxp) * esz);
                }
            }
        }
        __syncthreads();

        // ---- per-warp block transforms
        {
            float* wb0 = s_wbuf + warp * BPW * L::BSTR;
            // row phase: 2 tasks per lane; the DC of each block is summed
            // over its rows with shuffles (lanes of a block are contiguous)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int gr = k * 32 + lane;
                const int b = gr / B, y = gr % B;
                const int bl = warp * BPW + b;
                const bool valid = bl < nbx;
                const int blr = valid ? bl : nbx - 1;
                const float dc = row_task<B, T>(wb0 + b * L::BSTR, s_in, pitch, (by * S + y) % B, blr * S, s_win, y,
                                                vec, valid);
                const float tot = block_row_sum<B>(dc);
                // g = DC / Re(WF[0]) (cpu_source/kernel.hpp:1945)
                if (y == 0 && valid) s_g[warp * BPW + b] = a.g_div != 0.0f ? __fdiv_rn(tot, a.g_div) : 0.0f;
            }
            __syncwarp();
            {
                const int b = lane / H, c = lane % H;
                const int bl = warp * BPW + b;
                if (bl < nbx)
                    column_task<B, T, FC>(wb0 + b * L::BSTR, s_g[warp * BPW + b], s_sig, s_sig2, s_wfe, c, dual_tables,
                                          a);
            }
            __syncwarp();
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int gr = k * 32 + lane;
                const int b = gr / B, y = gr % B;
                const int bl = warp * BPW + b;
                if (bl < nbx) inverse_row_task<B>(wb0 + b * L::BSTR, s_wsyn, y);
            }
        }
        __syncthreads();

        // ---- overlap-add: every ring pixel sums the blocks covering it
        {
            const int rowlen = nbx * S + O;
            if (vec) {
                const int nq = rowlen >> 2;
                const float inv_nq = 1.0f / (float)nq;
                for (int i = tid; i < B * nq; i += NT) {
                    const int r = div_small(i, inv_nq), q = i - r * nq;
                    const int px = 4 * q;
                    int b_lo = px - B + 4;
                    b_lo = b_lo <= 0 ? 0 : (b_lo + S - 1) / S;
                    int b_hi = px / S;
                    b_hi = b_hi < nbx - 1 ? b_hi : nbx - 1;
                    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
                    for (int bl = b_lo; bl <= b_hi; ++bl) {
                        const float* ob = s_wbuf + bl * L::BSTR;
                        const float4 v = *reinterpret_cast<const float4*>(ob + TL::off(r, px - bl * S));
                        acc.x += v.x;
                        acc.y += v.y;
                        acc.z += v.z;
                        acc.w += v.w;
                    }
                    float4* cell = reinterpret_cast<float4*>(s_ola + ((by * S + r) % B) * pitch + px);
                    float4 c4 = *cell;
                    c4.x += acc.x;
                    c4.y += acc.y;
                    c4.z += acc.z;
                    c4.w += acc.w;
                    *cell = c4;
                }
            } else {
                const float inv_rl = 1.0f / (float)rowlen;
                for (int i = tid; i < B * rowlen; i += NT) {
                    const int r = div_small(i, inv_rl), px = i - r * rowlen;
                    int b_lo = px - B + 1;
                    b_lo = b_lo <= 0 ? 0 : (b_lo + S - 1) / S;
                    int b_hi = px / S;
                    b_hi = b_hi < nbx - 1 ? b_hi : nbx - 1;
                    float acc = 0.0f;
                    for (int bl = b_lo; bl <= b_hi; ++bl) acc += s_wbuf[bl * L::BSTR + TL::off(r, px - bl * S)];
                    s_ola[((by * S + r) % B) * pitch + px] += acc;
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// fix-up: pixels shared by neighbouring units
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cover(int p, int S, int O, int pn, int ns, int& s_lo, int& s_hi) {
    // units whose footprint [lo*S, hi*S + O) contains padded coordinate p
    int b = p / S;
    b = b < pn - 1 ? b : pn - 1;
    int s = (int)(((long long)b * ns) / pn);
    while (s + 1 < ns && split_lo(s + 1, pn, ns) <= b) ++s;
    while (s > 0 && split_lo(s, pn, ns) > b) --s;
    s_hi = s;
    s_lo = s;
    while (s_lo > 0 && p < split_lo(s_lo, pn, ns) * S + O) --s_lo;
}

template <int B>
__global__ void __launch_bounds__(256) dfttest_fixup_kernel(const __grid_constant__ KernelArgs a) {
    const int S = a.block_step;
    const int O = B - S;
    for (int gid = blockIdx.x * blockDim.x + threadIdx.x; gid < a.nfix; gid += gridDim.x * blockDim.x) {
        int lo = 0, hi = a.njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.jobs[mid].fix_base <= gid) lo = mid; else hi = mid - 1;
        }
        const PlaneJob& job = a.jobs[lo];
        const int W = job.width, Hh = job.height;
        const int pw = pad_size(W, B, S), ph = pad_size(Hh, B, S);
        const int pnx = (pw - B) / S + 1, pny = (ph - B) / S + 1;
        const int ox = (pw - W) / 2, oy = (ph - Hh) / 2;
        int idx = gid - job.fix_base;
        const int nv = (job.nsx - 1) * O * Hh;
        int px, py;
        if (idx < nv) {
            const int k = idx / (O * Hh);
            const int rem = idx - k * O * Hh;
            py = oy + rem / O;
            px = split_lo(k + 1, pnx, job.nsx) * S + rem % O;
        } else {
            idx -= nv;
            const int j = idx / (O * W);
            const int rem = idx - j * O * W;
            px = ox + rem % W;
            py = split_lo(j + 1, pny, job.nsy) * S + rem / W;
            int sxl, sxh;
            cover(px, S, O, pnx, job.nsx, sxl, sxh);
            if (sxl != sxh) continue;  // handled by the vertical zone
        }
        if (px < ox || px >= ox + W || py < oy || py >= oy + Hh) continue;
        int sxl, sxh, syl, syh;
        cover(px, S, O, pnx, job.nsx, sxl, sxh);
        cover(py, S, O, pny, job.nsy, syl, syh);
        float acc = 0.0f;
        for (int sy = syl; sy <= syh; ++sy) {
            for (int sx = sxl; sx <= sxh; ++sx) {
                const UnitGeom u = unit_geom(sx, sy, job.nsx, job.nsy, pnx, pny, B, S);
                const int uid = job.unit_base + sy * job.nsx + sx;
                acc += a.scratch[(size_t)uid * a.rec_stride + band_index(px - u.bx0 * S, py - u.by0 * S, u.fw, u.fh, O)];
            }
        }
        store_sample(job.dst, (long long)(py - oy) * job.dst_stride + (px - ox), acc, a.kind, a.scale, a.peak);
    }
}

}  // namespace dft2
