// Adjoint of the DFTTest per-plane pipeline (float planes): gradients of a
// loss w.r.t. the input pixels and the per-bin sigma array, given the
// gradient w.r.t. the output plane.
//
// Forward (per block, reference semantics cpu_source/kernel.hpp:1899-1983,
// cpu_source/getframe_impl.cpp:105-221):
//   z = scale * w .* gather(x)          Z = DFT3(z) (real x, then y, then t)
//   g = Re Z(0) / Re WF(0)              d = Z - g WF
//   Y = m(|d|^2, sigma) d + g WF        y = c2r_x(IDFT_y(sum_t w^(t r) Y))   (centre frame)
//   out += w_syn .* y,  out / scale
// Adjoint, per block, with G = dL/dRe + i dL/dIm for complex quantities:
//   gy  = w_syn .* dL/dout / scale           (transposed overlap-add)
//   Gy  = c_k * DFT_y(r2c_x(gy)),  c_k = 2 for 0 < kx < B/2 else 1
//   G   = conj(w^(kt r)) Gy                  (every temporal bin)
//   dd  = m G + 2 m'(psd) Re(conj(G) d) d,    dsigma += dm/dsigma Re(conj(G) d)
//   dg  = sum Re(conj(G) WF) - Re(conj(dd) WF),  dZ = dd (+ dg / Re WF(0) on bin 0)
//   dz  = c2r_x(h_k * IDFT_y(IDFT_t(dZ))),  h_k = 1/2 for 0 < kx < B/2 else 1
//   dx += scale * w .* dz                    (transposed gather, through the mirror)
// Block spectra are recomputed from the input, not stored by the forward.
// A CTA takes a tile of neighbouring blocks at a time (persistent grid over
// tiles); the sigma gradient is summed in shared memory across the tiles and
// added to global memory once per CTA.  DFT_t, the gain adjoint and IDFT_t
// run in one pass, in registers, per (ky, kx) bin.
#pragma once

#include "dfttest_kernel.cuh"

namespace dft2 {

struct GradJob {
    const float* src[7];   // the 2r+1 input planes (time clamp applied)
    float* gsrc[7];        // their gradient accumulators (added to)
    const float* gdst;     // gradient w.r.t. the output plane
    long long src_stride, gsrc_stride, gdst_stride;  // elements
    int width, height;
    int tile_base;         // first global tile id of this job
    int ntx;               // tiles per tile row
};

struct AdjointArgs {
    const GradJob* jobs;
    int njobs;
    int ntiles;
    float scale;
    int block_step;
    int filter_type;
    float sigma2, pmin, pmax;
    int zero_mean;
    int patch_h, patch_w;  // source-gradient patch of a tile: B + (TBY-1) S rows, B + (TBX-1) S columns
    const float* win;      // [T][B][B]
    const float* wsyn;     // [B][B]
    const float* sigma;    // [T][B][X]
    const float* wf;       // [T][B][X][2]
    float* gsigma;         // [T][B][X], added to (may be null)
};

// m(psd, s) of frequency_filtering and its partial derivatives, for filter type FT
template <int FT>
__device__ __forceinline__ void gain_grad(float psd, float s, const AdjointArgs& a, float& m, float& dpsd,
                                          float& dsig) {
    const float eps = 1e-15f;
    dpsd = 0.0f;
    dsig = 0.0f;
    if constexpr (FT == 0) {
        // one MUFU reciprocal (< 1 ulp, as the forward kernel's Wiener gain) for the quotient and
        // both derivatives
        const float r = rcp_approx(psd + eps);
        const float u = (psd - s) * r;
        m = fmaxf(u, 0.0f);
        if (u > 0.0f) {
            dpsd = (s + eps) * r * r;
            dsig = -r;
        }
    } else if constexpr (FT == 1) {
        m = psd < s ? 0.0f : 1.0f;
    } else if constexpr (FT == 2) {
        m = s;
        dsig = 1.0f;
    } else if constexpr (FT == 3) {
        const bool in = psd >= a.pmin && psd <= a.pmax;
        m = in ? s : a.sigma2;
        dsig = in ? 1.0f : 0.0f;
    } else if constexpr (FT == 4) {
        const float D = (psd + a.pmin) * (psd + a.pmax) + eps;
        const float rD = rcp_approx(D);
        const float h = psd * a.pmax * rD;
        const float sh = sqrtf(h);
        m = s * sh;
        dsig = sh;
        if (h > 0.0f) {
            const float dh = a.pmax * rD - psd * a.pmax * (2.0f * psd + a.pmin + a.pmax) * rD * rD;
            dpsd = 0.5f * s * dh * rcp_approx(sh);
        }
    } else {  // 5: u^pmin, 6: sqrt(u)
        const float den = psd + eps;
        const float u0 = (psd - s) / den;
        const float u = fmaxf(u0, 0.0f);
        const float p = FT == 5 ? a.pmin : 0.5f;
        m = FT == 5 ? powf(u, p) : sqrtf(u);
        if (u0 > 0.0f) {
            const float dmu = p * m / u;
            dpsd = dmu * (s + eps) / (den * den);
            dsig = -dmu / den;
        }
    }
}

template <int V> struct IntC {
    static constexpr int value = V;
};

template <int B> __device__ __forceinline__ void r2c_n(const float (&x)[B], float (&y)[B]) {
    if constexpr (B == 8) r2c_8(x, y);
    if constexpr (B == 16) r2c_16(x, y);
    if constexpr (B == 32) r2c_32(x, y);
}
template <int B> __device__ __forceinline__ void c2r_n(const float (&y)[B], float (&x)[B]) {
    if constexpr (B == 8) c2r_8(y, x);
    if constexpr (B == 16) c2r_16(y, x);
    if constexpr (B == 32) c2r_32(y, x);
}
template <int N> __device__ __forceinline__ void cdft_n(float (&re)[N], float (&im)[N], bool inverse) {
    if constexpr (N == 3) {
        if (inverse) {
            for (int k = 0; k < N; ++k) im[k] = -im[k];
            cdft_3_fwd(re, im);
            for (int k = 0; k < N; ++k) im[k] = -im[k];
        } else {
            cdft_3_fwd(re, im);
        }
    }
    if constexpr (N == 5) {
        if (inverse) {
            for (int k = 0; k < N; ++k) im[k] = -im[k];
            cdft_5_fwd(re, im);
            for (int k = 0; k < N; ++k) im[k] = -im[k];
        } else {
            cdft_5_fwd(re, im);
        }
    }
    if constexpr (N == 7) {
        if (inverse) {
            for (int k = 0; k < N; ++k) im[k] = -im[k];
            cdft_7_fwd(re, im);
            for (int k = 0; k < N; ++k) im[k] = -im[k];
        } else {
            cdft_7_fwd(re, im);
        }
    }
    if constexpr (N == 8) { if (inverse) cdft_8_inv(re, im); else cdft_8_fwd(re, im); }
    if constexpr (N == 16) { if (inverse) cdft_16_inv(re, im); else cdft_16_fwd(re, im); }
    if constexpr (N == 32) { if (inverse) cdft_32_inv(re, im); else cdft_32_fwd(re, im); }
}

// Tile geometry of the adjoint: TBX x TBY neighbouring blocks per CTA and
// tile, NTH threads.  All threads work on all blocks of the tile in every
// phase; the tile's source gradient is accumulated in shared memory and added
// to global memory once per tile.
template <int B, int T>
struct AdjTile {
    static constexpr int X = B / 2 + 1;
    static constexpr int SPEC = T * B * X;  // complex bins of a block
    // 8x8 and 16x16 blocks with up to 3 frames: tiles of 4 x 3 blocks on 12
    // warps (two CTAs per SM at up to 85 registers); longer temporal sizes
    // and 32x32 blocks need more registers per thread and run 8 warps
    static constexpr bool WIDE = B <= 16 && T <= 3;
    static constexpr int TBX = B == 32 ? 2 : 4;
    static constexpr int TBY = WIDE ? 3 : (B == 32 ? (T >= 5 ? 1 : 2) : (B == 16 && T >= 5 ? 2 : 4));
    static constexpr int NBLK = TBX * TBY;
    static constexpr int NTH = WIDE ? 384 : 256;
    static constexpr int GT = NTH / NBLK;              // threads per block in the gain phase
    static_assert(NTH % NBLK == 0 && (GT & (GT - 1)) == 0, "the zero-mean reduction shuffles over a power of two");
    static constexpr int NPER = (B * X + GT - 1) / GT;  // (ky, kx) bins per thread in the gain phase
    // shared memory (floats), in order
    // window rows WP = B + 1 floats apart: the row tasks of a warp differ in y and read the same x
    static constexpr int WP = B + 1;
    static constexpr int o_win = 0;                    // scale * window   [T][B][WP]
    static constexpr int o_wsyn = o_win + T * B * WP;  // wsyn / scale     [B][WP]
    static constexpr int o_sig = o_wsyn + B * WP;      // sigma            [SPEC]
    static constexpr int o_wf = o_sig + SPEC;          // window spectrum  [SPEC][2]
    static constexpr int o_tw = o_wf + 2 * SPEC;       // conj temporal twiddles [T][2]
    static_assert(o_wf % 2 == 0, "the window spectrum is read as float2");
    static constexpr int o_dg = o_tw + 2 * T;          // zero-mean partials [NBLK]
    static constexpr int o_gs = o_dg + NBLK;           // sigma-gradient partials of the CTA [SPEC]
    // spectra [NBLK][T][B][X]: temporal planes TS floats apart, TS = X (mod
    // 32), so that the X-bin runs of the T planes that the column passes read
    // side by side fall in disjoint shared-memory banks
    static constexpr int TS = B * X + (((X - B * X) % 32) + 32) % 32;
    static constexpr int ZB = T * TS;                  // floats per block
    static constexpr int o_zr = (o_gs + SPEC + 3) & ~3;  // spectra [NBLK][ZB]
    static constexpr int o_zi = o_zr + NBLK * ZB;
    static constexpr int o_gr = o_zi + NBLK * ZB;      // output-gradient spectra [NBLK][B][X]
    static constexpr int o_gi = o_gr + NBLK * B * X;
    static constexpr int o_dx = o_gi + NBLK * B * X;   // the tile's source patch, then its gradient [T][patch_h][pitch]
    // patch rows are an odd number of floats apart (bank spread of the row tasks)
    __host__ __device__ static int patch_pitch(int pw) { return pw | 1; }
    static size_t smem_bytes(int ph, int pw) {
        return sizeof(float) * ((size_t)o_dx + (size_t)T * ph * patch_pitch(pw));
    }
};

// rows of a packed real-spectrum layout <-> complex (kx = 0..B/2) arrays
template <int B>
__device__ __forceinline__ void packed_to_complex(const float (&y)[B], float* re, float* im) {
    re[0] = y[0];
    im[0] = 0.0f;
    re[B / 2] = y[1];
    im[B / 2] = 0.0f;
#pragma unroll
    for (int k = 1; k < B / 2; ++k) {
        re[k] = y[2 * k];
        im[k] = y[2 * k + 1];
    }
}

template <int B, int T>
__global__ void __launch_bounds__(AdjTile<B, T>::NTH, 2) dfttest_adjoint_kernel(const __grid_constant__ AdjointArgs a) {
    using L = AdjTile<B, T>;
    constexpr int X = L::X, SPEC = L::SPEC, NBLK = L::NBLK, TBX = L::TBX, TBY = L::TBY, GT = L::GT;
    constexpr int TS = L::TS, ZB = L::ZB, WP = L::WP;
    constexpr int R = (T - 1) / 2;
    extern __shared__ __align__(16) float smem[];
    float* s_win = smem + L::o_win;
    float* s_wsyn = smem + L::o_wsyn;
    float* s_sig = smem + L::o_sig;
    float* s_wf = smem + L::o_wf;
    float* s_tw = smem + L::o_tw;
    float* s_dg = smem + L::o_dg;
    float* zr = smem + L::o_zr;
    float* zi = smem + L::o_zi;
    float* gr = smem + L::o_gr;
    float* gi = smem + L::o_gi;
    float* dxp = smem + L::o_dx;
    const int tid = threadIdx.x;
    const int S = a.block_step, PH = a.patch_h, PW = a.patch_w, PP = L::patch_pitch(a.patch_w);

    for (int i = tid; i < T * B * B; i += L::NTH) s_win[(i / B) * WP + i % B] = a.scale * a.win[i];
    for (int i = tid; i < B * B; i += L::NTH) s_wsyn[(i / B) * WP + i % B] = a.wsyn[i] / a.scale;
    for (int i = tid; i < SPEC; i += L::NTH) {
        s_sig[i] = a.sigma[i];
        s_wf[2 * i] = a.zero_mean ? a.wf[2 * i] : 0.0f;
        s_wf[2 * i + 1] = a.zero_mean ? a.wf[2 * i + 1] : 0.0f;
    }
    if (tid < T) {
        float sn, cs;
        sincosf(-6.283185307179586f * (float)((tid * R) % T) / (float)T, &sn, &cs);
        s_tw[2 * tid] = cs;
        s_tw[2 * tid + 1] = sn;
    }
    const float wf0 = a.zero_mean ? a.wf[0] : 1.0f;
    // gain-phase ownership: block gblk of the tile, bins gj + k GT
    const int gblk = tid / GT, gj = tid - gblk * GT;
    // sigma-gradient partials of the CTA (summed over its tiles in shared
    // memory rather than registers, which leaves room for a third CTA per SM)
    float* s_gs = smem + L::o_gs;
    for (int i = tid; i < SPEC; i += L::NTH) s_gs[i] = 0.0f;

    const int lane = tid & 31, warp = tid >> 5;
    int jn = 0;  // job of the current tile: a CTA visits its tiles in increasing order
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        if (jn + 1 < a.njobs && a.jobs[jn + 1].tile_base <= tile) {
            int lo = jn + 1, hi = a.njobs - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (a.jobs[mid].tile_base <= tile) lo = mid; else hi = mid - 1;
            }
            jn = lo;
        }
        const GradJob& job = a.jobs[jn];
        const int W = job.width, Hh = job.height;
        const int pw = pad_size(W, B, S), ph = pad_size(Hh, B, S);
        const int pnx = (pw - B) / S + 1, pny = (ph - B) / S + 1;
        const int ox = (pw - W) / 2, oy = (ph - Hh) / 2;
        const int lt = tile - job.tile_base;
        const int ty = lt / job.ntx, tx = lt - ty * job.ntx;
        const int bx0 = tx * TBX, by0 = ty * TBY;
        if (tid < NBLK) s_dg[tid] = 0.0f;
        const int py0 = by0 * S, px0 = bx0 * S;
        // walks the T x PH x PW patch: rows per warp (frame, row and mirrored row warp-uniform),
        // columns per lane (mirrored column computed once per lane and column group)
        auto over_patch = [&](auto&& body) {
            for (int c = lane; c < PW; c += 32) {
                const int px = px0 + c;
                const bool cin = px < pw;
                const int mx = cin ? mirror(px - ox, W) : 0;
#pragma unroll
                for (int t = 0; t < T; ++t)
                    for (int r = warp; r < PH; r += L::NTH / 32) {
                        const int py = py0 + r;
                        const bool in = cin && py < ph;
                        body(t, r, c, in, (long long)(py < ph ? mirror(py - oy, Hh) : 0), mx);
                    }
            }
        };
        __syncthreads();  // tables and the previous tile's flush are complete
        // the tile's source patch through the mirror, coalesced
        over_patch([&](int t, int r, int c, bool in, long long my, int mx) {
            dxp[(t * PH + r) * PP + c] = in ? __ldg(job.src[t] + my * job.src_stride + mx) : 0.0f;
        });
        __syncthreads();

        // ---- rows: r2c_x of the windowed source blocks (t < T) and of the
        //      weighted output gradient (t == T, bins 0 < kx < B/2 doubled)
        for (int task = tid; task < NBLK * (T + 1) * B; task += L::NTH) {
            const int blk = task / ((T + 1) * B), rem = task - blk * ((T + 1) * B);
            const int t = rem / B, y = rem - t * B;
            const int bx = bx0 + blk % TBX, by = by0 + blk / TBX;
            const bool valid = bx < pnx && by < pny;
            const int py = by * S + y, px0 = bx * S;
            float v[B], o[B];
            if (t < T) {
                if (valid) {
                    const float* row = dxp + (t * PH + (blk / TBX) * S + y) * PP + (blk % TBX) * S;
#pragma unroll
                    for (int x = 0; x < B; ++x) v[x] = s_win[(t * B + y) * WP + x] * row[x];
                } else {
#pragma unroll
                    for (int x = 0; x < B; ++x) v[x] = 0.0f;
                }
                r2c_n<B>(v, o);
                packed_to_complex<B>(o, zr + blk * ZB + t * TS + y * X, zi + blk * ZB + t * TS + y * X);
            } else {
                const bool rin = valid && py >= oy && py < oy + Hh;
                const float* row = job.gdst + (long long)(rin ? py - oy : 0) * job.gdst_stride;
#pragma unroll
                for (int x = 0; x < B; ++x) {
                    const int px = px0 + x;
                    v[x] = rin && px >= ox && px < ox + W ? __ldg(row + px - ox) * s_wsyn[y * WP + x] : 0.0f;
                }
                r2c_n<B>(v, o);
                float* dr = gr + blk * B * X + y * X;
                float* di = gi + blk * B * X + y * X;
                packed_to_complex<B>(o, dr, di);
#pragma unroll
                for (int k = 1; k < B / 2; ++k) {
                    dr[k] *= 2.0f;
                    di[k] *= 2.0f;
                }
            }
        }
        __syncthreads();
        // the patch now accumulates the source gradient (used again after the inverse transforms)
        for (int i = tid; i < T * PH * PP; i += L::NTH) dxp[i] = 0.0f;

        // ---- columns: DFT_y of every (t, kx) column and of the gradient columns
        for (int task = tid; task < NBLK * (T + 1) * X; task += L::NTH) {
            const int blk = task / ((T + 1) * X), rem = task - blk * ((T + 1) * X);
            const int t = rem / X, kx = rem - t * X;
            float* pr = t < T ? zr + blk * ZB + t * TS + kx : gr + blk * B * X + kx;
            float* pi = t < T ? zi + blk * ZB + t * TS + kx : gi + blk * B * X + kx;
            float re[B], im[B];
#pragma unroll
            for (int y = 0; y < B; ++y) {
                re[y] = pr[y * X];
                im[y] = pi[y * X];
            }
            cdft_n<B>(re, im, false);
#pragma unroll
            for (int y = 0; y < B; ++y) {
                pr[y * X] = re[y];
                pi[y * X] = im[y];
            }
        }
        __syncthreads();

        // ---- per (ky, kx) bin: DFT_t, the gain and its adjoint, the inverse DFT_t, in registers;
        //      thread owns bins gj + k GT of block gblk (every temporal bin of each)
        {
            constexpr int BX = B * X;
            float* br = zr + gblk * ZB;
            float* bi = zi + gblk * ZB;
            const float* cr = gr + gblk * B * X;
            const float* ci = gi + gblk * B * X;
            // g = Re Z(0) / Re WF(0), Z(0) = the sum over the frames of bin (0, 0)
            float g = 0.0f;
            if (a.zero_mean) {
#pragma unroll
                for (int t = 0; t < T; ++t) g += br[t * TS];
                g /= wf0;
            }
            float dg = 0.0f;
            // the filter type is uniform: one switch around the bins keeps the executed code one straight run
            auto bins = [&](auto ftc) {
                constexpr int FT = decltype(ftc)::value;
#pragma unroll
                for (int k = 0; k < L::NPER; ++k) {
                    const int bin = gj + k * GT;
                    if (BX % GT == 0 || bin < BX) {
                        float re[T], im[T];
#pragma unroll
                        for (int t = 0; t < T; ++t) {
                            re[t] = br[t * TS + bin];
                            im[t] = bi[t * TS + bin];
                        }
                        if constexpr (T > 1) cdft_n<T>(re, im, false);
                        const float hr = cr[bin], hi = ci[bin];
#pragma unroll
                        for (int kt = 0; kt < T; ++kt) {
                            const int i = kt * BX + bin;
                            const float cs = s_tw[2 * kt], sn = s_tw[2 * kt + 1];
                            const float Gr = hr * cs - hi * sn;
                            const float Gi = hr * sn + hi * cs;
                            const float2 w2 = reinterpret_cast<const float2*>(s_wf)[i];
                            const float wr = w2.x, wi = w2.y;
                            const float dr = re[kt] - g * wr, di = im[kt] - g * wi;
                            float m, dpsd, dsig;
                            gain_grad<FT>(dr * dr + di * di, s_sig[i], a, m, dpsd, dsig);
                            const float q = Gr * dr + Gi * di;
                            const float ddr = m * Gr + 2.0f * dpsd * q * dr;
                            const float ddi = m * Gi + 2.0f * dpsd * q * di;
                            if (a.gsigma && dsig != 0.0f) atomicAdd(&s_gs[i], dsig * q);
                            dg += (Gr * wr + Gi * wi) - (ddr * wr + ddi * wi);
                            re[kt] = ddr;
                            im[kt] = ddi;
                        }
                        if constexpr (T > 1) cdft_n<T>(re, im, true);
#pragma unroll
                        for (int t = 0; t < T; ++t) {
                            br[t * TS + bin] = re[t];
                            bi[t * TS + bin] = im[t];
                        }
                    }
                }
            };
            switch (a.filter_type) {
            case 0: bins(IntC<0>{}); break;
            case 1: bins(IntC<1>{}); break;
            case 2: bins(IntC<2>{}); break;
            case 3: bins(IntC<3>{}); break;
            case 4: bins(IntC<4>{}); break;
            case 5: bins(IntC<5>{}); break;
            default: bins(IntC<6>{}); break;
            }
            constexpr int RW = GT < 32 ? GT : 32;
#pragma unroll
            for (int o = RW / 2; o > 0; o >>= 1) dg += __shfl_xor_sync(0xffffffffu, dg, o);
            if ((tid & (RW - 1)) == 0) atomicAdd(&s_dg[gblk], dg);
        }
        __syncthreads();

        // ---- adjoint of the forward transform: inverse over y, halved c2r over x (the inverse
        //      over t ran with the gain).  The zero-mean term dg / Re WF(0) of bin (0, 0, 0) is, after
        //      the inverse DFT_t, the same constant on bin (ky 0, kx 0) of every frame.
        for (int task = tid; task < NBLK * T * X; task += L::NTH) {
            const int blk = task / (T * X), rem = task - blk * (T * X);
            const int t = rem / X, kx = rem - t * X;
            float* pr = zr + blk * ZB + t * TS + kx;
            float* pi = zi + blk * ZB + t * TS + kx;
            float re[B], im[B];
#pragma unroll
            for (int y = 0; y < B; ++y) {
                re[y] = pr[y * X];
                im[y] = pi[y * X];
            }
            if (a.zero_mean && kx == 0) re[0] += s_dg[blk] / wf0;
            cdft_n<B>(re, im, true);
#pragma unroll
            for (int y = 0; y < B; ++y) {
                pr[y * X] = re[y];
                pi[y * X] = im[y];
            }
        }
        __syncthreads();
        for (int task = tid; task < NBLK * T * B; task += L::NTH) {
            const int blk = task / (T * B), rem = task - blk * (T * B);
            const int t = rem / B, y = rem - t * B;
            const float* pr = zr + blk * ZB + t * TS + y * X;
            const float* pi = zi + blk * ZB + t * TS + y * X;
            float v[B], o[B];
            v[0] = pr[0];
            v[1] = pr[B / 2];
#pragma unroll
            for (int k = 1; k < B / 2; ++k) {
                v[2 * k] = 0.5f * pr[k];
                v[2 * k + 1] = 0.5f * pi[k];
            }
            c2r_n<B>(v, o);
            float* dst = dxp + (t * PH + (blk / TBX) * S + y) * PP + (blk % TBX) * S;
#pragma unroll
            for (int x = 0; x < B; ++x) atomicAdd(dst + x, s_win[(t * B + y) * WP + x] * o[x]);
        }
        __syncthreads();

        // ---- transposed gather: the patch back through the mirror into the source gradients
        over_patch([&](int t, int r, int c, bool in, long long my, int mx) {
            const float v = dxp[(t * PH + r) * PP + c];
            if (in && v != 0.0f) atomicAdd(job.gsrc[t] + my * job.gsrc_stride + mx, v);
        });
    }

    // ---- sigma gradient: the CTA's partials -> global
    if (a.gsigma) {
        __syncthreads();
        for (int i = tid; i < SPEC; i += L::NTH)
            if (s_gs[i] != 0.0f) atomicAdd(&a.gsigma[i], s_gs[i]);
    }
}

}  // namespace dft2
