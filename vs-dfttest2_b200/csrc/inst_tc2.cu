// Tensor-core strip form (dfttest_tc2.cuh): the constant image of a filter
// and the kernel shapes (one translation unit).
#include <cmath>
#include <cstring>

#include "dfttest_host.h"
#include "dfttest_tc2.cuh"

namespace dft2h {

namespace {

constexpr double kPi = 3.14159265358979323846;

int align128(int v) { return (v + 127) & ~127; }

// 16-bit hi and lo parts of v at byte offsets hi_off and lo_off of the image
void put_split(std::vector<char>& img, size_t hi_off, size_t lo_off, double v, int fmt) {
    if (fmt == dft2::kTc2Fp16) {
        const __half h = __float2half_rn((float)v);
        const __half l = __float2half_rn((float)(v - (double)__half2float(h)));
        std::memcpy(&img[hi_off], &h, 2);
        std::memcpy(&img[lo_off], &l, 2);
    } else {
        const __nv_bfloat16 h = __float2bfloat16_rn((float)v);
        const __nv_bfloat16 l = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
        std::memcpy(&img[hi_off], &h, 2);
        std::memcpy(&img[lo_off], &l, 2);
    }
}

// byte offset of element (row r, k) of a K-major 16-bit operand with K = 16
// (8-row x 16-byte core matrices: K halves 128 bytes apart, row groups 256)
size_t kmaj16(int r, int k) { return (size_t)(r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2; }

}  // namespace

int tc2_build(const Tc2Input& in, std::vector<char>& img, Tc2Shape& shape, std::string& why) {
    const int T = in.T, S = in.S, r = in.radius;
    constexpr int B = 16, X = 9;
    if (T != 1 && T != 3) {
        why = "the strip form supports radius 0 and 1";
        return 1;
    }
    if (S != 1 && S != 2 && S != 4) {
        why = "the strip form supports block_step 1, 2 and 4";
        return 1;
    }
    // window = wt[t] wy[y] wx[x] (the front end's window is this product)
    const double* w = in.window;
    int t0 = 0, y0 = 0, x0 = 0;
    double wmax = 0.0;
    for (int t = 0; t < T; ++t)
        for (int y = 0; y < B; ++y)
            for (int x = 0; x < B; ++x)
                if (std::fabs(w[(t * B + y) * B + x]) > wmax) {
                    wmax = std::fabs(w[(t * B + y) * B + x]);
                    t0 = t;
                    y0 = y;
                    x0 = x;
                }
    if (wmax == 0.0) {
        why = "the window is zero";
        return 1;
    }
    const double c = w[(t0 * B + y0) * B + x0];
    double wt[3], wy[B], wx[B];
    for (int t = 0; t < T; ++t) wt[t] = w[(t * B + y0) * B + x0];
    for (int y = 0; y < B; ++y) wy[y] = w[(t0 * B + y) * B + x0] / c;
    for (int x = 0; x < B; ++x) wx[x] = w[(t0 * B + y0) * B + x] / c;
    for (int t = 0; t < T; ++t)
        for (int y = 0; y < B; ++y)
            for (int x = 0; x < B; ++x)
                if (std::fabs(wt[t] * wy[y] * wx[x] - w[(t * B + y) * B + x]) > 1e-6 * wmax) {
                    why = "the strip form needs a separable window";
                    return 1;
                }

    dft2::Tc2Head h{};
    h.S = S;
    h.nrot = B / S;
    h.nks = (B + 7 * S + 15) / 16;
    h.voff = (h.nks - 1) * (B / S);
    h.nvb = h.voff + 8;
    h.nbx = 16;
    const int fw = h.nbx * S + B - S;
    const int xread = 8 * S + 16 * h.nks;  // x rows the second tile's products read
    h.xg = ((fw > xread ? fw : xread) + 7) / 8;
    h.np = T;
    for (int t = 0; t < T; ++t) {
        const int tau = ((t - r) % T + T) % T;  // centre-first time of frame t
        h.q[0][t] = (float)wt[t];
        if (T == 3) {
            h.q[1][t] = (float)(wt[t] * std::cos(2.0 * kPi * tau / T));
            h.q[2][t] = (float)(-wt[t] * std::sin(2.0 * kPi * tau / T));
        }
    }
    // synthesis window = window slice syn = (wt[syn] wy[y]) * wx[x]
    double sy[B];
    for (int y = 0; y < B; ++y) sy[y] = wt[in.syn] * wy[y];
    for (int x = 0; x < B; ++x) h.sx[x] = (float)wx[x];

    const int wy_bytes = h.nrot * 1024;
    const int wx_part = h.nvb * 16 * 16 * 2;
    h.off_wy = dft2::kTc2HeadBytes;
    h.off_wx = align128(h.off_wy + wy_bytes);
    h.off_wi = align128(h.off_wx + 4 * wx_part);
    h.off_tab = align128(h.off_wi + h.nrot * 1024);
    h.total = align128(h.off_tab + T * 9 * 16 * 16);
    img.assign((size_t)h.total, 0);

    // Wy rotated by rot: K = ring row k (window row (k - rot S) mod 16), N = packed y-bin j
    for (int rot = 0; rot < h.nrot; ++rot) {
        const size_t base = (size_t)h.off_wy + rot * 1024;
        for (int k = 0; k < B; ++k) {
            const int y = ((k - rot * S) % B + B) % B;
            for (int ky = 0; ky <= 8; ++ky) {
                const double th = 2.0 * kPi * (double)(ky * y % B) / B;
                const int jr = dft2::tc2_jre(ky);
                put_split(img, base + kmaj16(jr, k), base + 512 + kmaj16(jr, k), wy[y] * std::cos(th), in.fmt);
                if (ky >= 1 && ky <= 7) {
                    const int ji = dft2::tc2_jim(ky);
                    put_split(img, base + kmaj16(ji, k), base + 512 + kmaj16(ji, k), -wy[y] * std::sin(th), in.fmt);
                }
            }
        }
    }
    // tall x constants: row (virtual block vb, kx), K = 16 footprint columns of K step 0
    for (int cs = 0; cs < 2; ++cs) {
        const size_t hi = (size_t)h.off_wx + (2 * cs) * wx_part, lo = hi + wx_part;
        for (int row = 0; row < h.nvb * 16; ++row) {
            const int vb = row >> 4, kx = row & 15;
            for (int k = 0; k < 16; ++k) {
                const int xr = k - S * (vb - h.voff);
                if (xr < 0 || xr >= B) continue;
                const double th = 2.0 * kPi * (double)(kx * xr % B) / B;
                const double v = wx[xr] * (cs == 0 ? std::cos(th) : std::sin(th));
                put_split(img, hi + kmaj16(row, k), lo + kmaj16(row, k), v, in.fmt);
            }
        }
    }
    // inverse y (c2r over the packed bins j), y synthesis window: N = accumulator column c (output
    // row y = (c - rot S) mod 16 of the block), K = j; one copy per rotation
    for (int rot = 0; rot < h.nrot; ++rot) {
        const size_t base = (size_t)h.off_wi + rot * 1024;
        for (int c = 0; c < B; ++c) {
            const int y = ((c - rot * S) % B + B) % B;
            for (int ky = 0; ky <= 8; ++ky) {
                const double cw = (ky == 0 || ky == 8) ? 1.0 : 2.0;
                const double th = 2.0 * kPi * (double)(ky * y % B) / B;
                const int jr = dft2::tc2_jre(ky);
                put_split(img, base + kmaj16(c, jr), base + 512 + kmaj16(c, jr), cw * std::cos(th) * sy[y], in.fmt);
                if (ky >= 1 && ky <= 7) {
                    const int ji = dft2::tc2_jim(ky);
                    put_split(img, base + kmaj16(c, ji), base + 512 + kmaj16(c, ji), -cw * std::sin(th) * sy[y],
                              in.fmt);
                }
            }
        }
    }
    // gain table [kt][ky 0..8][kx 0..15]: (sigma, window spectrum re, im) of the bin; a bin with
    // kx > 8 is the conjugate of the reference's bin (-kt, -ky, 16 - kx); the window spectrum is
    // rotated to the centre-first time origin, W'(kt) = W(kt) e^(2 pi i kt r / T)
    {
        float* tab = reinterpret_cast<float*>(&img[h.off_tab]);
        for (int kt = 0; kt < T; ++kt)
            for (int ky = 0; ky <= 8; ++ky)
                for (int kx = 0; kx < 16; ++kx) {
                    int tt = kt, yy = ky, xx = kx;
                    double conj = 1.0;
                    if (kx > 8) {
                        tt = (T - kt) % T;
                        yy = (B - ky) % B;
                        xx = B - kx;
                        conj = -1.0;
                    }
                    const int bin = (tt * B + yy) * X + xx;
                    float* e = tab + 4 * ((kt * 9 + ky) * 16 + kx);
                    e[0] = in.sigma[bin];
                    e[1] = e[2] = e[3] = 0.0f;
                    if (in.wfreq) {
                        const double re = in.wfreq[2 * bin], im = in.wfreq[2 * bin + 1];
                        const double ang = 2.0 * kPi * (double)((tt * r) % T) / T;
                        e[1] = (float)(re * std::cos(ang) - im * std::sin(ang));
                        e[2] = (float)(conj * (re * std::sin(ang) + im * std::cos(ang)));
                    }
                }
    }
    for (int kt = 0; kt < T; ++kt)
        for (int i = 0; i < 9 * 16; ++i) {
            const float* e = reinterpret_cast<const float*>(&img[h.off_tab]) + 4 * (kt * 9 * 16 + i);
            if (e[1] != 0.0f || e[2] != 0.0f) h.wmask |= 1 << kt;
        }
    // sum over the temporal bins of the window spectrum of each (ky, kx): re in the w slot of bin 0,
    // im in the w slot of bin 1 (the gain adds g times it back once)
    if (T == 3) {
        float* tab = reinterpret_cast<float*>(&img[h.off_tab]);
        for (int i = 0; i < 9 * 16; ++i) {
            double sre = 0.0, sim = 0.0;
            for (int kt = 0; kt < T; ++kt) {
                sre += tab[4 * (kt * 9 * 16 + i) + 1];
                sim += tab[4 * (kt * 9 * 16 + i) + 2];
            }
            tab[4 * i + 3] = (float)sre;
            tab[4 * (9 * 16 + i) + 3] = (float)sim;
        }
    }
    std::memcpy(&img[0], &h, sizeof(h));
    shape.nbx = h.nbx;
    shape.xg = h.xg;
    shape.smem = (size_t)dft2::Tc2Smem::make(h.total - h.off_wy, T, h.xg).total;
    return 0;
}

namespace {
template <int T, int FMT, int S>
Variant make_tc2() {
    Variant v;
    v.main = dft2::dfttest_tc2_kernel<T, dft2::kFilterWiener, FMT, S>;
    v.generic = dft2::dfttest_tc2_kernel<T, dft2::kFilterGeneric, FMT, S>;
    v.fixup = dft2::dfttest_fixup_kernel<16>;
    v.nw = 8;
    v.bpw = 2;
    v.minb = 2;
    return v;
}
template <int T, int FMT>
Variant make_tc2_s(int S) {
    switch (S) {
    case 1: return make_tc2<T, FMT, 1>();
    case 2: return make_tc2<T, FMT, 2>();
    case 4: return make_tc2<T, FMT, 4>();
    }
    return Variant{};
}
}  // namespace

Variant tc2_variant(int T, int fmt, int S) {
    if (T == 1) return fmt == dft2::kTc2Fp16 ? make_tc2_s<1, dft2::kTc2Fp16>(S) : make_tc2_s<1, dft2::kTc2Bf16>(S);
    if (T == 3) return fmt == dft2::kTc2Fp16 ? make_tc2_s<3, dft2::kTc2Fp16>(S) : make_tc2_s<3, dft2::kTc2Bf16>(S);
    return Variant{};
}

}  // namespace dft2h
