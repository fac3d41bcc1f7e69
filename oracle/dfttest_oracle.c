/*
 * TEST INFRASTRUCTURE ONLY -- the checker, never part of the product path.
 *
 * FP64 restatement of DFTTest's per-plane pipeline (the vs-dfttest2
 * reference computes it in FP32):
 *
 *   geometry          cpu_source/getframe_impl.cpp:11-20
 *   mirror padding    cpu_source/getframe_impl.cpp:22-65
 *   gather + window   cpu_source/getframe_impl.cpp:105-156
 *   3D real DFT       cpu_source/kernel.hpp:1899-1936 (x real, then y, then t)
 *   zero mean         cpu_source/kernel.hpp:1819-1824, 1892-1897, 1943-1952
 *   gain              cpu_source/kernel.hpp:1826-1890
 *   inverse, slice r  cpu_source/kernel.hpp:1954-1983
 *   overlap-add       cpu_source/getframe_impl.cpp:158-175
 *   output            cpu_source/getframe_impl.cpp:177-221 (before rounding)
 *
 * Transforms are direct (O(n^2)) sums with FP64 twiddles; any block size and
 * odd temporal size are accepted (the cuFFT backend's general-B semantics,
 * cuda_source/kernels.cu:84-246).  Tables arrive in FP64 and are rounded to
 * FP32 first, as the plugin stores them, so that the oracle evaluates the
 * same function the GPU evaluates, in exact arithmetic up to FP64 rounding.
 *
 * The output is the un-rounded value acc / scale per pixel (double); callers
 * round / clamp for integer formats.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int pad_size(int n, int B, int S) {
    int m = B - S > S ? B - S : S;
    return n + ((n % B) ? B - n % B : 0) + 2 * m;
}
static int pad_num(int n, int B, int S) { return (pad_size(n, B, S) - B) / S + 1; }

static int mirror(int i, int n) {
    if (i < 0) i = -i;
    if (i >= n) i = 2 * (n - 1) - i;
    return i;
}

static double sample_at(const void* base, long long idx, int kind) {
    if (kind == 0) return (double)((const uint8_t*)base)[idx];
    if (kind == 1) return (double)((const uint16_t*)base)[idx];
    return (double)((const float*)base)[idx];
}

static double gain(int ft, double psd, double s, double sigma2, double pmin, double pmax) {
    double m;
    switch (ft) {
    case 0: m = (psd - s) / (psd + 1e-15); return m > 0 ? m : 0;
    case 1: return psd < s ? 0.0 : 1.0;
    case 2: return s;
    case 3: return (psd >= pmin && psd <= pmax) ? s : sigma2;
    case 4: return s * sqrt(psd * (pmax / ((psd + pmin) * (psd + pmax) + 1e-15)));
    case 5: m = (psd - s) / (psd + 1e-15); return pow(m > 0 ? m : 0, pmin);
    default: m = (psd - s) / (psd + 1e-15); return sqrt(m > 0 ? m : 0);
    }
}

/*
 * src: 2r+1 planes (time clamp done by the caller); kind 0 = u8, 1 = u16,
 * 2 = f32; scale as the plugin: 2^-(bits-8) or 255.  window (T*B*B),
 * sigma (T*B*X, X = B/2+1), window_freq (T*B*X*2, may be NULL when
 * zero_mean == 0).  syn_slice selects the synthesis window slice.
 * out: height x width doubles.  Returns 0 on success.
 */
int oracle_dfttest_plane(const void* const* src, int width, int height, long long src_stride, int kind, double scale,
                         double* out, const double* window, const double* sigma, double sigma2, double pmin,
                         double pmax, int filter_type, int zero_mean, const double* window_freq, int radius, int B,
                         int S, int syn_slice) {
    const int T = 2 * radius + 1, X = B / 2 + 1;
    const int pw = pad_size(width, B, S), ph = pad_size(height, B, S);
    const int pnx = pad_num(width, B, S), pny = pad_num(height, B, S);
    const int ox = (pw - width) / 2, oy = (ph - height) / 2;
    const double pi = 3.14159265358979323846;
    const float sigma2f = (float)sigma2, pminf = (float)pmin, pmaxf = (float)pmax;

    double* w = malloc(sizeof(double) * T * B * B);
    double* sg = malloc(sizeof(double) * T * B * X);
    double* wf = malloc(sizeof(double) * T * B * X * 2);
    double *cx = malloc(sizeof(double) * B * B), *sx = malloc(sizeof(double) * B * B);
    double *ct = malloc(sizeof(double) * T * T), *st = malloc(sizeof(double) * T * T);
    double* acc = calloc((size_t)pw * ph, sizeof(double));
    double* blk = malloc(sizeof(double) * T * B * B);
    /* spectra: [t][y][kx] complex */
    double *fr = malloc(sizeof(double) * T * B * X), *fi = malloc(sizeof(double) * T * B * X);
    double *gr = malloc(sizeof(double) * T * B * X), *gi = malloc(sizeof(double) * T * B * X);
    double *vr = malloc(sizeof(double) * B * X), *vi = malloc(sizeof(double) * B * X);
    double *ur = malloc(sizeof(double) * B * X), *ui = malloc(sizeof(double) * B * X);
    if (!w || !sg || !wf || !cx || !sx || !ct || !st || !acc || !blk || !fr || !fi || !gr || !gi || !vr || !vi ||
        !ur || !ui)
        return -1;

    for (int i = 0; i < T * B * B; ++i) w[i] = (double)(float)window[i];
    for (int i = 0; i < T * B * X; ++i) sg[i] = (double)(float)sigma[i];
    for (int i = 0; i < T * B * X * 2; ++i) wf[i] = zero_mean ? (double)(float)window_freq[i] : 0.0;
    for (int k = 0; k < B; ++k)
        for (int n = 0; n < B; ++n) {
            cx[k * B + n] = cos(2 * pi * ((long long)k * n % B) / B);
            sx[k * B + n] = sin(2 * pi * ((long long)k * n % B) / B);
        }
    for (int k = 0; k < T; ++k)
        for (int n = 0; n < T; ++n) {
            ct[k * T + n] = cos(2 * pi * ((k * n) % T) / T);
            st[k * T + n] = sin(2 * pi * ((k * n) % T) / T);
        }
    const double sc = (double)(float)scale;
    const double* wsyn = w + (size_t)syn_slice * B * B;

    for (int by = 0; by < pny; ++by) {
        for (int bx = 0; bx < pnx; ++bx) {
            /* gather */
            for (int t = 0; t < T; ++t)
                for (int y = 0; y < B; ++y) {
                    const int syy = mirror(by * S + y - oy, height);
                    for (int x = 0; x < B; ++x) {
                        const int sxx = mirror(bx * S + x - ox, width);
                        blk[(t * B + y) * B + x] =
                            sc * w[(t * B + y) * B + x] * sample_at(src[t], (long long)syy * src_stride + sxx, kind);
                    }
                }
            /* x: real DFT, bins 0..B/2 (sign -1) */
            for (int t = 0; t < T; ++t)
                for (int y = 0; y < B; ++y)
                    for (int k = 0; k < X; ++k) {
                        double re = 0, im = 0;
                        const double* row = blk + (t * B + y) * B;
                        for (int n = 0; n < B; ++n) {
                            re += row[n] * cx[k * B + n];
                            im -= row[n] * sx[k * B + n];
                        }
                        fr[(t * B + y) * X + k] = re;
                        fi[(t * B + y) * X + k] = im;
                    }
            /* y */
            for (int t = 0; t < T; ++t)
                for (int k = 0; k < B; ++k)
                    for (int kx = 0; kx < X; ++kx) {
                        double re = 0, im = 0;
                        for (int n = 0; n < B; ++n) {
                            const double a = fr[(t * B + n) * X + kx], b = fi[(t * B + n) * X + kx];
                            const double c = cx[k * B + n], s = sx[k * B + n];
                            re += a * c + b * s;
                            im += b * c - a * s;
                        }
                        gr[(t * B + k) * X + kx] = re;
                        gi[(t * B + k) * X + kx] = im;
                    }
            /* t */
            for (int k = 0; k < T; ++k)
                for (int i = 0; i < B * X; ++i) {
                    double re = 0, im = 0;
                    for (int n = 0; n < T; ++n) {
                        const double a = gr[n * B * X + i], b = gi[n * B * X + i];
                        const double c = ct[k * T + n], s = st[k * T + n];
                        re += a * c + b * s;
                        im += b * c - a * s;
                    }
                    fr[k * B * X + i] = re;
                    fi[k * B * X + i] = im;
                }
            /* zero mean + gain */
            const double g = zero_mean ? fr[0] / wf[0] : 0.0;
            for (int i = 0; i < T * B * X; ++i) {
                const double dre = fr[i] - g * wf[2 * i], dim = fi[i] - g * wf[2 * i + 1];
                const double m = gain(filter_type, dre * dre + dim * dim, sg[i], sigma2f, pminf, pmaxf);
                fr[i] = m * dre + g * wf[2 * i];
                fi[i] = m * dim + g * wf[2 * i + 1];
            }
            /* inverse t at the centre frame r (sign +1) */
            for (int i = 0; i < B * X; ++i) {
                double re = 0, im = 0;
                for (int k = 0; k < T; ++k) {
                    const double a = fr[k * B * X + i], b = fi[k * B * X + i];
                    const double c = ct[k * T + radius], s = st[k * T + radius];
                    re += a * c - b * s;
                    im += a * s + b * c;
                }
                vr[i] = re;
                vi[i] = im;
            }
            /* inverse y */
            for (int y = 0; y < B; ++y)
                for (int kx = 0; kx < X; ++kx) {
                    double re = 0, im = 0;
                    for (int k = 0; k < B; ++k) {
                        const double a = vr[k * X + kx], b = vi[k * X + kx];
                        const double c = cx[k * B + y], s = sx[k * B + y];
                        re += a * c - b * s;
                        im += a * s + b * c;
                    }
                    ur[y * X + kx] = re;
                    ui[y * X + kx] = im;
                }
            /* c2r x: imaginary parts of bins 0 and B/2 ignored */
            for (int y = 0; y < B; ++y)
                for (int x = 0; x < B; ++x) {
                    double v = ur[y * X] + ((x & 1) ? -ur[y * X + B / 2] : ur[y * X + B / 2]);
                    for (int k = 1; k < B / 2; ++k) {
                        const double a = ur[y * X + k], b = ui[y * X + k];
                        v += 2.0 * (a * cx[k * B + x] - b * sx[k * B + x]);
                    }
                    acc[(size_t)(by * S + y) * pw + bx * S + x] += v * wsyn[y * B + x];
                }
        }
    }
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) out[(size_t)y * width + x] = acc[(size_t)(oy + y) * pw + ox + x] / sc;

    free(w); free(sg); free(wf); free(cx); free(sx); free(ct); free(st); free(acc); free(blk);
    free(fr); free(fi); free(gr); free(gi); free(vr); free(vi); free(ur); free(ui);
    return 0;
}
