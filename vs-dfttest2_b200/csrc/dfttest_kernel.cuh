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

// polls of a bounded device wait before it gives up and reports an error
constexpr int kDefaultWaitLimit = 1 << 22;

// Checked build (-DDFT_CHECKS): the unit and fix-up kernels test their
// shared-memory ring, staging and block-buffer indices and their global
// band-record, source and output indices against the buffers before each
// access; an index outside its buffer skips the access and records error
// code 3 (nothing traps).  The normal build compiles the tests away.
#ifdef DFT_CHECKS
__device__ __forceinline__ bool in_range(long long i, long long n, int* flag) {
    if (i >= 0 && i < n) return true;
    atomicExch(flag, 3);
    return false;
}
#define DFT_IN_RANGE(i, n, flag) ::dft2::in_range((long long)(i), (long long)(n), (flag))
#else
#define DFT_IN_RANGE(i, n, flag) true
#endif

// ---- PTX wrappers: shared-memory mbarriers and TMA tile loads ---------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
}

// bounded wait for the completion of the phase with the given parity; false
// when `limit` polls ran out first
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = kDefaultWaitLimit) {
    const uint32_t a = smem_addr(bar);
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// arrive on the barrier, announcing `bytes` of asynchronous copies that will complete its phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// TMA load of one box of a 2D tensor map (in global memory, 64-byte aligned)
// at element coordinates (x, y) into shared memory, completing on `bar`.  No
// cluster multicast: the map covers this GPU's own memory.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        :: "r"(smem_addr(dst)), "l"(tmap), "r"(x), "r"(y), "r"(smem_addr(bar)) : "memory");
}

// generic-proxy accesses of this thread to shared memory are ordered before
// its later asynchronous-proxy (TMA) accesses
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

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
    int param;            // index into KernelArgs::params (batched launches)
    int seam_base;        // first seam counter of this job (KernelArgs::seam_count)
    int tmap[7];          // tensor map of src[t] in KernelArgs::tmaps; -1: rows staged by plain loads
};

// sample format and filter of a plane: launch-wide, or per job in a batch
struct FilterParams {
    int kind;          // SampleKind
    float scale;       // 2^-(bits-8) for integers, 255 for float
    float peak;        // 2^bits - 1
    int filter_type;   // 0..6
    float sigma2, pmin, pmax;
    float g_div;       // Re(window_freq[0,0,0]); 0 disables zero-mean
    int wmask;         // bit p set when temporal plane p of the window spectrum is not identically zero
    int pad_;
    const float* win;  // [T][B][B] analysis window
    const float* wsyn; // [B][B] synthesis window
    const float* sig;  // [T][B/2+2][B] sigma per gain slot and column lane
    const float* sig2; // [T][B/2+2][B] partner sigma (packed lanes, asymmetric sigma), may be null
    const float* wfe;  // [T][B/2+2][B][2] window spectrum per gain slot (zero-mean)
};

struct KernelArgs {
    const PlaneJob* jobs;
    int njobs;
    int nunits;
    int nfix;
    int block_step;    // S
    FilterParams p;    // every job's format and filter, unless params is set
    const FilterParams* params;  // per-job formats and filters (PlaneJob::param), may be null
    float* scratch;    // per-unit band records
    int rec_stride;    // floats per unit record
    int ring_pitch;    // floats per ring row
    int* error_flag;   // set to a non-zero code on an internal consistency failure
    // Launches whose units are full-height strips (nsy = 1 for every job): one
    // arrival counter per seam between neighbouring strips, zeroed before the
    // launch; the second strip to finish sums the seam, and no fix-up kernel
    // runs.  Null: the fix-up kernel sums the shared pixels.
    int* seam_count;
    // TMA staging of input rows: 2D tensor maps (CUtensorMap, 128 bytes each,
    // one row high and stage_bw samples wide) of the jobs' source planes, and
    // the byte offset of the two staging slots in dynamic shared memory.
    // Null: every job is staged by plain loads.
    const void* tmaps;
    int stage_bw;
    int stage_off;
    // Persistent grid: after its first unit (blockIdx.x) a CTA takes unit
    // gridDim.x + atomicAdd(unit_counter, 1) until none is left; the counter
    // is zeroed before the launch.  Null: one unit per CTA.
    int* unit_counter;
    // constant image of the tensor-core strip form (dfttest_tc2.cuh) and the poll limit of its
    // waits for the tensor cores; unused by the FP32 kernels
    const char* tc_consts;
    int wait_limit;
};

constexpr int kTmapBytes = 128;

// bytes of one staged row (a TMA destination starts on a 128-byte boundary)
__host__ __device__ inline int stage_row_bytes(int bw, int esz) { return (bw * esz + 127) & ~127; }
// both staging slots: T planes x S rows each
__host__ __device__ inline int stage_bytes(int bw, int esz, int T, int S) { return 2 * T * S * stage_row_bytes(bw, esz); }

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

// A unit less than 2 O wide or tall (strips narrower than O = B-S, which high
// overlap forces: 32x32 blocks at sosize 26..31) shares every footprint pixel
// with a neighbour; its record then holds the whole footprint.
__host__ __device__ inline bool band_full(int fw, int fh, int O) { return fw < 2 * O || fh < 2 * O; }

// offset of footprint pixel (lx, ly) inside the unit's band record; the band
// is every footprint pixel within O = B-S of the footprint edge.
__host__ __device__ inline int band_index(int lx, int ly, int fw, int fh, int O) {
    if (band_full(fw, fh, O)) return ly * fw + lx;
    if (ly < O) return ly * fw + lx;
    if (ly >= fh - O) return (O + ly - (fh - O)) * fw + lx;
    const int r = ly - O;
    const int base = 2 * O * fw;
    if (lx < O) return base + r * O + lx;
    return base + (fh - 2 * O) * O + r * O + (lx - (fw - O));
}

__host__ __device__ inline int band_record_size(int fw, int fh, int O) {
    return band_full(fw, fh, O) ? fw * fh : 2 * O * fw + 2 * (fh - 2 * O) * O;
}

__device__ __forceinline__ int mirror(int i, int n) {
    // reflection without edge repeat (cpu_source/getframe_impl.cpp:44-62)
    i = i < 0 ? -i : i;
    return i >= n ? 2 * (n - 1) - i : i;
}

// raw sample bits (integer value or float bits); converting later keeps the
// load in flight instead of stalling on it
__device__ __forceinline__ unsigned load_raw(const void* base, long long idx, int kind) {
    if (kind == kU8) return __ldg(reinterpret_cast<const uint8_t*>(base) + idx);
    if (kind == kU16) return __ldg(reinterpret_cast<const uint16_t*>(base) + idx);
    return __float_as_uint(__ldg(reinterpret_cast<const float*>(base) + idx));
}

__device__ __forceinline__ float raw_to_float(unsigned v, int kind) {
    return kind == kF32 ? __uint_as_float(v) : (float)v;
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

// samples of a staged row (raw format) as FP32: four from element e0 (a
// multiple of 4), or one
__device__ __forceinline__ float4 stage_load4(const unsigned char* row, int e0, int kind) {
    if (kind == kF32) return *reinterpret_cast<const float4*>(row + 4 * e0);
    if (kind == kU16) {
        const uint2 v = *reinterpret_cast<const uint2*>(row + 2 * e0);
        return make_float4((float)(v.x & 0xFFFFu), (float)(v.x >> 16), (float)(v.y & 0xFFFFu), (float)(v.y >> 16));
    }
    const unsigned v = *reinterpret_cast<const unsigned*>(row + e0);
    return make_float4((float)(v & 0xFFu), (float)((v >> 8) & 0xFFu), (float)((v >> 16) & 0xFFu), (float)(v >> 24));
}
__device__ __forceinline__ float stage_load1(const unsigned char* row, int e, int kind) {
    if (kind == kF32) return reinterpret_cast<const float*>(row)[e];
    if (kind == kU16) return (float)reinterpret_cast<const uint16_t*>(row)[e];
    return (float)row[e];
}

// Four consecutive output samples (a segment of the overlap-add) with the
// conversion of store_sample; one vector store where the address is aligned
// to the four samples (rows of 8 B / 16 B multiples), else scalar stores.
__device__ __forceinline__ void store4(void* base, long long idx, float4 a, int kind, float peak, float inv_scale) {
    if (kind == kF32) {
        // float output: acc / 255 (inv_scale is 0 for float: IEEE division as store_sample)
        float4 v = make_float4(__fdiv_rn(a.x, 255.0f), __fdiv_rn(a.y, 255.0f), __fdiv_rn(a.z, 255.0f),
                               __fdiv_rn(a.w, 255.0f));
        float* p = reinterpret_cast<float*>(base) + idx;
        if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
            *reinterpret_cast<float4*>(p) = v;
        } else {
            p[0] = v.x;
            p[1] = v.y;
            p[2] = v.z;
            p[3] = v.w;
        }
        return;
    }
    const int pk = (int)peak;
    auto q = [&](float x) {
        int v = __float2int_rz(__fadd_rn(x * inv_scale, 0.5f));
        return v < 0 ? 0 : (v > pk ? pk : v);
    };
    const unsigned q0 = q(a.x), q1 = q(a.y), q2 = q(a.z), q3 = q(a.w);
    if (kind == kU16) {
        uint16_t* p = reinterpret_cast<uint16_t*>(base) + idx;
        if ((reinterpret_cast<uintptr_t>(p) & 7) == 0) {
            *reinterpret_cast<uint2*>(p) = make_uint2(q0 | (q1 << 16), q2 | (q3 << 16));
        } else {
            p[0] = (uint16_t)q0;
            p[1] = (uint16_t)q1;
            p[2] = (uint16_t)q2;
            p[3] = (uint16_t)q3;
        }
    } else {
        uint8_t* p = reinterpret_cast<uint8_t*>(base) + idx;
        if ((reinterpret_cast<uintptr_t>(p) & 3) == 0) {
            *reinterpret_cast<unsigned*>(p) = q0 | (q1 << 8) | (q2 << 16) | (q3 << 24);
        } else {
            p[0] = (uint8_t)q0;
            p[1] = (uint8_t)q1;
            p[2] = (uint8_t)q2;
            p[3] = (uint8_t)q3;
        }
    }
}

// reciprocal from the MUFU unit (PTX rcp.approx.ftz.f32, < 1 ulp)
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// multiplier of frequency_filtering (cpu_source/kernel.hpp:1826-1890).
// FT 0 is the Wiener gain max((psd - s) / (psd + 1e-15), 0), evaluated as
// max(1 - s * rcp(psd), 0): the 1e-15 only keeps the reference's division
// finite at psd = 0, where rcp gives +inf and the gain is 0 either way
// (fmaxf drops the NaN of 0 * inf); the other types keep IEEE division.
template <int FT>
__device__ __forceinline__ float gain(float psd, float s, const FilterParams& a) {
    if constexpr (FT == 0) {
        return fmaxf(fmaf(-s, rcp_approx(psd), 1.0f), 0.0f);
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

__device__ __forceinline__ float gain_rt(int ft, float psd, float s, const FilterParams& a) {
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
// ZM = false: the plane's window spectrum is zero, so the zero-mean terms vanish
template <int FC, bool ZM = true>
__device__ __forceinline__ void apply_bin(float& re, float& im, float s, float s2, bool dual, float2 w, float g,
                                          const FilterParams& a) {
    const float dre = ZM ? fmaf(-g, w.x, re) : re;
    const float dim = ZM ? fmaf(-g, w.y, im) : im;
    const float psd = fmaf(dim, dim, dre * dre);
    float m;
    if constexpr (FC == kFilterWiener) {
        m = gain<0>(psd, s, a);
    } else {
        m = gain_rt(a.filter_type, psd, s, a);
        if (dual) m = 0.5f * (m + gain_rt(a.filter_type, psd, s2, a));
    }
    if constexpr (ZM) {
        re = fmaf(m, dre, re - dre);
        im = fmaf(m, dim, im - dim);
    } else {
        re *= m;
        im *= m;
    }
}

template <int B> struct Tile {
    static constexpr int H = B / 2;          // packed x-bins per block
    static constexpr int M = B / 2;          // y-bins per column lane (lane pair splits by parity)
    static constexpr int BPW = 32 / B;       // blocks per warp (B lanes per block)
    static constexpr int WP = B + 4;         // padded window row pitch (floats)
    static constexpr int RPL = 32 / B;       // rows per 128-byte line in the warp buffer
    static constexpr int NCH = B / 4;        // 16-byte chunks per buffer row
    static constexpr int NSLOT = M + 2;      // gain slots per lane and plane
    __device__ static __forceinline__ int swz(int y) { return (y / RPL) & (NCH - 1); }
    // float offset of (y, x) inside one B x B plane of the warp buffer
    __device__ static __forceinline__ int off(int y, int x) { return y * B + ((((x >> 2) ^ swz(y)) << 2) | (x & 3)); }
};

// Large blocks (32x32 with 3, 5 or 7 frames) read the window,
// synthesis-window and gain tables from global memory (L1-cached) and run the
// row phase in two passes, which leaves shared memory and registers for wide
// enough strips and more warps; smaller blocks keep the tables in shared
// memory (faster for them: 16x16x5 with global tables ran 17 % slower).
template <int B, int T> struct Large {
    static constexpr bool value = B == 32 && T >= 3;
};

template <int B, int T, int NW>
struct Layout {
    static constexpr int M = B / 2;
    static constexpr int BPW = 32 / B;
    static constexpr int WP = B + 4;
    static constexpr int NSLOT = M + 2;
    static constexpr int TAB = Large<B, T>::value ? 0 : 1;  // tables held in shared memory
    // warp-buffer floats per block; the stride is 4 (mod 32) floats so that the
    // overlap-add, whose lanes read the same 16-byte chunk of consecutive
    // blocks, spreads over 8 bank groups
    static constexpr int BSTR = T * B * B + 4;
    // offsets in floats (ring sizes depend on the runtime pitch)
    static constexpr int o_win = 0;
    static constexpr int o_wsyn = o_win + TAB * T * B * WP;
    static constexpr int o_sig = o_wsyn + TAB * B * WP;
    static constexpr int o_sig2 = o_sig + TAB * T * NSLOT * B;
    static constexpr int o_wfe = o_sig2 + TAB * T * NSLOT * B;
    static constexpr int o_g = o_wfe + TAB * 2 * T * NSLOT * B;
    static constexpr int o_wbuf = o_g + ((NW * BPW + 3) & ~3);
    static constexpr int o_ring = o_wbuf + NW * BPW * BSTR;
    __host__ __device__ static int in_ring_floats(int pitch) { return T * B * pitch; }
    __host__ __device__ static int ola_floats(int pitch) { return B * pitch; }
    __host__ __device__ static size_t smem_bytes(int pitch) {
        return sizeof(float) * (size_t)(o_ring + in_ring_floats(pitch) + ola_floats(pitch));
    }
};

// a table element: shared memory, or global memory through the read-only path
template <bool G> __device__ __forceinline__ float ldt(const float* p) { return G ? __ldg(p) : *p; }
template <bool G> __device__ __forceinline__ float2 ldt2(const float* p) {
    return G ? __ldg(reinterpret_cast<const float2*>(p)) : *reinterpret_cast<const float2*>(p);
}
template <bool G> __device__ __forceinline__ float4 ldt4(const float* p) {
    return G ? __ldg(reinterpret_cast<const float4*>(p)) : *reinterpret_cast<const float4*>(p);
}

// i / n for small non-negative i, n through a float reciprocal (exact while
// i * n < 2^22, which the shared-memory extents guarantee)
__device__ __forceinline__ int div_small(int i, float inv_n) { return __float2int_rz(((float)i + 0.5f) * inv_n); }

// ---------------------------------------------------------------------------
// row phase: T rows of one block at one y -> packed spectra per temporal plane;
// returns this row's contribution to the block's 3D DC (zero-mean)
// ---------------------------------------------------------------------------
template <int B, int T>
__device__ __forceinline__ float row_task(float* __restrict__ wb, const float* __restrict__ ring, int pitch, int slot_y,
                                          int xoff, const float* __restrict__ win, float wscale, int y, bool vec,
                                          bool store) {
    using TL = Tile<B>;
    constexpr int H = B / 2;
    constexpr int R = (T - 1) / 2;
    constexpr bool G = Large<B, T>::value;
    constexpr int WPITCH = G ? B : TL::WP;
    // frames in centre-first order (t' = 0 is frame r): the temporal DFT of the
    // shifted sequence is w^(p r) times that of the original, which is the
    // centre-frame weight of the inverse, so the inverse becomes a plain sum.
    // Windowed row of frame t'; a global window table is scaled here, giving
    // the same product scale * window (rounded once) as the shared table.
    auto windowed_row = [&](int t, float (&v)[B]) {
        const int ft = (t + R) % T;
        const float* src = ring + (ft * B + slot_y) * pitch + xoff;
        const float* w = win + (ft * B + y) * WPITCH;
        if (vec) {
#pragma unroll
            for (int q = 0; q < B / 4; ++q) {
                const float4 s4 = *reinterpret_cast<const float4*>(src + 4 * q);
                float4 w4 = ldt4<G>(w + 4 * q);
                if (G) {
                    w4.x *= wscale;
                    w4.y *= wscale;
                    w4.z *= wscale;
                    w4.w *= wscale;
                }
                v[4 * q + 0] = s4.x * w4.x;
                v[4 * q + 1] = s4.y * w4.y;
                v[4 * q + 2] = s4.z * w4.z;
                v[4 * q + 3] = s4.w * w4.w;
            }
        } else {
#pragma unroll
            for (int x = 0; x < B; ++x) v[x] = src[x] * (G ? wscale * __ldg(w + x) : w[x]);
        }
    };
    auto r2c = [](float (&v)[B], float (&X)[B]) {
        if constexpr (B == 8) r2c_8(v, X);
        if constexpr (B == 16) r2c_16(v, X);
        if constexpr (B == 32) r2c_32(v, X);
    };
    if constexpr (G && T > 1) {
        // Two passes: every frame's row spectrum goes to its plane of the block
        // buffer (registers for T x B spectra would leave room for few warps),
        // then the temporal DFT runs in place, one 4-float chunk (two packed
        // x-bins) at a time. The lane owns row y of every plane of its block
        // buffer, so no barrier is needed; lanes of a block past the strip end
        // work on their own (unused) buffer.
#pragma unroll
        for (int t = 0; t < T; ++t) {
            float v[B], X[B];
            windowed_row(t, v);
            r2c(v, X);
            float* dst = wb + t * B * B;
#pragma unroll
            for (int q = 0; q < B / 4; ++q)
                *reinterpret_cast<float4*>(dst + TL::off(y, 4 * q)) =
                    make_float4(X[4 * q], X[4 * q + 1], X[4 * q + 2], X[4 * q + 3]);
        }
        auto cdft = [](float (&re)[T], float (&im)[T]) {
            if constexpr (T == 3) cdft_3_fwd(re, im);
            if constexpr (T == 5) cdft_5_fwd(re, im);
            if constexpr (T == 7) cdft_7_fwd(re, im);
        };
        float dc = 0.0f;
#pragma unroll
        for (int q = 0; q < B / 4; ++q) {
            float4 z[T];
#pragma unroll
            for (int t = 0; t < T; ++t) z[t] = *reinterpret_cast<const float4*>(wb + t * B * B + TL::off(y, 4 * q));
            float re[T], im[T];
            if (q == 0) {
                // x-bins 0 and B/2: two real sequences
                float xa[T], xb[T], a_re[R + 1], a_im[R + 1], b_re[R + 1], b_im[R + 1];
#pragma unroll
                for (int t = 0; t < T; ++t) {
                    xa[t] = z[t].x;
                    xb[t] = z[t].y;
                }
                if constexpr (T == 3) { rdftT_3(xa, a_re, a_im); rdftT_3(xb, b_re, b_im); }
                if constexpr (T == 5) { rdftT_5(xa, a_re, a_im); rdftT_5(xb, b_re, b_im); }
                if constexpr (T == 7) { rdftT_7(xa, a_re, a_im); rdftT_7(xb, b_re, b_im); }
                z[0].x = a_re[0];
                z[0].y = b_re[0];
#pragma unroll
                for (int p = 1; p <= R; ++p) {
                    z[p].x = a_re[p];
                    z[p].y = a_im[p];
                    z[T - p].x = b_re[p];
                    z[T - p].y = b_im[p];
                }
                dc = a_re[0];
            } else {
#pragma unroll
                for (int t = 0; t < T; ++t) {
                    re[t] = z[t].x;
                    im[t] = z[t].y;
                }
                cdft(re, im);
#pragma unroll
                for (int t = 0; t < T; ++t) {
                    z[t].x = re[t];
                    z[t].y = im[t];
                }
            }
#pragma unroll
            for (int t = 0; t < T; ++t) {
                re[t] = z[t].z;
                im[t] = z[t].w;
            }
            cdft(re, im);
#pragma unroll
            for (int t = 0; t < T; ++t) {
                z[t].z = re[t];
                z[t].w = im[t];
                *reinterpret_cast<float4*>(wb + t * B * B + TL::off(y, 4 * q)) = z[t];
            }
        }
        return dc;
    } else {
        float X[T][B];
#pragma unroll
        for (int t = 0; t < T; ++t) {
            float v[B];
            windowed_row(t, v);
            r2c(v, X[t]);
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
}

// sum over the B lanes of one block; lanes of a block are contiguous
template <int B> __device__ __forceinline__ float block_row_sum(float v) {
#pragma unroll
    for (int o = (B < 32 ? B : 32) / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// column phase
// ---------------------------------------------------------------------------
template <int M> __device__ __forceinline__ void half_dft_fwd(float (&re)[M], float (&im)[M]) {
    if constexpr (M == 4) cdft_4_fwd(re, im);
    if constexpr (M == 8) cdft_8_fwd(re, im);
    if constexpr (M == 16) cdft_16_fwd(re, im);
}
template <int M> __device__ __forceinline__ void half_dft_inv(float (&re)[M], float (&im)[M]) {
    if constexpr (M == 4) cdft_4_inv(re, im);
    if constexpr (M == 8) cdft_8_inv(re, im);
    if constexpr (M == 16) cdft_16_inv(re, im);
}

// gain of the M bins a lane holds; slot tables are [NSLOT][B] per plane
// the gain of the general filter class with the filter type fixed (type 0
// with IEEE division, as gain_rt), for the partner-sigma average of `dual`
template <int FT, bool ZM>
__device__ __forceinline__ void apply_bin_ft(float& re, float& im, float s, float s2, bool dual, float2 w, float g,
                                             const FilterParams& a) {
    const float dre = ZM ? fmaf(-g, w.x, re) : re;
    const float dim = ZM ? fmaf(-g, w.y, im) : im;
    const float psd = fmaf(dim, dim, dre * dre);
    auto gx = [&](float sg) {
        if constexpr (FT == 0) return fmaxf(__fdiv_rn(psd - sg, psd + 1e-15f), 0.0f);
        else return gain<FT>(psd, sg, a);
    };
    float m = gx(s);
    if (dual) m = 0.5f * (m + gx(s2));
    if constexpr (ZM) {
        re = fmaf(m, dre, re - dre);
        im = fmaf(m, dim, im - dim);
    } else {
        re *= m;
        im *= m;
    }
}

template <int M, int B, int FT, bool ZM, bool G>
__device__ __forceinline__ void gain_lane_ft(float (&re)[M], float (&im)[M], const float* __restrict__ sig,
                                             const float* __restrict__ sig2, const float* __restrict__ wfe, int w,
                                             float g, bool dual, const FilterParams& a) {
#pragma unroll
    for (int j = 0; j < M; ++j) {
        const float s = ldt<G>(sig + j * B + w);
        const float s2 = dual ? ldt<G>(sig2 + j * B + w) : s;
        const float2 wv = ZM ? ldt2<G>(wfe + 2 * (j * B + w)) : make_float2(0.0f, 0.0f);
        apply_bin_ft<FT, ZM>(re[j], im[j], s, s2, dual, wv, g, a);
    }
}

template <int M, int B, int FC, bool ZM, bool G>
__device__ __forceinline__ void gain_lane_zm(float (&re)[M], float (&im)[M], const float* __restrict__ sig,
                                             const float* __restrict__ sig2, const float* __restrict__ wfe, int w,
                                             float g, bool dual, const FilterParams& a) {
    if constexpr (FC == kFilterWiener) {
#pragma unroll
        for (int j = 0; j < M; ++j) {
            const float s = ldt<G>(sig + j * B + w);
            const float2 wv = ZM ? ldt2<G>(wfe + 2 * (j * B + w)) : make_float2(0.0f, 0.0f);
            apply_bin<FC, ZM>(re[j], im[j], s, s, false, wv, g, a);
        }
    } else {
        // the filter type is uniform: one switch around the bins keeps the
        // executed code a single straight run (a switch per bin interleaves
        // all seven gains in the instruction stream)
        switch (a.filter_type) {
        case 0: gain_lane_ft<M, B, 0, ZM, G>(re, im, sig, sig2, wfe, w, g, dual, a); break;
        case 1: gain_lane_ft<M, B, 1, ZM, G>(re, im, sig, sig2, wfe, w, g, dual, a); break;
        case 2: gain_lane_ft<M, B, 2, ZM, G>(re, im, sig, sig2, wfe, w, g, dual, a); break;
        case 3: gain_lane_ft<M, B, 3, ZM, G>(re, im, sig, sig2, wfe, w, g, dual, a); break;
        case 4: gain_lane_ft<M, B, 4, ZM, G>(re, im, sig, sig2, wfe, w, g, dual, a); break;
        case 5: gain_lane_ft<M, B, 5, ZM, G>(re, im, sig, sig2, wfe, w, g, dual, a); break;
        default: gain_lane_ft<M, B, 6, ZM, G>(re, im, sig, sig2, wfe, w, g, dual, a); break;
        }
    }
}

template <int M, int B, int FC, bool G>
__device__ __forceinline__ void gain_lane(float (&re)[M], float (&im)[M], const float* __restrict__ sig,
                                          const float* __restrict__ sig2, const float* __restrict__ wfe, int w, float g,
                                          bool dual, bool has_w, const FilterParams& a) {
    if (has_w)
        gain_lane_zm<M, B, FC, true, G>(re, im, sig, sig2, wfe, w, g, dual, a);
    else
        gain_lane_zm<M, B, FC, false, G>(re, im, sig, sig2, wfe, w, g, dual, a);
}

// x *= (c + i s) for a compile-time constant (after unrolling) twiddle
__device__ __forceinline__ void cmul_const(float& re, float& im, float c, float s) {
    if (s == 0.0f) {
        if (c != 1.0f) {
            re *= c;
            im *= c;
        }
    } else if (c == 0.0f) {
        const float t = re;
        re = -im * s;
        im = t * s;
    } else {
        const float r = fmaf(re, c, -im * s);
        im = fmaf(re, s, im * c);
        re = r;
    }
}

// In-lane partner pairs (k, -k mod B) of the y-bins k = 2m + h a lane holds:
// h = 0: (m, M-m) for 0 < m < M/2, with m = 0 and m = M/2 self-paired;
// h = 1: (m, M-1-m) for 0 <= m < M/2.
template <int M, typename F>
__device__ __forceinline__ void for_pairs(int h, F&& f) {
    if (h == 0) {
#pragma unroll
        for (int m = 1; m < M / 2; ++m) f(m, M - m);
    } else {
#pragma unroll
        for (int m = 0; m < M / 2; ++m) f(m, M - 1 - m);
    }
}

// One column task: lane w = 2c + h of a block (`wb` = the block's buffer).
//
// Packed x-column c (c = 0 carries x-bins 0 and B/2) is split over the lane
// pair h = 0, 1 by y-bin parity: lane h forms t[y] = (x[y] + (-1)^h x[y+M])
// * W_B^(h y), y < M, whose M-point DFT is bins k = 2m + h (one radix-2
// decimation-in-frequency step).  Every temporal plane is transformed,
// filtered, weighted by its centre-frame twiddle w^(p r) and summed into S;
// the packed lanes enter each plane through its Hermitian part (B-column
// planes multiplied by i) so that S = S_A + i S_B.  The inverse y-DFT runs
// per half (M points, post-twiddle W_B^(-h n)) and the halves are combined
// with one shuffle exchange: y[n] = f0 + f1, y[n+M] = f0 - f1.
template <int B, int T, int FC>
__device__ __forceinline__ void column_task(float* __restrict__ wb, float g, const float* __restrict__ sm_sig,
                                            const float* __restrict__ sm_sig2, const float* __restrict__ sm_wfe, int w,
                                            bool dual_tables, bool store, const FilterParams& a) {
    using TL = Tile<B>;
    constexpr int M = B / 2;
    constexpr int R = (T - 1) / 2;
    constexpr int NS = M + 2;
    constexpr bool G = Large<B, T>::value;  // tables in global memory
    const int c = w >> 1, h = w & 1;
    const bool packed = (c == 0);
    const bool dual = dual_tables && packed;
    const float hs = h ? -1.0f : 1.0f;

    float sr[M], si[M];
#pragma unroll
    for (int k = 0; k < M; ++k) sr[k] = si[k] = 0.0f;
    float qr[M], qi[M];

    auto load_half = [&](const float* plane) {
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const float2 x0 = *reinterpret_cast<const float2*>(plane + TL::off(m, 2 * c));
            const float2 x1 = *reinterpret_cast<const float2*>(plane + TL::off(m + M, 2 * c));
            qr[m] = fmaf(hs, x1.x, x0.x);
            qi[m] = fmaf(hs, x1.y, x0.y);
        }
        if (h) {
#pragma unroll
            for (int m = 0; m < M; ++m) cmul_const(qr[m], qi[m], HalfTwiddle<B>::re(m), HalfTwiddle<B>::im(m));
        }
        half_dft_fwd<M>(qr, qi);
    };

#pragma unroll
    for (int p = 1; p < T; ++p) {
        load_half(wb + p * B * B);
        gain_lane<M, B, FC, G>(qr, qi, sm_sig + p * NS * B, sm_sig2 + p * NS * B, sm_wfe + 2 * p * NS * B, w, g, dual,
                               (a.wmask >> p) & 1, a);
        // the centre-frame weight w^(p r) is already in the spectrum (centre-first
        // frame order); the packed lane enters a B-column plane multiplied by i
        if (packed && p > R) {
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const float vr = -qi[k];
                qi[k] = qr[k];
                qr[k] = vr;
            }
        }
        if (packed) {
            // Hermitian part (A planes) or anti-Hermitian part (i * B planes)
            const float sg = (p <= R) ? 1.0f : -1.0f;
            if (h == 0) {
                qr[0] += sg * qr[0];
                qi[0] -= sg * qi[0];
                qr[M / 2] += sg * qr[M / 2];
                qi[M / 2] -= sg * qi[M / 2];
            }
            for_pairs<M>(h, [&](int i, int j) {
                const float ar = qr[i], ai = qi[i], br = qr[j], bi = qi[j];
                qr[i] = fmaf(sg, br, ar);
                qi[i] = fmaf(-sg, bi, ai);
                qr[j] = fmaf(sg, ar, br);
                qi[j] = fmaf(-sg, ai, bi);
            });
        }
#pragma unroll
        for (int k = 0; k < M; ++k) {
            sr[k] += qr[k];
            si[k] += qi[k];
        }
    }

    // plane 0 last
    load_half(wb);
    float e1r = 0.0f, e1i = 0.0f, e2r = 0.0f, e2i = 0.0f;
    if (packed) {
        // untangle Q = A + iB (A, B Hermitian in y): A(k) -> reg of k, B(k) -> reg of -k
        for_pairs<M>(h, [&](int i, int j) {
            const float ar = qr[i], ai = qi[i], br = qr[j], bi = qi[j];
            qr[i] = 0.5f * (ar + br);
            qi[i] = 0.5f * (ai - bi);
            qr[j] = 0.5f * (ai + bi);
            qi[j] = 0.5f * (br - ar);
        });
        if (h == 0) {
            // bins 0 and B/2 are self-paired: A and B are the real and imaginary parts
            e1r = qi[0];
            e2r = qi[M / 2];
            qi[0] = 0.0f;
            qi[M / 2] = 0.0f;
        }
    }
    gain_lane<M, B, FC, G>(qr, qi, sm_sig, sm_sig2, sm_wfe, w, g, dual, a.wmask & 1, a);
    if (packed) {
        if (h == 0) {
            const float2 w1 = ldt2<G>(sm_wfe + 2 * (M * B + w));
            const float2 w2 = ldt2<G>(sm_wfe + 2 * ((M + 1) * B + w));
            apply_bin<FC>(e1r, e1i, ldt<G>(sm_sig + M * B + w), dual ? ldt<G>(sm_sig2 + M * B + w) : 0.0f, dual, w1,
                          g, a);
            apply_bin<FC>(e2r, e2i, ldt<G>(sm_sig + (M + 1) * B + w), dual ? ldt<G>(sm_sig2 + (M + 1) * B + w) : 0.0f,
                          dual, w2, g, a);
            sr[0] += qr[0];
            si[0] += e1r;
            sr[M / 2] += qr[M / 2];
            si[M / 2] += e2r;
        }
        // add Y_A0 + i Y_B0, both Hermitian in y
        for_pairs<M>(h, [&](int i, int j) {
            const float ar = qr[i], ai = qi[i], br = qr[j], bi = qi[j];
            sr[i] += ar - bi;
            si[i] += ai + br;
            sr[j] += ar + bi;
            si[j] += br - ai;
        });
    } else {
#pragma unroll
        for (int k = 0; k < M; ++k) {
            sr[k] += qr[k];
            si[k] += qi[k];
        }
    }
    // inverse y-DFT: M points per half, post-twiddle, combine the halves
    half_dft_inv<M>(sr, si);
    if (h) {
#pragma unroll
        for (int n = 0; n < M; ++n) cmul_const(sr[n], si[n], HalfTwiddle<B>::re(n), -HalfTwiddle<B>::im(n));
    }
#pragma unroll
    for (int n = 0; n < M; ++n) {
        const float orr = __shfl_xor_sync(0xffffffffu, sr[n], 1);
        const float oi = __shfl_xor_sync(0xffffffffu, si[n], 1);
        sr[n] = fmaf(hs, sr[n], orr);
        si[n] = fmaf(hs, si[n], oi);
    }
    if (store) {
#pragma unroll
        for (int n = 0; n < M; ++n)
            *reinterpret_cast<float2*>(wb + TL::off(n + h * M, 2 * c)) = make_float2(sr[n], si[n]);
    }
}

// inverse rows: packed row -> real, synthesis window, in place
template <int B, bool G>
__device__ __forceinline__ void inverse_row_task(float* __restrict__ wb, const float* __restrict__ wsyn, int y) {
    using TL = Tile<B>;
    constexpr int WPITCH = G ? B : TL::WP;
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
    const float* w = wsyn + y * WPITCH;
#pragma unroll
    for (int q = 0; q < B / 4; ++q) {
        const float4 w4 = ldt4<G>(w + 4 * q);
        *reinterpret_cast<float4*>(wb + TL::off(y, 4 * q)) =
            make_float4(o[4 * q] * w4.x, o[4 * q + 1] * w4.y, o[4 * q + 2] * w4.z, o[4 * q + 3] * w4.w);
    }
}

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Plain-load staging of input rows [r_lo, r_lo + nr) of every temporal frame
// of a unit into the FP32 input ring (mirror padding by index math).  Used for
// a unit's first B rows, and for every step of units whose planes the TMA
// copies cannot take; kept out of line so that the unit kernel's step loop
// stays compact.
struct StageGeom {
    const void* const* src;  // the job's 2r+1 source planes
    long long src_stride;
    int kind, rowlen, pitch, x0, ox, oy, W, H;
    int* err;                // error word (checked build)
};
template <int B, int T, int NT>
__device__ __noinline__ void stage_rows_plain(float* __restrict__ s_in, const StageGeom g, int r_lo, int nr, int tid) {
    const float inv_rl = 1.0f / (float)g.rowlen;
    const float inv_nr_rl = 1.0f / (float)(nr * g.rowlen);
    for (int i = tid; i < T * nr * g.rowlen; i += NT) {
        const int t = div_small(i, inv_nr_rl);
        const int rem = i - t * nr * g.rowlen;
        const int r = div_small(rem, inv_rl);
        const int lx = rem - r * g.rowlen;
        const int py = r_lo + r;
        const int sy = mirror(py - g.oy, g.H), sx = mirror(g.x0 + lx - g.ox, g.W);
        const long long gidx = (long long)sy * g.src_stride + sx;
        const int si = (t * B + (py & (B - 1))) * g.pitch + lx;
        if (DFT_IN_RANGE(sy, g.H, g.err) && DFT_IN_RANGE(sx, g.W, g.err) && DFT_IN_RANGE(lx, g.pitch, g.err) &&
            DFT_IN_RANGE(si, T * B * g.pitch, g.err))
            s_in[si] = load_sample(g.src[t], gidx, g.kind);
    }
}

// Where a final overlap-add pixel goes: the output plane (pixels of the
// unit's exclusive zone), or the unit's band record (pixels it shares).
struct FinishGeom {
    void* dst;
    long long dst_stride;
    int kind;
    float scale, peak, inv_scale;  // inv_scale 0: float output (IEEE division by scale)
    int x0, ox, oy, W, H;
    int excl_x0, excl_x1, excl_y0, excl_y1;
    float* rec;
    int fw, fh, ry0, O, rec_stride;
    int* err;
};

__device__ __forceinline__ void finish_px(const FinishGeom& g, int py, int lx, float v) {
    const int px = g.x0 + lx;
    if (px < g.ox || px >= g.ox + g.W || py < g.oy || py >= g.oy + g.H) return;
    if (px >= g.excl_x0 && px < g.excl_x1 && py >= g.excl_y0 && py < g.excl_y1) {
        store_sample(g.dst, (long long)(py - g.oy) * g.dst_stride + (px - g.ox), v, g.kind, g.scale, g.peak,
                     g.inv_scale);
    } else {
        const int bi = band_index(lx, py - g.ry0, g.fw, g.fh, g.O);
        if (DFT_IN_RANGE(bi, g.rec_stride, g.err)) g.rec[bi] = v;
    }
}

// Overlap-add of one step for block steps that are not multiples of 4
// (pixel items, any number of covering blocks); out of line, so that the
// unit kernel's step loop carries only the 4-pixel segment path.
template <int B, int T, int NW>
__device__ __noinline__ void ola_scalar(const FinishGeom g, float* __restrict__ s_ola,
                                        const float* __restrict__ s_wbuf, int pitch, int rowlen, int by, int S, int nbx,
                                        int nfin, int tid) {
    using L = Layout<B, T, NW>;
    using TL = Tile<B>;
    constexpr int NT = NW * 32;
    const float inv_rl = 1.0f / (float)rowlen, inv_S = 1.0f / (float)S;
    for (int i = tid; i < B * rowlen; i += NT) {
        const int r = div_small(i, inv_rl), px = i - r * rowlen;
        // blocks k with k*S <= px <= k*S + B - 1
        const int b_lo = px <= B - 1 ? 0 : div_small(px - B + S, inv_S);
        const int b_hi = min(div_small(px, inv_S), nbx - 1);
        const int py = by * S + r;
        float* cell = s_ola + (py & (B - 1)) * pitch + px;
        float acc = *cell;
        for (int k = b_lo; k <= b_hi; ++k) acc += s_wbuf[k * L::BSTR + TL::off(r, px - k * S)];
        if (r < nfin) {
            finish_px(g, py, px, acc);
            acc = 0.0f;
        }
        *cell = acc;
    }
}

// Seams shared by neighbouring full-height strips (launches with
// KernelArgs::seam_count): the second of the two strips to finish sums both
// band records (left strip first, as the fix-up kernel does) and stores the
// result.  Nothing waits, so this is safe for any launch order.  Out of line
// (runs once per unit).
template <int B>
__device__ __noinline__ void sum_seams(const KernelArgs& a, const PlaneJob& job, const FilterParams& P, int sx, int pnx,
                                       int pny, int ox, int oy, int W, int Hh, float inv_scale, int tid, int NT) {
    const int S = a.block_step, O = B - S;
    __shared__ int s_arrival;
    __threadfence();  // this unit's band records are visible before it arrives
    __syncthreads();
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        const int k = side == 0 ? sx - 1 : sx;  // seam k lies between strips k and k + 1
        if (k < 0 || k >= job.nsx - 1) continue;
        if (tid == 0) s_arrival = atomicAdd(a.seam_count + job.seam_base + k, 1);
        __syncthreads();
        const bool second = (s_arrival == 1);
        __syncthreads();
        if (!second) continue;
        __threadfence();
        const UnitGeom ul = unit_geom(k, 0, job.nsx, 1, pnx, pny, B, S);
        const UnitGeom ur = unit_geom(k + 1, 0, job.nsx, 1, pnx, pny, B, S);
        const float* recl = a.scratch + (size_t)(job.unit_base + k) * a.rec_stride;
        const float* recr = a.scratch + (size_t)(job.unit_base + k + 1) * a.rec_stride;
        const int pxs = ur.bx0 * S;  // first padded column of the seam
        for (int i = tid; i < O * Hh; i += NT) {
            const int r = i / O;
            const int py = oy + r, px = pxs + (i - r * O);
            if (px < ox || px >= ox + W) continue;
            const int il = band_index(px - ul.bx0 * S, py - ul.by0 * S, ul.fw, ul.fh, O);
            const int ir = band_index(px - ur.bx0 * S, py - ur.by0 * S, ur.fw, ur.fh, O);
            if (!DFT_IN_RANGE(il, a.rec_stride, a.error_flag) || !DFT_IN_RANGE(ir, a.rec_stride, a.error_flag))
                continue;
            const float v = 0.0f + __ldcg(recl + il) + __ldcg(recr + ir);
            store_sample(job.dst, (long long)(py - oy) * job.dst_stride + (px - ox), v, P.kind, P.scale, P.peak,
                         inv_scale);
        }
    }
}

// ---------------------------------------------------------------------------
// main kernel
// ---------------------------------------------------------------------------
template <int B, int T, int NW, int FC, int MINB = 1>
__global__ void __launch_bounds__(NW * 32, MINB) dfttest_unit_kernel(const __grid_constant__ KernelArgs a) {
    static_assert((B & (B - 1)) == 0, "ring rows are indexed with a mask of B - 1");
    using L = Layout<B, T, NW>;
    using TL = Tile<B>;
    constexpr int M = B / 2;
    constexpr int BPW = 32 / B;
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
    // the plane descriptor is read many times per step: keep it on chip
    __shared__ PlaneJob s_job;
    // and so are its format and filter
    __shared__ FilterParams s_par;
    // staging slots of the TMA path: barrier per slot
    __shared__ uint64_t s_sbar[2];
    __shared__ int s_next;
    constexpr int NJI = sizeof(PlaneJob) / sizeof(int), NPI = sizeof(FilterParams) / sizeof(int);
    static_assert(NJI <= 64 && NPI <= 64 && NT >= 128, "descriptor size");
    if (tid == 0) {
        mbar_init(&s_sbar[0], 1);
        mbar_init(&s_sbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // TMA batches this CTA has issued: batch n uses slot n & 1, and is that
    // slot's (n >> 1)-th phase
    uint32_t tma_batches = 0;

    for (int uid = blockIdx.x; uid < a.nunits;) {
    int lo = 0, hi = a.njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.jobs[mid].unit_base <= uid) lo = mid; else hi = mid - 1;
    }
    if (tid < NJI) reinterpret_cast<int*>(&s_job)[tid] = reinterpret_cast<const int*>(&a.jobs[lo])[tid];
    if (tid >= 64 && tid < 64 + NPI) {
        const FilterParams* src = a.params ? a.params + a.jobs[lo].param : &a.p;
        reinterpret_cast<int*>(&s_par)[tid - 64] = reinterpret_cast<const int*>(src)[tid - 64];
    }
    __syncthreads();
    const PlaneJob& job = s_job;
    const FilterParams& P = s_par;
    const int W = job.width, Hh = job.height;
    const int pw = pad_size(W, B, S), ph = pad_size(Hh, B, S);
    const int pnx = (pw - B) / S + 1, pny = (ph - B) / S + 1;
    const int ox = (pw - W) / 2, oy = (ph - Hh) / 2;
    const int lid = uid - job.unit_base;
    const int sx = lid % job.nsx, sy = lid / job.nsx;
    const UnitGeom u = unit_geom(sx, sy, job.nsx, job.nsy, pnx, pny, B, S);
    const int nbx = u.bx1 - u.bx0;
    if (nbx > BPS) {  // uniform: no thread of the CTA touches this unit
        if (tid == 0) atomicExch(a.error_flag, 1);
        return;
    }
    float* rec = a.scratch + (size_t)uid * a.rec_stride;
    const bool is_float = (P.kind == kF32);
    const float inv_scale = 1.0f / P.scale;  // exact for the power-of-two integer scales

    // --- constants into shared memory -----------------------------------
    constexpr bool G = Large<B, T>::value;  // tables read from global memory
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
    const bool dual_tables = (FC != kFilterWiener) && P.sig2 != nullptr;
    if constexpr (!G) {
        for (int i = tid; i < T * B * B; i += NT) s_win[(i / B) * TL::WP + (i % B)] = P.scale * P.win[i];
        for (int i = tid; i < B * B; i += NT) s_wsyn[(i / B) * TL::WP + (i % B)] = P.wsyn[i];
        for (int i = tid; i < T * L::NSLOT * B; i += NT) {
            s_sig[i] = P.sig[i];
            if (dual_tables) s_sig2[i] = P.sig2[i];
        }
        for (int i = tid; i < 2 * T * L::NSLOT * B; i += NT) s_wfe[i] = P.wfe[i];
    }
    const float* t_win = G ? P.win : s_win;
    const float* t_wsyn = G ? P.wsyn : s_wsyn;
    const float* t_sig = G ? P.sig : s_sig;
    const float* t_sig2 = G ? P.sig2 : s_sig2;
    const float* t_wfe = G ? P.wfe : s_wfe;
    for (int i = tid; i < L::ola_floats(pitch); i += NT) s_ola[i] = 0.0f;

    const int fw = u.fw;
    const int x0 = u.bx0 * S;            // footprint origin (padded coordinates)
    const int rowlen = nbx * S + O;      // footprint width
    const bool vec = ((S & 3) == 0);

    // TMA staging: the S new rows of every frame of the next step are copied
    // one row per box (row index through the mirror map, so no mirrored row
    // needs a special path) into a staging slot while this step computes,
    // then converted to FP32 into the input ring.  The box starts at xa, the
    // footprint's first source column rounded down to 16 bytes (negative at
    // the left edge: the copy fills zeros there, and the mirror map of the
    // conversion never reads them).
    const int esz_s = P.kind == kF32 ? 4 : (P.kind == kU16 ? 2 : 1);
    const int al = 16 / esz_s;
    const int xa = (x0 - ox) >= 0 ? ((x0 - ox) / al) * al : -(((ox - x0) + al - 1) / al) * al;
    bool use_tma = a.tmaps != nullptr && job.tmap[0] >= 0;
    {
        // every source column the footprint reads, mirrored ones included, must lie in the box
        const int c_lo = x0 - ox, c_hi = x0 - ox + rowlen - 1;
        int need_lo = max(c_lo, 0), need_hi = min(c_hi, W - 1);
        if (c_lo < 0) need_hi = max(need_hi, -c_lo);
        if (c_hi >= W) need_lo = min(need_lo, 2 * (W - 1) - c_hi);
        use_tma = use_tma && need_lo >= xa && need_hi < xa + a.stage_bw && need_lo >= 0 && need_hi < W;
    }
    const int srb = stage_row_bytes(a.stage_bw, esz_s);
    // staging slots: the first 128-byte boundary at or after stage_off (the host adds 128 bytes)
    unsigned char* s_stg = reinterpret_cast<unsigned char*>(sm) + a.stage_off;
    s_stg += (128u - (smem_addr(s_stg) & 127u)) & 127u;
    // Issued by the last warp (whose threads carry the fewest overlap-add
    // items): lane 0 announces the bytes, then lane k copies row k % S of frame
    // k / S of the next step (rows [n_lo_next, n_lo_next + S)) into slot
    // j_next & 1.
    auto tma_issue = [&](uint32_t batch, int n_lo_next) {
        const int slot = batch & 1;
        if (lane == 0) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&s_sbar[slot], (uint32_t)(T * S * a.stage_bw * esz_s));
        }
        __syncwarp();
        for (int k = lane; k < T * S; k += 32) {
            const int t = k / S, r = k - t * S;
            const unsigned char* map = reinterpret_cast<const unsigned char*>(a.tmaps) + (size_t)job.tmap[t] * kTmapBytes;
            tma_load_2d(s_stg + ((slot * T + t) * S + r) * srb, map, xa, mirror(n_lo_next + r - oy, Hh),
                        &s_sbar[slot]);
        }
    };
    // Conversion items of the TMA path: (frame t, row r, chunk c of cw
    // samples), the same every step; thread tid takes items NT - 1 - tid + j NT
    // (the reverse order of the overlap-add items); the first CJ stay in
    // registers.  Packed: t | r << 3 | c << 9 | fast << 17 (fast: four
    // in-plane samples, aligned in the staged row).
    const int cw = vec ? 4 : 1;
    const int nch = rowlen / cw;
    const int n_conv = use_tma ? T * S * nch : 0;
    auto conv_item = [&](int ci) -> int {
        const int t = ci / (S * nch);
        const int rem = ci - t * S * nch;
        const int r = rem / nch, c = rem - r * nch;
        const int sc = x0 + c * cw - ox;
        const int fast = (cw == 4 && sc >= 0 && sc + 4 <= W && ((sc - xa) & 3) == 0) ? 1 : 0;
        return t | (r << 3) | (c << 9) | (fast << 17);
    };
    constexpr int CJ = 2;
    int conv_it[CJ];
#pragma unroll
    for (int j = 0; j < CJ; ++j) conv_it[j] = NT - 1 - tid + j * NT < n_conv ? conv_item(NT - 1 - tid + j * NT) : -1;
    const int excl_y0 = u.by0 * S + O, excl_y1 = u.by1 * S;
    const int excl_x0 = x0 + O, excl_x1 = u.bx1 * S;

    const StageGeom sgeo{job.src, job.src_stride, P.kind, rowlen, pitch, x0, ox, oy, W, Hh, a.error_flag};
    // prologue: the first B rows of the unit
    stage_rows_plain<B, T, NT>(s_in, sgeo, u.by0 * S, B, tid);

    // Overlap-add items of the vector path (S a multiple of 4, so a segment
    // of 4 pixels never straddles a block edge): item (r, q) is footprint row
    // r of the step, pixels [4q, 4q + 4), covered by blocks b_lo .. b_lo +
    // nk - 1; `ex` marks a segment inside the unit's exclusive columns and
    // the plane.  Thread tid takes items tid + j NT; the first OJ stay in
    // registers for the whole unit.  Packed: r | q << 5 | b_lo << 13 | nk <<
    // 21 | ex << 25.
    constexpr int OJ = 2;
    const int nseg = rowlen >> 2;
    const int n_ola = vec ? B * nseg : 0;
    auto ola_item = [&](int i) -> int {
        const int r = i / nseg, q = i - r * nseg;
        const int px = 4 * q;
        const int b_lo = px + 4 <= B ? 0 : (px + 4 - B + S - 1) / S;
        const int b_hi = min(px / S, nbx - 1);
        const int gx = x0 + px;
        const int ex = (gx >= excl_x0 && gx + 4 <= excl_x1 && gx >= ox && gx + 4 <= ox + W) ? 1 : 0;
        return r | (q << 5) | (b_lo << 13) | ((b_hi - b_lo + 1) << 21) | (ex << 25);
    };
    int ola_it[OJ];
#pragma unroll
    for (int j = 0; j < OJ; ++j) ola_it[j] = tid + j * NT < n_ola ? ola_item(tid + j * NT) : -1;

    // lane roles: rows (b, y) and columns (b, w = 2c + h), B lanes per block
    const int lb = lane / B, lw = lane % B;
    const int bl = warp * BPW + lb;  // local block index of this lane
    float* wbl = s_wbuf + bl * L::BSTR;
    const bool valid = bl < nbx;
    const int blr = valid ? bl : nbx - 1;

    for (int by = u.by0; by < u.by1; ++by) {
        __syncthreads();  // input rows of this step staged; block buffers free
        // next step's new input rows: TMA copies in flight during this step
        if (use_tma && warp == NW - 1 && by + 1 < u.by1) tma_issue(tma_batches, by * S + B);

        // ---- per-warp block transforms (B lanes per block, BPW blocks per warp)
        {
            // row phase: the DC of each block is summed over its rows with shuffles
            int xoff = blr * S;
            if (!DFT_IN_RANGE(xoff + B - 1, pitch, a.error_flag)) xoff = 0;
            const float dc = row_task<B, T>(wbl, s_in, pitch, (by * S + lw) & (B - 1), xoff, t_win, P.scale, lw, vec, valid);
            const float tot = block_row_sum<B>(dc);
            // g = DC / Re(WF[0]) (cpu_source/kernel.hpp:1945)
            if (lw == 0 && valid) s_g[bl] = P.g_div != 0.0f ? __fdiv_rn(tot, P.g_div) : 0.0f;
            __syncwarp();
            column_task<B, T, FC>(wbl, s_g[bl], t_sig, t_sig2, t_wfe, lw, dual_tables, valid, P);
            __syncwarp();
            if (valid) inverse_row_task<B, G>(wbl, t_wsyn, lw);
        }
        __syncthreads();  // block outputs complete; this step's input rows consumed

        const bool last = (by + 1 == u.by1);
        const int n_lo = (by + 1) * S + B - S;  // first new input row of the next step
        // ---- overlap-add of this step's blocks into the ring; rows that no
        // later block reaches are final and leave the ring (same thread, no barrier)
        const int nfin = last ? B : S;
        const FinishGeom fg{job.dst, job.dst_stride, P.kind, P.scale, P.peak, is_float ? 0.0f : inv_scale,
                            x0, ox, oy, W, Hh, excl_x0, excl_x1, excl_y0, excl_y1, rec, fw, u.fh, u.by0 * S, O,
                            a.rec_stride, a.error_flag};
        auto finish = [&](int py, int lx, float v) { finish_px(fg, py, lx, v); };
        if (vec) {
            // segment items (see ola_item): ring cell + covering blocks in ascending order
            auto do_item = [&](int it) {
                const int r = it & 31, q = (it >> 5) & 255, b_lo = (it >> 13) & 255, nk = (it >> 21) & 15;
                const int py = by * S + r;
#ifdef DFT_CHECKS
                if (!DFT_IN_RANGE((py & (B - 1)) * pitch + 4 * q + 3, L::ola_floats(pitch), a.error_flag) ||
                    !DFT_IN_RANGE(4 * q + 3, pitch, a.error_flag) || !DFT_IN_RANGE(b_lo + nk - 1, nbx, a.error_flag))
                    return;
                for (int m = 0; m < nk; ++m)
                    if (!DFT_IN_RANGE(q - (b_lo + m) * (S >> 2), B / 4, a.error_flag)) return;
#endif
                float4* cell = reinterpret_cast<float4*>(s_ola + (py & (B - 1)) * pitch + 4 * q);
                float4 acc = *cell;
                const int sw = TL::swz(r), sq = S >> 2;
                const float* wb0 = s_wbuf + b_lo * L::BSTR + r * B;
                const int c0 = q - b_lo * sq;  // 4-float chunk of segment q in block b_lo
                constexpr int MK = B / 4 < 4 ? B / 4 : 4;  // loads issued together
                float4 v[MK];
#pragma unroll
                for (int m = 0; m < MK; ++m)
                    v[m] = m < nk ? *reinterpret_cast<const float4*>(wb0 + m * L::BSTR + (((c0 - m * sq) ^ sw) << 2))
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int m = 0; m < MK; ++m) {
                    if (m < nk) {
                        acc.x += v[m].x;
                        acc.y += v[m].y;
                        acc.z += v[m].z;
                        acc.w += v[m].w;
                    }
                }
                for (int m = MK; m < nk; ++m) {  // 32x32 blocks at block step 4
                    const float4 w4 = *reinterpret_cast<const float4*>(wb0 + m * L::BSTR + (((c0 - m * sq) ^ sw) << 2));
                    acc.x += w4.x;
                    acc.y += w4.y;
                    acc.z += w4.z;
                    acc.w += w4.w;
                }
                if (r < nfin) {
                    const int px = x0 + 4 * q;
                    if (((it >> 25) & 1) && py >= excl_y0 && py < excl_y1 && py >= oy && py < oy + Hh &&
                        DFT_IN_RANGE(px - ox + 3, W, a.error_flag)) {
                        store4(job.dst, (long long)(py - oy) * job.dst_stride + (px - ox), acc, P.kind, P.peak,
                               inv_scale);
                    } else {
                        finish(py, 4 * q, acc.x);
                        finish(py, 4 * q + 1, acc.y);
                        finish(py, 4 * q + 2, acc.z);
                        finish(py, 4 * q + 3, acc.w);
                    }
                    acc = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                *cell = acc;
            };
#pragma unroll
            for (int j = 0; j < OJ; ++j)
                if (ola_it[j] >= 0) do_item(ola_it[j]);
            for (int i = tid + OJ * NT; i < n_ola; i += NT) do_item(ola_item(i));
        } else {
            ola_scalar<B, T, NW>(fg, s_ola, s_wbuf, pitch, rowlen, by, S, nbx, nfin, tid);
        }

        // ---- the next step's new input rows: by plain loads (planes the TMA copies cannot take)
        if (!use_tma && !last) stage_rows_plain<B, T, NT>(s_in, sgeo, n_lo, S, tid);
        // TMA path: wait for the next step's rows and convert them into the
        // ring.  Items (t, r, 4-sample chunk) go to the threads from the top
        // down, the reverse of the overlap-add items above (the first
        // threads carry one overlap-add item more).
        if (use_tma && !last) {
            // the batch issued at the top of this step
            const int slot = tma_batches & 1;
            const uint32_t parity = (tma_batches >> 1) & 1;
            ++tma_batches;
            if (!mbar_wait(&s_sbar[slot], parity)) {
                // the copies did not complete in time: record it, and let them land before
                // this unit's shared memory can be handed to another unit
                if (tid == 0) atomicExch(a.error_flag, 4);
                mbar_wait(&s_sbar[slot], parity, 16 * kDefaultWaitLimit);
            }
            auto do_conv = [&](int it) {
                const int t = it & 7, r = (it >> 3) & 63, c = (it >> 9) & 255;
                float* dst = s_in + (t * B + ((n_lo + r) & (B - 1))) * pitch + c * cw;
                const unsigned char* srow = s_stg + ((slot * T + t) * S + r) * srb;
                const int sc = x0 + c * cw - ox;  // source column of the first sample
#ifdef DFT_CHECKS
                if (!DFT_IN_RANGE((t * B + ((n_lo + r) & (B - 1))) * pitch + c * cw + cw - 1, T * B * pitch,
                                  a.error_flag) ||
                    !DFT_IN_RANGE(((slot * T + t) * S + r) * srb, stage_bytes(a.stage_bw, esz_s, T, S), a.error_flag))
                    return;
                for (int i = 0; i < cw; ++i)
                    if (!DFT_IN_RANGE(mirror(sc + i, W) - xa, a.stage_bw, a.error_flag)) return;
#endif
                if ((it >> 17) & 1) {
                    *reinterpret_cast<float4*>(dst) = stage_load4(srow, sc - xa, P.kind);
                } else {
                    for (int i = 0; i < cw; ++i) dst[i] = stage_load1(srow, mirror(sc + i, W) - xa, P.kind);
                }
            };
#pragma unroll
            for (int jj = 0; jj < CJ; ++jj)
                if (conv_it[jj] >= 0) do_conv(conv_it[jj]);
            for (int ci = NT - 1 - tid + CJ * NT; ci < n_conv; ci += NT) do_conv(conv_item(ci));
        }
    }

    // ---- seams shared with the neighbouring full-height strips
    if (a.seam_count != nullptr) sum_seams<B>(a, job, P, sx, pnx, pny, ox, oy, W, Hh, is_float ? 0.0f : inv_scale, tid, NT);

    // ---- the next unit (persistent grid)
    if (a.unit_counter == nullptr) break;
    __syncthreads();  // this unit's work is done before its descriptor and rings are replaced
    if (tid == 0) s_next = (int)gridDim.x + atomicAdd(a.unit_counter, 1);
    __syncthreads();
    uid = s_next;
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
        const FilterParams& P = a.params ? a.params[job.param] : a.p;
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
                const int bi = band_index(px - u.bx0 * S, py - u.by0 * S, u.fw, u.fh, O);
                if (DFT_IN_RANGE(bi, a.rec_stride, a.error_flag) && DFT_IN_RANGE(uid, a.nunits, a.error_flag))
                    acc += a.scratch[(size_t)uid * a.rec_stride + bi];
            }
        }
        store_sample(job.dst, (long long)(py - oy) * job.dst_stride + (px - ox), acc, P.kind, P.scale, P.peak);
    }
}

}  // namespace dft2
