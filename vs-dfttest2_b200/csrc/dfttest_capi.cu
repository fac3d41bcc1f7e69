// C ABI of the B200 DFTTest hot path (declared in include/dfttest2_b200.h).
//
// Host responsibilities, mirroring the reference's plugin glue:
//   * argument validation with the reference's messages
//     (nvrtc_source/source.cpp:629-858),
//   * conversion of the FP64 plugin arrays to the FP32 tables the kernel
//     reads (window, per-gain-slot sigma and window spectrum),
//   * splitting every plane into units, sizing the per-unit scratch,
//   * stream slots for concurrent callers (nvrtc_source/source.cpp:272-291),
//   * the host-memory paths and RDFT (cpu_source/source.cpp:269-340).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <complex>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <string>
#include <utility>
#include <vector>

#include "dfttest2_b200.h"
#include "dfttest_host.h"

namespace {
thread_local std::string g_last_error;
}  // namespace

int dft2h::fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int dft2h::prepare_kernel(const void* kern, size_t smem, int threads, int* per_sm) {
    // the limit only ever grows (every launch of the kernel, whatever its
    // size, stays within it); occupancy is cached per launch shape
    struct Limit {
        int dev;
        const void* kern;
        size_t smem;
    };
    struct Occ {
        int dev;
        const void* kern;
        size_t smem;
        int threads;
        int per_sm;
    };
    static std::mutex lock;
    static std::vector<Limit> limits;
    static std::vector<Occ> occ;
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(lock);
    Limit* lim = nullptr;
    for (Limit& l : limits)
        if (l.dev == dev && l.kern == kern) lim = &l;
    if (!lim || lim->smem < smem) {
        CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (lim) lim->smem = smem;
        else limits.push_back(Limit{dev, kern, smem});
    }
    if (!per_sm) return 0;
    for (const Occ& e : occ)
        if (e.dev == dev && e.kern == kern && e.smem == smem && e.threads == threads) {
            *per_sm = e.per_sm;
            return 0;
        }
    int n = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem));
    if (occ.size() > 4096) occ.clear();
    occ.push_back(Occ{dev, kern, smem, threads, n});
    *per_sm = n;
    return 0;
}

dft2h::Variant dft2h::unit_variant(int B, int T, int NW, int MINB) {
    switch (B) {
    case 8: return unit_variant_b8(T, NW, MINB);
    case 16: return unit_variant_b16(T, NW, MINB);
    case 32: return unit_variant_b32(T, NW, MINB);
    }
    return Variant{};
}

#ifndef DFTTEST2_B200_VERSION
#define DFTTEST2_B200_VERSION "0.1.0"
#endif

namespace {

using namespace dft2h;

// kernel variants per (block size, temporal size): NW warps per CTA keeps
// the per-warp block buffers plus the rings within 227 KB of shared memory
// (and 16 warps cap registers at 128 per thread). Strips must be at least
// (B-S)/S blocks wide, so a shape needs enough blocks per step to split
// every plane width: 32x32 shapes have at least 5 (sosize 24 needs 5 for
// some widths; larger overlaps need more, and planes that cannot be split
// are rejected). 32x32 blocks with 3 to 7 frames keep their tables in
// global memory, which leaves room for those strips. 16x16x3 runs two 10-warp
// CTAs per SM (96 registers per thread): 20 warps hide more latency than
// two 8-warp CTAs at 128 registers (2.5 % faster on the 1080p workload).
int strip_blocks(const Variant& v, int B, int S);

Variant select_variant(int B, int T, int S) {
    // DFTTEST2_B200_WARPS=16 / 8 / 4 select other 16x16x3 shapes
    const char* env = std::getenv("DFTTEST2_B200_WARPS");
    if (env && B == 16 && T == 3 && std::atoi(env) == 16) return unit_variant(16, 3, 16, 1);
    if (env && B == 16 && T == 3 && std::atoi(env) == 8) return unit_variant(16, 3, 8, 2);
    if (env && B == 16 && T == 3 && std::atoi(env) == 4) return unit_variant(16, 3, 4, 4);
    switch (B) {
    case 8:
        switch (T) {
        case 1: return unit_variant(8, 1, 16, 1);
        case 3: return unit_variant(8, 3, 16, 1);
        case 5: return unit_variant(8, 5, 16, 1);
        case 7: return unit_variant(8, 7, 16, 1);
        }
        break;
    case 16:
        switch (T) {
        case 1: return unit_variant(16, 1, 16, 1);
        case 3: return unit_variant(16, 3, 10, 2);
        case 5: return unit_variant(16, 5, 12, 1);
        case 7: return unit_variant(16, 7, 8, 1);
        }
        break;
    case 32:
        switch (T) {
        case 1: return unit_variant(32, 1, 16, 1);
        // one 8-warp CTA per SM (8-block strips): at block step 8 it ran 21 % faster than two
        // 6-warp CTAs on the 32-clip batch (65.1 against 82.8 ms) and 17 % on its 640x360 form
        case 3: return unit_variant(32, 3, 8, 1);
        case 5: {
            // one CTA per SM of 5, 6 or 7 warps: the shape whose strip (as wide as shared memory
            // allows, at most one block per warp) keeps the most warps busy, the fewest warps on a tie
            Variant best;
            int best_w = 0;
            for (int nw : {5, 6, 7}) {
                const Variant v = unit_variant(32, 5, nw, 1);
                const int w = std::min(strip_blocks(v, B, S), nw);
                if (w > best_w) {
                    best = v;
                    best_w = w;
                }
            }
            return best;
        }
        case 7: return unit_variant(32, 7, 5, 1);
        }
        break;
    }
    return Variant{};
}

// Blocks per strip for a kernel shape and block step: the shape's blocks per
// step, fewer when the rings for a large step would not fit in the 227 KB of
// shared memory a CTA may have.
int strip_blocks(const Variant& v, int B, int S) {
    constexpr size_t kMaxSmem = 227 * 1024;
    int w = v.nw * v.bpw;
    while (w > 1 && v.smem((((w * S) + (B - S)) + 3) & ~3) > kMaxSmem) --w;
    return w;
}

// Kernel shapes the batch autotuner may time besides select_variant's
// choice: other warp counts per CTA for the block sizes and temporal sizes of
// multi-clip batches (fewer warps per CTA = narrower strips, more CTAs).
std::vector<Variant> candidate_variants(int B, int T, int S) {
    std::vector<Variant> v;
    v.push_back(select_variant(B, T, S));
    if (!v.back().main) return {};
    if (B == 8 && T == 1) v.push_back(unit_variant(8, 1, 8, 2));
    if (B == 8 && T == 3) v.push_back(unit_variant(8, 3, 8, 2));
    if (B == 32 && T == 1) v.push_back(unit_variant(32, 1, 8, 1));
    if (B == 32 && T == 3) {
        v.push_back(unit_variant(32, 3, 6, 2));
        v.push_back(unit_variant(32, 3, 4, 2));
    }
    if (B == 16 && T == 1) v.push_back(unit_variant(16, 1, 8, 2));
    if (B == 16 && T == 3) {
        v.push_back(unit_variant(16, 3, 8, 2));
        v.push_back(unit_variant(16, 3, 16, 1));
        v.push_back(unit_variant(16, 3, 4, 4));
    }
    // 32x32x5: the warp buffers (20.5 KB each) and the strip ring share 227 KB; 5, 6 and 7 warps
    // fit with strips of up to 5 / 6 / 7 blocks (one CTA per SM each)
    if (B == 32 && T == 5)
        for (int nw : {7, 6, 5}) {
            const Variant o = unit_variant(32, 5, nw, 1);
            if (o.main != v.front().main) v.push_back(o);
        }
    return v;
}

// Encoded tensor maps kept across launches (a slot's launches reuse its
// frame buffers): key = (plane pointer, width, height, stride, format, box).
struct MapKey {
    const void* p;
    int w, h, kind, box;
    long long stride;
    bool operator==(const MapKey& o) const {
        return p == o.p && w == o.w && h == o.h && kind == o.kind && box == o.box && stride == o.stride;
    }
};
struct MapKeyHash {
    size_t operator()(const MapKey& k) const {
        size_t h = std::hash<const void*>()(k.p);
        for (long long v : {(long long)k.w, (long long)k.h, (long long)k.kind, (long long)k.box, k.stride})
            h = h * 1000003u ^ std::hash<long long>()(v);
        return h;
    }
};
using MapCache = std::unordered_map<MapKey, CUtensorMap, MapKeyHash>;

struct Slot {
    cudaEvent_t done = nullptr;
    cudaStream_t stream = nullptr;        // own stream (host paths)
    cudaStream_t up = nullptr;            // host -> device copies of the clip path
    cudaStream_t down = nullptr;          // device -> host copies of the clip path
    cudaEvent_t ev_up[2] = {};
    cudaEvent_t ev_comp[2] = {};
    cudaEvent_t ev_down[2] = {};
    dft2::PlaneJob* d_jobs = nullptr;
    size_t jobs_cap = 0;
    float* d_scratch = nullptr;
    size_t scratch_cap = 0;               // floats
    int* d_seams = nullptr;               // seam arrival counters (full-strip launches)
    size_t seams_cap = 0;
    void* d_tmaps = nullptr;              // tensor maps of the TMA row staging
    size_t tmaps_cap = 0;
    MapCache map_cache;                   // encoded tensor maps of earlier launches
    int* d_error = nullptr;               // error word of the slot's kernels (0 = no failure)
    int* h_error = nullptr;               // pinned copy of d_error read by the host-synchronous paths
    // host path staging
    void* d_frames = nullptr;
    size_t frames_cap = 0;
    void* h_pinned = nullptr;
    size_t pinned_cap = 0;
    float* d_sigtab = nullptr;       // gain-slot sigma tables built from a device sigma array
    size_t sigtab_cap = 0;
    dft2::GradJob* d_gjobs = nullptr;
    size_t gjobs_cap = 0;
    dft2::TcJob* d_tcjobs = nullptr;      // tensor-core form: work-list and accumulator planes
    size_t tcjobs_cap = 0;
    float* d_acc = nullptr;
    size_t acc_cap = 0;
};

}  // namespace

struct dfttest2_b200_filter {
    int device = 0;
    int radius = 0, T = 1, B = 16, S = 16, H = 8;
    int filter_type = 0;
    bool zero_mean = true;
    float sigma2 = 0, pmin = 0, pmax = 0;
    int syn_slice = 0;
    float g_div = 0.0f;
    bool asym = false;
    Variant var;
    int num_sms = 148;

    float* d_win = nullptr;
    float* d_wsyn = nullptr;
    float* d_sig = nullptr;
    float* d_sig2 = nullptr;
    float* d_wfe = nullptr;
    int wmask = 0;
    // differentiable path: full (t, y, x) arrays and the gain-slot -> bin maps
    float* d_sigma_full = nullptr;  // [T][B][X]
    float* d_wf_full = nullptr;     // [T][B][X][2]
    int* d_sig_idx = nullptr;       // [T][B/2+2][B]
    int* d_sig2_idx = nullptr;
    int n_slots = 0;
    // tensor-core form (dfttest2_b200_set_precision)
    int tc_mode = 0;
    void* d_gmat = nullptr;
    int gmat_bytes = 0;
    // tensor-core strip form (dfttest_tc2.cuh): kernels, constant image, shape; tc2.main is
    // null when the tensor-core mode runs the tile form of dfttest_tc.cuh instead
    Variant tc2;
    char* d_tc2 = nullptr;
    Tc2Shape tc2_shape;
    // plugin arrays kept on the host for the constant images of the tensor-core forms
    std::vector<double> h_win, h_wf;
    std::vector<float> h_sig;
    int wait_limit = dft2::kDefaultWaitLimit;  // iteration limit of the kernels' bounded device waits

    std::vector<Slot> slots;
    std::vector<int> free_slots;
    std::mutex slot_lock;
    std::condition_variable slot_cv;

    // source planes already on the device, keyed by (clip frame number, plane
    // index), for the per-frame host path (dfttest2_b200_process_plane_host_cached)
    struct CacheEntry {
        int id = -1, plane = -1;
        size_t bytes = 0, cap = 0;
        void* d = nullptr;
        int refs = 0;                   // calls using the entry
        bool issued = false;            // its upload is queued (`ready` recorded)
        unsigned long long used = 0;    // last use, for least-recently-used eviction
        cudaEvent_t ready = nullptr;
    };
    std::vector<CacheEntry> cache;
    std::mutex cache_lock;
    std::condition_variable cache_cv;
    unsigned long long cache_clock = 0;
};

namespace {

struct SlotGuard {
    dfttest2_b200_filter* f;
    int idx;
    SlotGuard(dfttest2_b200_filter* f_) : f(f_) {
        std::unique_lock<std::mutex> lk(f->slot_lock);
        f->slot_cv.wait(lk, [&] { return !f->free_slots.empty(); });
        idx = f->free_slots.back();
        f->free_slots.pop_back();
    }
    ~SlotGuard() {
        {
            std::lock_guard<std::mutex> lk(f->slot_lock);
            f->free_slots.push_back(idx);
        }
        f->slot_cv.notify_one();
    }
    Slot& slot() { return f->slots[idx]; }
};

// grows a device buffer after the slot's previous work has finished
template <typename Tp>
int ensure(Tp*& ptr, size_t& cap, size_t need, cudaEvent_t done) {
    if (need <= cap) return 0;
    CUDA_TRY(cudaEventSynchronize(done));
    if (ptr) CUDA_TRY(cudaFree(ptr));
    ptr = nullptr;
    cap = 0;
    size_t n = std::max(need, cap * 2);
    if (cudaMalloc((void**)&ptr, n * sizeof(Tp)) != cudaSuccess) {
        cudaGetLastError();
        return fail(DFTTEST2_B200_ENOMEM, "device allocation failed");
    }
    cap = n;
    return 0;
}

int ensure_bytes(void*& ptr, size_t& cap, size_t need, cudaEvent_t done) {
    if (need <= cap) return 0;
    CUDA_TRY(cudaEventSynchronize(done));
    if (ptr) CUDA_TRY(cudaFree(ptr));
    ptr = nullptr;
    cap = 0;
    if (cudaMalloc(&ptr, need) != cudaSuccess) {
        cudaGetLastError();
        return fail(DFTTEST2_B200_ENOMEM, "device allocation failed");
    }
    cap = need;
    return 0;
}

int ensure_pinned(void*& ptr, size_t& cap, size_t need, cudaEvent_t done) {
    if (need <= cap) return 0;
    CUDA_TRY(cudaEventSynchronize(done));
    if (ptr) CUDA_TRY(cudaFreeHost(ptr));
    ptr = nullptr;
    cap = 0;
    if (cudaMallocHost(&ptr, need) != cudaSuccess) {
        cudaGetLastError();
        return fail(DFTTEST2_B200_ENOMEM, "pinned host allocation failed");
    }
    cap = need;
    return 0;
}

int bytes_of(int sample_type, int bits) {
    if (sample_type == DFTTEST2_B200_FLOAT) return 4;
    return bits <= 8 ? 1 : 2;
}

int check_format(int sample_type, int bits) {
    if (sample_type == DFTTEST2_B200_INTEGER) {
        if (bits < 8 || bits > 16) return fail(DFTTEST2_B200_EINVAL, "only 8-16 bit integer format input is supported");
        return 0;
    }
    if (sample_type == DFTTEST2_B200_FLOAT && bits == 32) return 0;
    return fail(DFTTEST2_B200_EINVAL, "only 8-16 bit integer and 32-bit float format input is supported");
}

// planning of one launch over a list of planes
struct Plan {
    std::vector<dft2::PlaneJob> jobs;
    int nunits = 0;
    int nfix = 0;
    int rec_stride = 0;
    int pitch = 0;
    int nseams = 0;            // seams between strips, summed over jobs
    bool full_strips = false;  // every job has nsy = 1
};

// a plane in the work-list: strides in elements, `param` indexes per-job formats and filters
struct PlaneRef {
    const void* src[7];
    void* dst;
    long long src_stride, dst_stride;
    int width, height;
    int param;
};

// Strips of a plane pnx blocks wide for a kernel of BPS blocks per step:
// at most BPS blocks each, and at least O/S blocks where possible so that the
// two edge bands of a strip stay apart (then every overlap seam is shared by
// exactly two strips).  With high overlap no such split may exist (32x32
// blocks at sosize 26..31): the strips are then BPS wide and `narrow` is set;
// their band records hold whole footprints and the fix-up kernel sums every
// unit that covers a pixel.
int strip_count(int pnx, int B, int S, int BPS, bool& narrow) {
    const int O = B - S;
    const int min_w = (O + S - 1) / S;
    int nsx = (pnx + BPS - 1) / BPS;
    while (nsx > 1 && pnx / nsx < min_w) --nsx;
    narrow = false;
    if ((pnx + nsx - 1) / nsx > BPS) {
        nsx = (pnx + BPS - 1) / BPS;
        narrow = nsx > 1;
    }
    return nsx;
}

// Unit split and work-list of planes that share (B, S) and a kernel shape of
// BPS blocks per step: strips of at most BPS blocks (strip_count); each strip
// is cut into segments until the launch has about `target` units (segments no
// shorter than max(O/S, 4) blocks).
int plan_units(int B, int S, int BPS, const std::vector<PlaneRef>& planes, long long target, Plan& plan) {
    const int O = B - S;
    const int n = (int)planes.size();
    plan.jobs.resize(n);
    long long strips_total = 0;
    int max_pny = 0;
    for (const PlaneRef& p : planes) {
        strips_total += (dft2::pad_num(p.width, B, S) + BPS - 1) / BPS;
        max_pny = std::max(max_pny, dft2::pad_num(p.height, B, S));
    }
    int nsy = 1;
    if (strips_total < target) nsy = (int)((target + strips_total - 1) / strips_total);
    const int min_seg = std::max((O + S - 1) / S, 4);
    nsy = std::max(1, std::min(nsy, max_pny / min_seg));

    int unit = 0, fix = 0, rec = 0, seams = 0;
    bool full = true;
    for (int i = 0; i < n; ++i) {
        const PlaneRef& p = planes[i];
        dft2::PlaneJob& j = plan.jobs[i];
        std::memset(&j, 0, sizeof(j));
        for (int t = 0; t < 7; ++t) {
            j.src[t] = p.src[t];
            j.tmap[t] = -1;
        }
        j.dst = p.dst;
        j.src_stride = p.src_stride;
        j.dst_stride = p.dst_stride;
        j.width = p.width;
        j.height = p.height;
        j.param = p.param;
        const int pnx = dft2::pad_num(p.width, B, S), pny = dft2::pad_num(p.height, B, S);
        bool narrow = false;
        j.nsx = strip_count(pnx, B, S, BPS, narrow);
        j.nsy = std::max(1, std::min(nsy, pny / min_seg));
        j.unit_base = unit;
        j.fix_base = fix;
        j.seam_base = seams;
        seams += j.nsx - 1;
        full = full && j.nsy == 1 && !narrow;
        unit += j.nsx * j.nsy;
        fix += (j.nsx - 1) * O * p.height + (j.nsy - 1) * O * p.width;
        const int wmax = (pnx + j.nsx - 1) / j.nsx, hmax = (pny + j.nsy - 1) / j.nsy;
        rec = std::max(rec, dft2::band_record_size(wmax * S + O, hmax * S + O, O));
    }
    plan.nunits = unit;
    plan.nfix = fix;
    plan.rec_stride = std::max(rec, 1);
    plan.pitch = ((BPS * S + O) + 3) & ~3;
    plan.nseams = seams;
    plan.full_strips = full;
    return 0;
}

// the mirror padding must stay inside the plane (cpu_source/getframe_impl.cpp:44-62 reads 2*ox - x)
bool plane_fits(int width, int height, int B, int S) {
    const int pw = dft2::pad_size(width, B, S), ph = dft2::pad_size(height, B, S);
    const int ox = (pw - width) / 2, oy = (ph - height) / 2;
    return width > std::max(ox, pw - width - ox) && height > std::max(oy, ph - height - oy);
}

// Segments per strip (nsy, the same for every plane, capped per plane as in
// plan_units) for a plain launch. Full-height strips keep the seams inside
// the unit kernel, so launches with at least four waves of strips on the
// resident CTA slots use them; smaller launches are cut into about eight
// waves of units (at most 16 segments per strip), which keeps the last,
// partly filled wave short at the price of the fix-up kernel. Measured on
// 1080p YUV420P16 clips with 16x16x3 blocks (two CTAs per SM): 12 frames
// 2,770 frames/s with full strips, 2,911 with 2 segments, 2,962 with 4; 4
// frames 2,573 with 3 segments, 2,748 with 6, 2,698 with 12; 1 frame 2,334
// with 16 segments, 1,705 with 6.
int choose_nsy(const std::vector<PlaneRef>& planes, int B, int S, int BPS, int slots) {
    long long strips_total = 0;
    for (const PlaneRef& p : planes) strips_total += (dft2::pad_num(p.width, B, S) + BPS - 1) / BPS;
    if (strips_total == 0 || strips_total >= 4LL * slots) return 1;
    return (int)std::min<long long>(16, (8LL * slots + strips_total - 1) / strips_total);
}

int make_plan(const dfttest2_b200_filter* f, const dfttest2_b200_plane* planes, int n, int bps_bytes, Plan& plan) {
    std::vector<PlaneRef> refs(n);
    for (int i = 0; i < n; ++i) {
        const dfttest2_b200_plane& p = planes[i];
        if (!plane_fits(p.width, p.height, f->B, f->S))
            return fail(DFTTEST2_B200_EINVAL, "plane too small for the block size");
        for (int t = 0; t < f->T; ++t) {
            if (p.src[t] == nullptr) return fail(DFTTEST2_B200_EINVAL, "null source plane");
        }
        if (!p.dst) return fail(DFTTEST2_B200_EINVAL, "null destination plane");
        if (p.src_stride % bps_bytes || p.dst_stride % bps_bytes || p.src_stride < (ptrdiff_t)p.width * bps_bytes ||
            p.dst_stride < (ptrdiff_t)p.width * bps_bytes)
            return fail(DFTTEST2_B200_EINVAL, "invalid stride");
        PlaneRef& r = refs[i];
        std::memset(&r, 0, sizeof(r));
        for (int t = 0; t < f->T; ++t) r.src[t] = p.src[t];
        r.dst = p.dst;
        r.src_stride = p.src_stride / bps_bytes;
        r.dst_stride = p.dst_stride / bps_bytes;
        r.width = p.width;
        r.height = p.height;
    }
    // units go out in plan order: tall planes first (their strips are the
    // longest units), so that short units fill the last wave
    std::stable_sort(refs.begin(), refs.end(), [](const PlaneRef& x, const PlaneRef& y) { return x.height > y.height; });
    const bool tc2 = f->tc_mode && f->tc2.main;
    const int BPS = tc2 ? f->tc2_shape.nbx : strip_blocks(f->var, f->B, f->S);
    const int minb = tc2 ? f->tc2.minb : f->var.minb;
    const int nsy = choose_nsy(refs, f->B, f->S, BPS, std::max(1, minb) * f->num_sms);
    long long strips_total = 0;
    for (const PlaneRef& r : refs) strips_total += (dft2::pad_num(r.width, f->B, f->S) + BPS - 1) / BPS;
    // plan_units derives nsy = ceil(target / strips) = nsy from this target
    return plan_units(f->B, f->S, BPS, refs, nsy > 1 ? nsy * strips_total : 1, plan);
}

// ---- tensor-core form ------------------------------------------------------
int launch_tc(dfttest2_b200_filter* f, Slot& slot, const Plan& plan, int kind, float scale, float peak,
              cudaStream_t stream) {
    const TcVariant v = select_tc(f->B, f->T, f->tc_mode);
    if (!v.wiener) return fail(DFTTEST2_B200_EINVAL, "tensor-core form not available for these arguments");
    const int B = f->B, S = f->S;
    CUDA_TRY(cudaStreamWaitEvent(stream, slot.done, 0));
    std::vector<dft2::TcJob> jobs(plan.jobs.size());
    long long ntiles = 0;
    size_t acc = 0;
    for (size_t i = 0; i < plan.jobs.size(); ++i) {
        const dft2::PlaneJob& p = plan.jobs[i];
        dft2::TcJob& j = jobs[i];
        std::memset(&j, 0, sizeof(j));
        for (int t = 0; t < 7; ++t) j.src[t] = p.src[t];
        j.dst = p.dst;
        j.src_stride = p.src_stride;
        j.dst_stride = p.dst_stride;
        j.width = p.width;
        j.height = p.height;
        j.ntx = (dft2::pad_num(p.width, B, S) + v.tb - 1) / v.tb;
        j.tile_base = (int)ntiles;
        ntiles += (long long)j.ntx * dft2::pad_num(p.height, B, S);
        if (ntiles > INT_MAX) return fail(DFTTEST2_B200_EINVAL, "too many planes in one call");
        j.acc = reinterpret_cast<float*>(acc);  // offset for now
        acc += (size_t)p.width * p.height;
    }
    if (jobs.size() > 65535) return fail(DFTTEST2_B200_EINVAL, "at most 65535 planes per call in the tensor-core form");
    if (int rc = ensure(slot.d_tcjobs, slot.tcjobs_cap, jobs.size(), slot.done)) return rc;
    if (int rc = ensure(slot.d_acc, slot.acc_cap, std::max<size_t>(acc, 1), slot.done)) return rc;
    for (auto& j : jobs) j.acc = slot.d_acc + reinterpret_cast<size_t>(j.acc);
    CUDA_TRY(cudaMemcpyAsync(slot.d_tcjobs, jobs.data(), jobs.size() * sizeof(dft2::TcJob), cudaMemcpyHostToDevice,
                             stream));
    CUDA_TRY(cudaMemsetAsync(slot.d_acc, 0, acc * sizeof(float), stream));
    dft2::TcArgs a{};
    a.jobs = slot.d_tcjobs;
    a.njobs = (int)jobs.size();
    a.ntiles = (int)ntiles;
    a.block_step = S;
    a.p.kind = kind;
    a.p.scale = scale;
    a.p.peak = peak;
    a.p.filter_type = f->filter_type;
    a.p.sigma2 = f->sigma2;
    a.p.pmin = f->pmin;
    a.p.pmax = f->pmax;
    a.p.g_div = f->zero_mean ? f->g_div : 0.0f;
    a.p.win = f->d_win;
    a.p.wsyn = f->d_wsyn;
    a.sigma = f->d_sigma_full;
    a.wf = f->d_wf_full;
    a.gmat = f->d_gmat;
    a.gmat_bytes = f->gmat_bytes;
    a.error_flag = slot.d_error;
    a.wait_limit = f->wait_limit;
    const int patch_w = B + (v.tb - 1) * S;
    const size_t smem = v.smem(patch_w);
    if (smem > 227 * 1024) return fail(DFTTEST2_B200_EINVAL, "block step too large for the tensor-core form");
    TcKernelFn kern = f->filter_type == 0 ? v.wiener : v.generic;
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    int per_sm = 0;
    if (int rc = prepare_kernel((const void*)kern, smem, 256, &per_sm)) return rc;
    if (per_sm < 1) return fail(DFTTEST2_B200_ECUDA, "tensor-core kernel does not fit on an SM");
    // two CTAs per SM (register bound of the kernel; tensor memory holds 2 x 256 columns); the occupancy
    // query can report one for this shared-memory size while two are resident, so it is not used for the grid
    const int grid = std::max(1, std::min(a.ntiles, f->num_sms * 2));
    kern<<<grid, 256, smem, stream>>>(a);
    CUDA_TRY(cudaGetLastError());
    dim3 fg((unsigned)std::max<long long>(1, std::min<long long>(64, (acc / jobs.size() + 255) / 256)),
            (unsigned)jobs.size());
    if (int rc = launch_tc_finalize(a, fg, stream)) return rc;
    CUDA_TRY(cudaEventRecord(slot.done, stream));
    return 0;
}

// ---- TMA staging of the unit kernel's input rows ---------------------------
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Tensor maps for the TMA staging of a launch: one 2D map (width x height
// samples, rows `stride` bytes apart, box bw x 1) per distinct source plane;
// jobs[i].tmap[t] indexes them.  kinds[i] is job i's sample format.  A job
// keeps tmap -1 (staged by plain loads) when its planes break the copy
// engine's rules (16-byte aligned base and stride, plane at least bw wide) or
// when some unit of it would read a mirrored column outside the box.  bw = 0
// (no staging) when the box would exceed 256 samples, no job qualifies, or
// DFTTEST2_B200_TMA=0.  bw is a multiple of 16 samples, valid for every
// format; `stage` receives the staging bytes the kernel needs (both slots,
// widest format) plus 128 for alignment.

void build_stage_maps(std::vector<dft2::PlaneJob>& jobs, const std::vector<int>& kinds, int B, int S, int T,
                      int pitch, std::vector<CUtensorMap>& maps, int& bw, size_t& stage, MapCache* cache = nullptr) {
    maps.clear();
    bw = 0;
    stage = 0;
    for (auto& j : jobs)
        for (int t = 0; t < 7; ++t) j.tmap[t] = -1;
    const char* env = std::getenv("DFTTEST2_B200_TMA");
    if (env && std::atoi(env) == 0) return;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return;
    const int box = ((pitch + 15) + 15) / 16 * 16;  // footprint + alignment slack of the narrowest format
    if (box > 256) return;
    const int O = B - S;
    if (cache && cache->size() > 8192) cache->clear();
    std::unordered_map<MapKey, int, MapKeyHash> index;  // this launch's maps
    for (size_t ji = 0; ji < jobs.size(); ++ji) {
        dft2::PlaneJob& j = jobs[ji];
        const int kind = kinds[ji];
        const int esz = kind == dft2::kF32 ? 4 : (kind == dft2::kU16 ? 2 : 1);
        const int al = 16 / esz;
        const long long sb = j.src_stride * esz;
        bool ok = sb % 16 == 0 && j.width >= box && sb < (1LL << 40);
        // every unit's footprint columns (mirrored ones included) inside its box, as the kernel checks
        const int pw = dft2::pad_size(j.width, B, S), pnx = dft2::pad_num(j.width, B, S);
        const int ox = (pw - j.width) / 2;
        for (int sx = 0; sx < j.nsx && ok; ++sx) {
            const int bx0 = dft2::split_lo(sx, pnx, j.nsx), bx1 = dft2::split_lo(sx + 1, pnx, j.nsx);
            const int x0 = bx0 * S, rowlen = (bx1 - bx0) * S + O;
            const int xa = (x0 - ox) >= 0 ? ((x0 - ox) / al) * al : -(((ox - x0) + al - 1) / al) * al;
            const int c_lo = x0 - ox, c_hi = x0 - ox + rowlen - 1;
            int need_lo = std::max(c_lo, 0), need_hi = std::min(c_hi, j.width - 1);
            if (c_lo < 0) need_hi = std::max(need_hi, -c_lo);
            if (c_hi >= j.width) need_lo = std::min(need_lo, 2 * (j.width - 1) - c_hi);
            ok = need_lo >= xa && need_hi < xa + box && need_lo >= 0 && need_hi < j.width;
        }
        int idx[7];
        const CUtensorMapDataType dt = kind == dft2::kF32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                       : kind == dft2::kU16 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                                            : CU_TENSOR_MAP_DATA_TYPE_UINT8;
        for (int t = 0; t < T && ok; ++t) {
            ok = (reinterpret_cast<uintptr_t>(j.src[t]) & 15) == 0;
            if (!ok) break;
            const MapKey key{j.src[t], j.width, j.height, kind, box, sb};
            auto it = index.find(key);
            if (it == index.end()) {
                CUtensorMap m;
                auto hit = cache ? cache->find(key) : MapCache::iterator();
                if (cache && hit != cache->end()) {
                    m = hit->second;
                } else {
                    const cuuint64_t dims[2] = {(cuuint64_t)j.width, (cuuint64_t)j.height};
                    const cuuint64_t strides[1] = {(cuuint64_t)sb};
                    const cuuint32_t boxd[2] = {(cuuint32_t)box, 1u};
                    const cuuint32_t estr[2] = {1u, 1u};
                    if (enc(&m, dt, 2, const_cast<void*>(j.src[t]), dims, strides, boxd, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
                        ok = false;
                        break;
                    }
                    if (cache) cache->emplace(key, m);
                }
                it = index.emplace(key, (int)maps.size()).first;
                maps.push_back(m);
            }
            idx[t] = it->second;
        }
        for (int t = 0; t < 7; ++t) j.tmap[t] = (ok && t < T) ? idx[t] : -1;
    }
    if (maps.empty()) return;
    bw = box;
    stage = (size_t)dft2::stage_bytes(bw, 4, T, S) + 128;
}

int launch(dfttest2_b200_filter* f, Slot& slot, const Plan& plan, int kind, float scale, float peak,
           cudaStream_t stream, const float* sig_override = nullptr, const float* sig2_override = nullptr) {
    if (plan.nunits == 0) return 0;
    // the tensor-core strip form runs in this framework; the tile form has its own launcher
    const bool tc2 = f->tc_mode && f->tc2.main && !sig_override;
    if (f->tc_mode && !sig_override && !tc2) return launch_tc(f, slot, plan, kind, scale, peak, stream);
    const Variant& var = tc2 ? f->tc2 : f->var;
    CUDA_TRY(cudaStreamWaitEvent(stream, slot.done, 0));
    if (int rc = ensure(slot.d_jobs, slot.jobs_cap, plan.jobs.size(), slot.done)) return rc;
    const size_t scratch_need = (size_t)plan.nunits * plan.rec_stride;
    if (int rc = ensure(slot.d_scratch, slot.scratch_cap, scratch_need, slot.done)) return rc;
    // input rows staged by TMA where the planes allow it (within the shared-memory budget)
    std::vector<dft2::PlaneJob> jobs(plan.jobs);
    std::vector<CUtensorMap> maps;
    int bw = 0;
    size_t stage = 0;
    const size_t smem_base = tc2 ? f->tc2_shape.smem : f->var.smem(plan.pitch);
    // the strip form reads 8 * xg footprint columns; its staging slots hold this launch's format
    build_stage_maps(jobs, std::vector<int>(jobs.size(), kind), f->B, f->S, f->T,
                     tc2 ? 8 * f->tc2_shape.xg : plan.pitch, maps, bw, stage, &slot.map_cache);
    if (tc2 && bw > 0)
        stage = (size_t)dft2::stage_bytes(bw, kind == dft2::kF32 ? 4 : (kind == dft2::kU16 ? 2 : 1), f->T, f->S) + 128;
    size_t smem = smem_base;
    if (bw > 0) {
        const size_t with_stage = ((smem_base + 127) & ~(size_t)127) + stage;
        if (with_stage <= 227 * 1024) {
            smem = with_stage;
        } else {
            bw = 0;
            for (auto& j : jobs)
                for (int t = 0; t < 7; ++t) j.tmap[t] = -1;
        }
    }
    if (bw > 0) {
        if (int rc = ensure_bytes(slot.d_tmaps, slot.tmaps_cap, maps.size() * sizeof(CUtensorMap), slot.done))
            return rc;
        CUDA_TRY(cudaMemcpyAsync(slot.d_tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                                 stream));
    }
    CUDA_TRY(cudaMemcpyAsync(slot.d_jobs, jobs.data(), jobs.size() * sizeof(dft2::PlaneJob), cudaMemcpyHostToDevice,
                             stream));

    dft2::KernelArgs a{};
    a.jobs = slot.d_jobs;
    a.njobs = (int)plan.jobs.size();
    a.nunits = plan.nunits;
    a.nfix = plan.nfix;
    a.p.kind = kind;
    a.p.scale = scale;
    a.p.peak = peak;
    a.block_step = f->S;
    a.p.filter_type = f->filter_type;
    a.p.sigma2 = f->sigma2;
    a.p.pmin = f->pmin;
    a.p.pmax = f->pmax;
    a.p.g_div = f->zero_mean ? f->g_div : 0.0f;
    a.p.win = f->d_win;
    a.p.wsyn = f->d_wsyn;
    a.p.sig = sig_override ? sig_override : f->d_sig;
    a.p.sig2 = sig_override ? sig2_override : (f->asym ? f->d_sig2 : nullptr);
    a.p.wfe = f->d_wfe;
    a.p.wmask = f->zero_mean ? f->wmask : 0;
    a.scratch = slot.d_scratch;
    a.rec_stride = plan.rec_stride;
    a.ring_pitch = plan.pitch;
    a.error_flag = slot.d_error;
    // full-height strips: the unit kernel sums its seams itself
    const bool inline_seams = plan.nfix > 0 && plan.full_strips && plan.nseams > 0;
    // Persistent grid (a work counter after the seam counters; both zeroed by
    // one memset) for launches of full-height strips, whose units are long;
    // launches of strip segments (short units) run one unit per CTA, which
    // measured 14 % faster there (the block scheduler balances as well, with
    // less per-unit synchronisation).  DFTTEST2_B200_PERSISTENT=0 / 1 forces
    // either.
    // (the tensor-core strip form runs one unit per CTA: its persistent grid measured 1.6x slower on
    // the 64-frame 1080p step, 42.1 against 25.7 ms)
    const char* penv = std::getenv("DFTTEST2_B200_PERSISTENT");
    const bool persistent = penv ? std::atoi(penv) != 0 : plan.full_strips && !tc2;
    if (inline_seams || persistent) {
        const size_t ncount = (size_t)(inline_seams ? plan.nseams : 0) + 1;
        if (int rc = ensure(slot.d_seams, slot.seams_cap, ncount, slot.done)) return rc;
        CUDA_TRY(cudaMemsetAsync(slot.d_seams, 0, ncount * sizeof(int), stream));
        if (inline_seams) a.seam_count = slot.d_seams;
        if (persistent) a.unit_counter = slot.d_seams + (inline_seams ? plan.nseams : 0);
    }

    if (bw > 0) {
        a.tmaps = slot.d_tmaps;
        a.stage_bw = bw;
        a.stage_off = (int)((smem_base + 127) & ~(size_t)127);
    }
    if (tc2) {
        a.tc_consts = f->d_tc2;
        a.wait_limit = f->wait_limit;
    }
    KernelFn kern = (f->filter_type == 0 && !f->asym && !sig_override) ? var.main : var.generic;
    int per_sm = 0;
    if (int rc = prepare_kernel((const void*)kern, smem, var.nw * 32, &per_sm)) return rc;
    int grid = plan.nunits;
    if (persistent) grid = std::min(plan.nunits, std::max(1, per_sm) * f->num_sms);  // one CTA per resident slot
    kern<<<grid, var.nw * 32, smem, stream>>>(a);
    CUDA_TRY(cudaGetLastError());
    if (plan.nfix > 0 && !inline_seams) {
        const int threads = 256;
        const int blocks = std::min((plan.nfix + threads - 1) / threads, f->num_sms * 8);
        var.fixup<<<blocks, threads, 0, stream>>>(a);
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaEventRecord(slot.done, stream));
    return 0;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Window-spectrum entry (re, im) of temporal bin t as the FP32 kernel sees
// it: the kernel feeds each block's frames centre first (frame r at time 0),
// which multiplies temporal bin t of every spectrum by w^(t r), w = e^(2 pi i / T).
void centre_first_wf(const double* wf, int t, int T, int r, float& re, float& im) {
    const double ang = 2.0 * 3.14159265358979323846 * (double)((t * r) % T) / T;
    const double c = std::cos(ang), sn = std::sin(ang);
    re = (float)(wf[0] * c - wf[1] * sn);
    im = (float)(wf[0] * sn + wf[1] * c);
}

// Storage for the FP32 tables the unit kernel reads (every pointer holds the
// capacity for the filter's T, B): analysis window [T][B][B], synthesis
// window [B][B], and per gain slot [T][B/2+2][B] the sigma, the sigma of the
// Hermitian partner bin and the window spectrum (re, im).  sig_idx and
// sig2_idx (may be null) receive the (t, y, x) index of each slot's bin.
struct TableSpans {
    float* win;
    float* wsyn;
    float* sig;
    float* sig2;
    float* wfe;
    int* sig_idx;
    int* sig2_idx;
};

// Builds the tables from the plugin arrays (load_block's window,
// frequency_filtering's sigma, remove_mean's window_freq:
// cpu_source/getframe_impl.cpp:137, cpu_source/kernel.hpp:1826-1952).  The
// gain-slot layout is the column phase's: lane w = 2c + h of a block holds
// the y-bins k = 2m + h of packed x-column c; column 0 carries x-bins 0 (A)
// and B/2 (B).  `asym` reports a packed-column bin whose Hermitian partner
// has a different sigma; `wmask` has bit p set when temporal plane p of the
// window spectrum is not identically zero.
void build_tables(const dfttest2_b200_params* p, int B, int radius, bool zero_mean, int syn, const TableSpans& o,
                  bool& asym, int& wmask) {
    const int T = 2 * radius + 1, H = B / 2, X = H + 1, M = B / 2, NS = M + 2;
    for (int i = 0; i < T * B * B; ++i) o.win[i] = (float)p->window[i];
    for (int i = 0; i < B * B; ++i) o.wsyn[i] = o.win[syn * B * B + i];
    auto sigma_at = [&](int t, int y, int x) -> float {
        return p->sigma_len == 1 ? (float)p->sigma[0] : (float)p->sigma[(t * B + y) * X + x];
    };
    asym = false;
    auto put = [&](int pl, int j, int w, int t, int y, int x, int t2, int y2) {
        const int idx = (pl * NS + j) * B + w;
        if (o.sig_idx) o.sig_idx[idx] = (t * B + y) * X + x;
        if (o.sig2_idx) o.sig2_idx[idx] = (t2 * B + y2) * X + x;
        o.sig[idx] = sigma_at(t, y, x);
        o.sig2[idx] = sigma_at(t2, y2, x);
        o.wfe[2 * idx] = o.wfe[2 * idx + 1] = 0.0f;
        if (zero_mean)
            centre_first_wf(&p->window_freq[((t * B + y) * X + x) * 2], t, T, radius, o.wfe[2 * idx], o.wfe[2 * idx + 1]);
        if (o.sig2[idx] != o.sig[idx]) asym = true;
    };
    auto neg = [&](int k) { return (B - k) % B; };
    for (int pl = 0; pl < T; ++pl) {
        for (int w = 0; w < B; ++w) {
            const int c = w >> 1, h = w & 1;
            for (int j = 0; j < NS; ++j) put(pl, j, w, 0, 0, 0, 0, 0);  // unused slots
            if (c > 0) {
                for (int m = 0; m < M; ++m) put(pl, m, w, pl, 2 * m + h, c, pl, 2 * m + h);
                continue;
            }
            if (pl > 0) {
                for (int m = 0; m < M; ++m) {
                    const int k = 2 * m + h;
                    if (pl <= radius) put(pl, m, w, pl, k, 0, T - pl, neg(k));
                    else put(pl, m, w, T - pl, k, H, pl, neg(k));
                }
                continue;
            }
            // plane 0 of the packed column: untangled A (x-bin 0) and B (x-bin B/2)
            if (h == 0) {
                put(0, 0, w, 0, 0, 0, 0, 0);            // A(0)
                put(0, M / 2, w, 0, H, 0, 0, H);        // A(B/2)
                for (int m = 1; m < M / 2; ++m) {
                    put(0, m, w, 0, 2 * m, 0, 0, neg(2 * m));      // A(2m)
                    put(0, M - m, w, 0, 2 * m, H, 0, neg(2 * m));  // B(2m)
                }
                put(0, M, w, 0, 0, H, 0, 0);            // B(0)
                put(0, M + 1, w, 0, H, H, 0, H);        // B(B/2)
            } else {
                for (int m = 0; m < M / 2; ++m) {
                    put(0, m, w, 0, 2 * m + 1, 0, 0, neg(2 * m + 1));          // A(2m+1)
                    put(0, M - 1 - m, w, 0, 2 * m + 1, H, 0, neg(2 * m + 1));  // B(2m+1)
                }
            }
        }
    }
    // temporal planes whose window spectrum is identically zero skip the
    // zero-mean terms (every plane but 0 for a rectangular temporal window)
    wmask = 0;
    for (int pl = 0; pl < T; ++pl)
        for (int i = 0; i < NS * B * 2; ++i)
            if (o.wfe[pl * NS * B * 2 + i] != 0.0f) wmask |= 1 << pl;
}

// Text of the codes the kernels leave in their error word.
std::string kernel_error_text(int code) {
    switch (code) {
    case 1: return "kernel error 1: a unit's strip is wider than the kernel's blocks per step (planner inconsistency)";
    case 2: return "kernel error 2: a bounded wait for the tensor cores ran out (no completion signal within the limit)";
    case 3: return "kernel error 3: a bounds check of the checked build failed (index outside its buffer)";
    case 4: return "kernel error 4: a bounded wait for the TMA copies of input rows ran out";
    default: return "kernel error " + std::to_string(code);
    }
}

// Reads and clears a slot's error word after its stream has been waited for
// (the caller queued a copy of d_error into h_error before the wait).
int slot_status(Slot& s) {
    const int code = *s.h_error;
    if (code == 0) return 0;
    *s.h_error = 0;
    CUDA_TRY(cudaMemset(s.d_error, 0, sizeof(int)));
    return fail(DFTTEST2_B200_EKERNEL, kernel_error_text(code));
}

void scale_peak(int sample_type, int bits, float& scale, float& peak, int& kind) {
    if (sample_type == DFTTEST2_B200_FLOAT) {
        scale = 255.0f;
        peak = 1.0f;
        kind = dft2::kF32;
    } else {
        scale = 1.0f / (float)(1 << (bits - 8));
        peak = (float)((1 << bits) - 1);
        kind = bits <= 8 ? dft2::kU8 : dft2::kU16;
    }
}

void free_filter(dfttest2_b200_filter* f) {
    if (!f) return;
    DeviceGuard g(f->device);
    for (auto& e : f->cache) {
        if (e.d) cudaFree(e.d);
        if (e.ready) cudaEventDestroy(e.ready);
    }
    for (Slot& s : f->slots) {
        if (s.done) cudaEventSynchronize(s.done);
        if (s.d_jobs) cudaFree(s.d_jobs);
        if (s.d_scratch) cudaFree(s.d_scratch);
        if (s.d_seams) cudaFree(s.d_seams);
        if (s.d_tmaps) cudaFree(s.d_tmaps);
        if (s.d_error) cudaFree(s.d_error);
        if (s.h_error) cudaFreeHost(s.h_error);
        if (s.d_frames) cudaFree(s.d_frames);
        if (s.d_sigtab) cudaFree(s.d_sigtab);
        if (s.d_gjobs) cudaFree(s.d_gjobs);
        if (s.d_tcjobs) cudaFree(s.d_tcjobs);
        if (s.d_acc) cudaFree(s.d_acc);
        if (s.h_pinned) cudaFreeHost(s.h_pinned);
        if (s.stream) cudaStreamDestroy(s.stream);
        if (s.up) cudaStreamDestroy(s.up);
        if (s.down) cudaStreamDestroy(s.down);
        for (int k = 0; k < 2; ++k) {
            if (s.ev_up[k]) cudaEventDestroy(s.ev_up[k]);
            if (s.ev_comp[k]) cudaEventDestroy(s.ev_comp[k]);
            if (s.ev_down[k]) cudaEventDestroy(s.ev_down[k]);
        }
        if (s.done) cudaEventDestroy(s.done);
    }
    cudaFree(f->d_win);
    cudaFree(f->d_wsyn);
    cudaFree(f->d_sig);
    cudaFree(f->d_sig2);
    cudaFree(f->d_wfe);
    cudaFree(f->d_sigma_full);
    cudaFree(f->d_wf_full);
    cudaFree(f->d_sig_idx);
    cudaFree(f->d_sig2_idx);
    if (f->d_gmat) cudaFree(f->d_gmat);
    if (f->d_tc2) cudaFree(f->d_tc2);
    delete f;
}

template <typename Tp>
int upload(Tp*& dptr, const std::vector<Tp>& h) {
    CUDA_TRY(cudaMalloc((void**)&dptr, std::max<size_t>(h.size(), 1) * sizeof(Tp)));
    if (!h.empty()) CUDA_TRY(cudaMemcpy(dptr, h.data(), h.size() * sizeof(Tp), cudaMemcpyHostToDevice));
    return 0;
}

}  // namespace

extern "C" {

void dfttest2_b200_params_init(dfttest2_b200_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->radius = -1;
    p->block_size = -1;
    p->block_step = -1;
    p->zero_mean = -1;
    p->device_id = -1;
    p->num_streams = -1;
    p->synthesis_slice = -1;
}

int dfttest2_b200_create(const dfttest2_b200_params* p, dfttest2_b200_filter** out) {
    if (!out) return fail(DFTTEST2_B200_EINVAL, "null output handle");
    *out = nullptr;
    if (!p) return fail(DFTTEST2_B200_EINVAL, "null parameters");
    const int radius = p->radius < 0 ? 0 : p->radius;
    if (p->radius > 3) return fail(DFTTEST2_B200_EINVAL, "\"radius\" must be in [0, 1, 2, 3]");
    const int B = p->block_size < 0 ? 16 : p->block_size;
    if (B != 8 && B != 16 && B != 32) return fail(DFTTEST2_B200_EINVAL, "\"block_size\" must be 8, 16 or 32");
    const int S = p->block_step < 0 ? B : p->block_step;
    if (S < 1 || S > B) return fail(DFTTEST2_B200_EINVAL, "\"block_step\" must be in [1, block_size]");
    const int T = 2 * radius + 1, H = B / 2, X = H + 1;
    const int zero_mean = p->zero_mean < 0 ? 1 : !!p->zero_mean;
    const int device_id = p->device_id < 0 ? 0 : p->device_id;
    const int num_streams = p->num_streams < 0 ? 1 : p->num_streams;
    if (num_streams < 1) return fail(DFTTEST2_B200_EINVAL, "\"num_streams\" must be positive");
    if (p->filter_type < 0 || p->filter_type > 6) return fail(DFTTEST2_B200_EINVAL, "\"filter_type\" must be in [0, 6]");

    if (p->window_len != T * B * B || !p->window) return fail(DFTTEST2_B200_EINVAL, "invalid window size");
    if (p->sigma_len <= 0 || !p->sigma) return fail(DFTTEST2_B200_EINVAL, "sigma must not be empty");
    if (p->sigma_len != 1 && p->sigma_len != T * B * X) return fail(DFTTEST2_B200_EINVAL, "invalid sigma array size");
    if (zero_mean && (p->window_freq_len != T * B * X * 2 || !p->window_freq))
        return fail(DFTTEST2_B200_EINVAL, "invalid window_freq size");
    const int syn = p->synthesis_slice < 0 ? radius : p->synthesis_slice;
    if (syn >= T) return fail(DFTTEST2_B200_EINVAL, "\"synthesis_slice\" out of range");

    std::unique_ptr<dfttest2_b200_filter, void (*)(dfttest2_b200_filter*)> f(new dfttest2_b200_filter, free_filter);
    f->device = device_id;
    f->radius = radius;
    f->T = T;
    f->B = B;
    f->S = S;
    f->H = H;
    f->filter_type = p->filter_type;
    f->zero_mean = zero_mean;
    f->sigma2 = (float)p->sigma2;
    f->pmin = (float)p->pmin;
    f->pmax = (float)p->pmax;
    f->syn_slice = syn;
    f->var = select_variant(B, T, f->S);
    if (!f->var.main) return fail(DFTTEST2_B200_EINVAL, "unsupported block_size / radius");

    // -- tables --------------------------------------------------------------
    const int NS = B / 2 + 2;
    std::vector<float> win(T * B * B), wsyn(B * B), sig(T * NS * B), sig2(T * NS * B), wfe(2 * T * NS * B);
    std::vector<int> sig_idx(T * NS * B), sig2_idx(T * NS * B);
    bool asym = false;
    int wmask = 0;
    build_tables(p, B, radius, zero_mean, syn,
                 TableSpans{win.data(), wsyn.data(), sig.data(), sig2.data(), wfe.data(), sig_idx.data(),
                            sig2_idx.data()},
                 asym, wmask);
    auto sigma_at = [&](int t, int y, int x) -> float {
        return p->sigma_len == 1 ? (float)p->sigma[0] : (float)p->sigma[(t * B + y) * X + x];
    };
    f->wmask = wmask;
    f->asym = asym;
    f->h_win.assign(p->window, p->window + T * B * B);
    if (zero_mean) f->h_wf.assign(p->window_freq, p->window_freq + T * B * X * 2);
    f->h_sig.resize(T * B * X);
    for (int t = 0; t < T; ++t)
        for (int y = 0; y < B; ++y)
            for (int x = 0; x < X; ++x) f->h_sig[(t * B + y) * X + x] = sigma_at(t, y, x);
    f->g_div = zero_mean ? (float)p->window_freq[0] : 0.0f;
    if (zero_mean && f->g_div == 0.0f) return fail(DFTTEST2_B200_EINVAL, "window_freq[0] must be non-zero");

    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device_id >= ndev) return fail(DFTTEST2_B200_EINVAL, "invalid device_id");
    DeviceGuard dg(device_id);
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device_id));
    if (prop.major < 10) return fail(DFTTEST2_B200_EINVAL, "device is not sm_100 class");
    f->num_sms = prop.multiProcessorCount;

    if (int rc = upload(f->d_win, win)) return rc;
    if (int rc = upload(f->d_wsyn, wsyn)) return rc;
    if (int rc = upload(f->d_sig, sig)) return rc;
    if (int rc = upload(f->d_sig2, sig2)) return rc;
    if (int rc = upload(f->d_wfe, wfe)) return rc;
    {
        std::vector<float> sfull(T * B * X), wffull(2 * T * B * X, 0.0f);
        for (int t = 0; t < T; ++t)
            for (int y = 0; y < B; ++y)
                for (int x = 0; x < X; ++x) {
                    const int i = (t * B + y) * X + x;
                    sfull[i] = sigma_at(t, y, x);
                    // natural frame order (the adjoint and tensor-core kernels)
                    wffull[2 * i] = zero_mean ? (float)p->window_freq[2 * i] : 0.0f;
                    wffull[2 * i + 1] = zero_mean ? (float)p->window_freq[2 * i + 1] : 0.0f;
                }
        if (int rc = upload(f->d_sigma_full, sfull)) return rc;
        if (int rc = upload(f->d_wf_full, wffull)) return rc;
        if (int rc = upload(f->d_sig_idx, sig_idx)) return rc;
        if (int rc = upload(f->d_sig2_idx, sig2_idx)) return rc;
        f->n_slots = T * NS * B;
    }

    f->cache.reserve(64);  // entries are referenced outside the lock: never reallocate
    f->slots.resize(num_streams);
    for (int i = 0; i < num_streams; ++i) {
        Slot& s = f->slots[i];
        CUDA_TRY(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
        CUDA_TRY(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamCreateWithFlags(&s.up, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamCreateWithFlags(&s.down, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            CUDA_TRY(cudaEventCreateWithFlags(&s.ev_up[k], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&s.ev_comp[k], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&s.ev_down[k], cudaEventDisableTiming));
        }
        CUDA_TRY(cudaMalloc((void**)&s.d_error, sizeof(int)));
        CUDA_TRY(cudaMemset(s.d_error, 0, sizeof(int)));
        CUDA_TRY(cudaMallocHost((void**)&s.h_error, sizeof(int)));
        *s.h_error = 0;
        CUDA_TRY(cudaEventRecord(s.done, s.stream));
        f->free_slots.push_back(i);
    }
    CUDA_TRY(cudaDeviceSynchronize());
    *out = f.release();
    g_last_error.clear();
    return 0;
}

void dfttest2_b200_free(dfttest2_b200_filter* f) { free_filter(f); }

int dfttest2_b200_set_precision(dfttest2_b200_filter* f, int mode) {
    if (!f) return fail(DFTTEST2_B200_EINVAL, "null filter");
    if (mode < DFTTEST2_B200_FP32 || mode > DFTTEST2_B200_TC_FP16X3)
        return fail(DFTTEST2_B200_EINVAL, "unknown precision mode");
    DeviceGuard dg(f->device);
    // no launch of this filter may still read the old constants
    for (Slot& s : f->slots)
        if (s.done) CUDA_TRY(cudaEventSynchronize(s.done));
    f->tc_mode = 0;
    f->tc2 = Variant{};
    if (mode == DFTTEST2_B200_FP32) return 0;
    // the split-product modes run the strip form where the arguments allow it
    // (DFTTEST2_B200_TC_STRIP=0 keeps BF16X3 on the tile form)
    if (mode == DFTTEST2_B200_TC_FP16X3 || mode == DFTTEST2_B200_TC_BF16X3) {
        const char* env = std::getenv("DFTTEST2_B200_TC_STRIP");
        const bool allow = !(env && std::atoi(env) == 0) || mode == DFTTEST2_B200_TC_FP16X3;
        std::string why = "the tensor-core strip form needs block_size 16";
        const int fmt = mode == DFTTEST2_B200_TC_FP16X3 ? kTc2FmtFp16 : kTc2FmtBf16;
        std::vector<char> img;
        Tc2Shape shape;
        int rc = 1;
        if (f->asym) why = "the tensor-core strip form needs sigma symmetric in the x-bins 0 and B/2";
        else if (f->B == 16 && allow) {
            const Tc2Input in{f->T, f->S, f->radius, f->syn_slice, f->h_win.data(),
                              f->zero_mean ? f->h_wf.data() : nullptr, f->h_sig.data(), fmt};
            rc = tc2_build(in, img, shape, why);
        }
        if (rc == 0) {
            if (f->d_tc2) CUDA_TRY(cudaFree(f->d_tc2));
            f->d_tc2 = nullptr;
            CUDA_TRY(cudaMalloc((void**)&f->d_tc2, img.size()));
            CUDA_TRY(cudaMemcpy(f->d_tc2, img.data(), img.size(), cudaMemcpyHostToDevice));
            f->tc2 = tc2_variant(f->T, fmt, f->S);
            f->tc2_shape = shape;
            for (KernelFn k : {f->tc2.main, f->tc2.generic})
                CUDA_TRY(cudaFuncSetAttribute((const void*)k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
            f->tc_mode = mode;
            return 0;
        }
        if (mode == DFTTEST2_B200_TC_FP16X3) return fail(DFTTEST2_B200_EINVAL, why);
    }
    const TcVariant v = select_tc(f->B, f->T, mode);
    if (!v.wiener)
        return fail(DFTTEST2_B200_EINVAL,
                    "the tensor-core form supports block_size 16 with radius 0 or 1 and block_size 32 with radius 0");
    std::vector<char> img;
    v.build(img);
    if (f->d_gmat) CUDA_TRY(cudaFree(f->d_gmat));
    f->d_gmat = nullptr;
    CUDA_TRY(cudaMalloc(&f->d_gmat, img.size()));
    CUDA_TRY(cudaMemcpy(f->d_gmat, img.data(), img.size(), cudaMemcpyHostToDevice));
    f->gmat_bytes = (int)img.size();
    f->tc_mode = mode;
    return 0;
}

int dfttest2_b200_check(dfttest2_b200_filter* f) {
    if (!f) return fail(DFTTEST2_B200_EINVAL, "null filter");
    DeviceGuard dg(f->device);
    int first = 0;
    for (Slot& s : f->slots) {
        CUDA_TRY(cudaEventSynchronize(s.done));
        int code = 0;
        CUDA_TRY(cudaMemcpy(&code, s.d_error, sizeof(int), cudaMemcpyDeviceToHost));
        if (code != 0) {
            CUDA_TRY(cudaMemset(s.d_error, 0, sizeof(int)));
            if (!first) first = code;
        }
    }
    if (first) return fail(DFTTEST2_B200_EKERNEL, kernel_error_text(first));
    return 0;
}

int dfttest2_b200_set_wait_limit(dfttest2_b200_filter* f, int iterations) {
    if (!f) return fail(DFTTEST2_B200_EINVAL, "null filter");
    f->wait_limit = iterations < 0 ? dft2::kDefaultWaitLimit : iterations;
    return 0;
}

int dfttest2_b200_process_planes(dfttest2_b200_filter* f, const dfttest2_b200_plane* planes, int nplanes,
                                 int sample_type, int bits_per_sample, void* stream) {
    if (!f) return fail(DFTTEST2_B200_EINVAL, "null filter");
    if (nplanes < 0 || (nplanes > 0 && !planes)) return fail(DFTTEST2_B200_EINVAL, "invalid plane list");
    if (int rc = check_format(sample_type, bits_per_sample)) return rc;
    DeviceGuard dg(f->device);
    Plan plan;
    if (int rc = make_plan(f, planes, nplanes, bytes_of(sample_type, bits_per_sample), plan)) return rc;
    float scale, peak;
    int kind;
    scale_peak(sample_type, bits_per_sample, scale, peak, kind);
    SlotGuard sg(f);
    return launch(f, sg.slot(), plan, kind, scale, peak, (cudaStream_t)stream);
}

int dfttest2_b200_process_plane_host(dfttest2_b200_filter* f, const dfttest2_b200_plane* plane, int sample_type,
                                     int bits_per_sample) {
    if (!f || !plane) return fail(DFTTEST2_B200_EINVAL, "null argument");
    if (int rc = check_format(sample_type, bits_per_sample)) return rc;
    DeviceGuard dg(f->device);
    const int bps = bytes_of(sample_type, bits_per_sample);
    const size_t row = (size_t)plane->width * bps;
    const size_t frame = row * plane->height;
    const int T = f->T;
    SlotGuard sg(f);
    Slot& s = sg.slot();
    // T input planes + 1 output plane, densely packed
    if (int rc = ensure_bytes(s.d_frames, s.frames_cap, frame * (T + 1), s.done)) return rc;
    if (int rc = ensure_pinned(s.h_pinned, s.pinned_cap, frame * (T + 1), s.done)) return rc;
    CUDA_TRY(cudaEventSynchronize(s.done));
    uint8_t* h = (uint8_t*)s.h_pinned;
    for (int t = 0; t < T; ++t) {
        const uint8_t* src = (const uint8_t*)plane->src[t];
        if (!src) return fail(DFTTEST2_B200_EINVAL, "null source plane");
        for (int y = 0; y < plane->height; ++y) std::memcpy(h + t * frame + y * row, src + y * plane->src_stride, row);
    }
    CUDA_TRY(cudaMemcpyAsync(s.d_frames, h, frame * T, cudaMemcpyHostToDevice, s.stream));
    dfttest2_b200_plane dp{};
    for (int t = 0; t < T; ++t) dp.src[t] = (uint8_t*)s.d_frames + t * frame;
    dp.src_stride = row;
    dp.dst = (uint8_t*)s.d_frames + T * frame;
    dp.dst_stride = row;
    dp.width = plane->width;
    dp.height = plane->height;
    Plan plan;
    if (int rc = make_plan(f, &dp, 1, bps, plan)) return rc;
    float scale, peak;
    int kind;
    scale_peak(sample_type, bits_per_sample, scale, peak, kind);
    if (int rc = launch(f, s, plan, kind, scale, peak, s.stream)) return rc;
    CUDA_TRY(cudaMemcpyAsync(s.h_error, s.d_error, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
    CUDA_TRY(cudaMemcpyAsync(h + T * frame, dp.dst, frame, cudaMemcpyDeviceToHost, s.stream));
    CUDA_TRY(cudaEventRecord(s.done, s.stream));
    CUDA_TRY(cudaEventSynchronize(s.done));
    if (int rc = slot_status(s)) return rc;
    uint8_t* dst = (uint8_t*)plane->dst;
    for (int y = 0; y < plane->height; ++y) std::memcpy(dst + y * plane->dst_stride, h + T * frame + y * row, row);
    return 0;
}

int dfttest2_b200_process_frame_host_cached(dfttest2_b200_filter* f, const dfttest2_b200_plane* planes, int nplanes,
                                            const int* plane_indices, const int* src_frame_ids, int sample_type,
                                            int bits_per_sample) {
    if (!f || !planes || !plane_indices || !src_frame_ids) return fail(DFTTEST2_B200_EINVAL, "null argument");
    if (nplanes <= 0 || nplanes > 4) return fail(DFTTEST2_B200_EINVAL, "nplanes must be in [1, 4]");
    if (int rc = check_format(sample_type, bits_per_sample)) return rc;
    const int bps = bytes_of(sample_type, bits_per_sample);
    size_t row[4], frame[4], out_off[4], out_total = 0;
    for (int i = 0; i < nplanes; ++i) {
        const dfttest2_b200_plane& pl = planes[i];
        if (pl.width <= 0 || pl.height <= 0) return fail(DFTTEST2_B200_EINVAL, "invalid plane size");
        if (!pl.dst) return fail(DFTTEST2_B200_EINVAL, "null destination plane");
        row[i] = (size_t)pl.width * bps;
        frame[i] = row[i] * pl.height;
        if (pl.src_stride < (ptrdiff_t)row[i] || pl.dst_stride < (ptrdiff_t)row[i])
            return fail(DFTTEST2_B200_EINVAL, "invalid stride");
        for (int t = 0; t < f->T; ++t)
            if (!pl.src[t]) return fail(DFTTEST2_B200_EINVAL, "null source plane");
        out_off[i] = out_total;
        out_total += frame[i];
    }
    DeviceGuard dg(f->device);
    const int T = f->T;
    const size_t kMaxEntries = f->cache.capacity();
    SlotGuard sg(f);
    Slot& s = sg.slot();
    // device output planes; pinned staging with room for every upload of the call
    // (so that none waits for another) and for all downloads
    size_t up_total = 0;
    for (int i = 0; i < nplanes; ++i) up_total += frame[i] * T;
    if (int rc = ensure_bytes(s.d_frames, s.frames_cap, out_total, s.done)) return rc;
    if (int rc = ensure_pinned(s.h_pinned, s.pinned_cap, up_total + out_total, s.done)) return rc;
    CUDA_TRY(cudaEventSynchronize(s.done));
    uint8_t* h_up = (uint8_t*)s.h_pinned;
    uint8_t* h_down = h_up + up_total;
    size_t up_used = 0;

    int idx[4][7];
    int acquired[4] = {0, 0, 0, 0};
    int rc = 0;
    for (int i = 0; i < nplanes && rc == 0; ++i) {
        const dfttest2_b200_plane& pl = planes[i];
        for (int t = 0; t < T && rc == 0; ++t) {
            bool upload = false;
            {
                std::unique_lock<std::mutex> lk(f->cache_lock);
                // the cache first grows to a working set for several frames in flight
                // (4 planes x (2r+1 + 5) frames), then evicts the least recently used
                // free entry whose buffer already fits (reallocating synchronises the
                // device), else grows up to its limit, else evicts any free entry
                int hit = -1, fit = -1, any = -1;
                for (size_t k = 0; k < f->cache.size(); ++k) {
                    auto& e = f->cache[k];
                    if (e.id == src_frame_ids[t] && e.plane == plane_indices[i] && e.bytes == frame[i]) {
                        hit = (int)k;
                        break;
                    }
                    if (e.refs != 0) continue;
                    if (any < 0 || e.used < f->cache[any].used) any = (int)k;
                    if (e.cap >= frame[i] && (fit < 0 || e.used < f->cache[fit].used)) fit = (int)k;
                }
                const size_t working_set = std::min(kMaxEntries, (size_t)(4 * (T + 5)));
                int victim = f->cache.size() >= working_set ? fit : -1;
                if (hit >= 0) {
                    auto& e = f->cache[hit];
                    ++e.refs;
                    e.used = ++f->cache_clock;
                    // another call is queuing this upload: wait until its event is recorded
                    f->cache_cv.wait(lk, [&] { return f->cache[hit].issued; });
                    if (f->cache[hit].id != src_frame_ids[t]) {  // that upload failed
                        --e.refs;
                        rc = fail(DFTTEST2_B200_ECUDA, "a concurrent upload of this source plane failed");
                        break;
                    }
                    idx[i][t] = hit;
                } else {
                    if (victim < 0 && f->cache.size() < kMaxEntries) {
                        f->cache.emplace_back();
                        victim = (int)f->cache.size() - 1;
                    }
                    if (victim < 0) victim = any;
                    if (victim < 0) {
                        rc = fail(DFTTEST2_B200_ENOMEM, "frame cache exhausted (too many concurrent calls)");
                        break;
                    }
                    auto& e = f->cache[victim];
                    if (!e.ready && cudaEventCreateWithFlags(&e.ready, cudaEventDisableTiming) != cudaSuccess) {
                        rc = fail(DFTTEST2_B200_ECUDA, "event creation failed");
                        break;
                    }
                    if (e.cap < frame[i]) {
                        if (e.d) cudaFree(e.d);
                        e.d = nullptr;
                        e.cap = 0;
                        if (cudaMalloc(&e.d, frame[i]) != cudaSuccess) {
                            cudaGetLastError();
                            e.id = -1;
                            rc = fail(DFTTEST2_B200_ENOMEM, "device allocation failed");
                            break;
                        }
                        e.cap = frame[i];
                    }
                    e.id = src_frame_ids[t];
                    e.plane = plane_indices[i];
                    e.bytes = frame[i];
                    e.refs = 1;
                    e.issued = false;
                    e.used = ++f->cache_clock;
                    idx[i][t] = victim;
                    upload = true;
                }
            }
            ++acquired[i];
            auto& e = f->cache[idx[i][t]];
            if (upload) {
                const uint8_t* src = (const uint8_t*)pl.src[t];
                uint8_t* stage = h_up + up_used;  // this upload's own staging, in use until the call's final wait
                up_used += frame[i];
                for (int y = 0; y < pl.height; ++y) std::memcpy(stage + y * row[i], src + y * pl.src_stride, row[i]);
                cudaError_t ce = cudaMemcpyAsync(e.d, stage, frame[i], cudaMemcpyHostToDevice, s.stream);
                if (ce == cudaSuccess) ce = cudaEventRecord(e.ready, s.stream);
                {
                    std::lock_guard<std::mutex> lk(f->cache_lock);
                    if (ce != cudaSuccess) e.id = -1;  // never a hit
                    e.issued = true;
                }
                f->cache_cv.notify_all();
                if (ce != cudaSuccess) rc = fail(DFTTEST2_B200_ECUDA, std::string("upload failed: ") + cudaGetErrorString(ce));
            } else {
                if (cudaStreamWaitEvent(s.stream, e.ready, 0) != cudaSuccess) rc = fail(DFTTEST2_B200_ECUDA, "event wait failed");
            }
        }
    }
    if (rc == 0) {
        // every plane of the frame in one launch
        dfttest2_b200_plane dp[4];
        for (int i = 0; i < nplanes; ++i) {
            std::memset(&dp[i], 0, sizeof(dp[i]));
            for (int t = 0; t < T; ++t) dp[i].src[t] = f->cache[idx[i][t]].d;
            dp[i].src_stride = row[i];
            dp[i].dst = (uint8_t*)s.d_frames + out_off[i];
            dp[i].dst_stride = row[i];
            dp[i].width = planes[i].width;
            dp[i].height = planes[i].height;
        }
        Plan plan;
        float scale, peak;
        int kind;
        scale_peak(sample_type, bits_per_sample, scale, peak, kind);
        rc = make_plan(f, dp, nplanes, bps, plan);
        if (rc == 0) rc = launch(f, s, plan, kind, scale, peak, s.stream);
        if (rc == 0) {
            cudaError_t ce = cudaMemcpyAsync(s.h_error, s.d_error, sizeof(int), cudaMemcpyDeviceToHost, s.stream);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(h_down, s.d_frames, out_total, cudaMemcpyDeviceToHost, s.stream);
            if (ce == cudaSuccess) ce = cudaEventRecord(s.done, s.stream);
            if (ce == cudaSuccess) ce = cudaEventSynchronize(s.done);
            if (ce != cudaSuccess) rc = fail(DFTTEST2_B200_ECUDA, std::string("filtering failed: ") + cudaGetErrorString(ce));
            if (rc == 0) rc = slot_status(s);
        }
        if (rc == 0) {
            for (int i = 0; i < nplanes; ++i) {
                uint8_t* dst = (uint8_t*)planes[i].dst;
                const uint8_t* src = h_down + out_off[i];
                for (int y = 0; y < planes[i].height; ++y)
                    std::memcpy(dst + y * planes[i].dst_stride, src + y * row[i], row[i]);
            }
        }
    }
    // uploads queued by this call read its staging: on failure, let them finish first
    if (rc != 0) cudaStreamSynchronize(s.stream);
    {
        std::lock_guard<std::mutex> lk(f->cache_lock);
        for (int i = 0; i < nplanes; ++i)
            for (int t = 0; t < acquired[i]; ++t) --f->cache[idx[i][t]].refs;
    }
    return rc;
}

int dfttest2_b200_process_plane_host_cached(dfttest2_b200_filter* f, const dfttest2_b200_plane* plane,
                                            const int* src_frame_ids, int plane_index, int sample_type,
                                            int bits_per_sample) {
    if (!plane) return fail(DFTTEST2_B200_EINVAL, "null argument");
    return dfttest2_b200_process_frame_host_cached(f, plane, 1, &plane_index, src_frame_ids, sample_type,
                                                   bits_per_sample);
}

int dfttest2_b200_process_clip_planes_host(dfttest2_b200_filter* f, const dfttest2_b200_host_plane* hp, int nplanes,
                                           int nframes, int sample_type, int bits_per_sample) {
    if (!f || !hp || nplanes <= 0 || nframes <= 0) return fail(DFTTEST2_B200_EINVAL, "invalid argument");
    if (int rc = check_format(sample_type, bits_per_sample)) return rc;
    const int bps = bytes_of(sample_type, bits_per_sample);
    std::vector<size_t> row(nplanes), frame(nplanes), src_off(nplanes), out_off(nplanes);
    size_t src_total = 0, out_chunk = 0;
    for (int i = 0; i < nplanes; ++i) {
        if (!hp[i].src || !hp[i].dst || hp[i].width <= 0 || hp[i].height <= 0)
            return fail(DFTTEST2_B200_EINVAL, "invalid argument");
        row[i] = (size_t)hp[i].width * bps;
        frame[i] = row[i] * hp[i].height;
        src_off[i] = src_total;
        src_total += frame[i] * nframes;
        out_off[i] = out_chunk;
        out_chunk += frame[i];  // per output frame of the chunk
    }
    DeviceGuard dg(f->device);
    const int r = f->radius;
    SlotGuard sg(f);
    Slot& s = sg.slot();
    // Chunks of output frames ramp up (2, 6, 16) and down at the end (16, 6,
    // 2) so that the first upload and the last download, which nothing
    // overlaps, stay short; the frames between are split into equal chunks
    // of at most kMaxChunk.  Uploads (stream `up`), filtering of every plane's
    // frames of a chunk in one launch (slot stream) and downloads (stream
    // `down`) of consecutive chunks overlap; every source frame is uploaded
    // once into a dense device array; outputs alternate between two chunk
    // buffers, so chunk k starts after the download of chunk k - 2: each chunk
    // is at most about 3x the one before it (its upload hides behind that
    // one's filtering) and at least a third of the one two before it (the
    // download of that one hides behind the filtering of the one between; a
    // small remainder right after a 32-frame chunk stalled a 1080p clip by
    // 3 ms).
    constexpr int kMaxChunk = 32;
    std::vector<int> chunks;
    {
        static constexpr int kRamp[3] = {2, 6, 16};
        int left = nframes;
        for (int c : kRamp) {
            if (left <= 0) break;
            const int take = std::min(c, left);
            chunks.push_back(take);
            left -= take;
        }
        std::vector<int> tail;
        for (int c : kRamp) {  // the last chunks, smallest last
            if (left <= 0) break;
            const int take = std::min(c, left);
            tail.push_back(take);
            left -= take;
        }
        const int nmid = (left + kMaxChunk - 1) / kMaxChunk;
        for (int m = 0; m < nmid; ++m) chunks.push_back(left * (m + 1) / nmid - left * m / nmid);
        chunks.insert(chunks.end(), tail.rbegin(), tail.rend());
    }
    if (int rc = ensure_bytes(s.d_frames, s.frames_cap, src_total + 2 * kMaxChunk * out_chunk, s.done)) return rc;
    CUDA_TRY(cudaEventSynchronize(s.done));
    uint8_t* dsrc = (uint8_t*)s.d_frames;
    uint8_t* dout[2] = {dsrc + src_total, dsrc + src_total + kMaxChunk * out_chunk};
    float scale, peak;
    int kind;
    scale_peak(sample_type, bits_per_sample, scale, peak, kind);
    int uploaded = 0, c0 = 0;
    for (size_t k = 0; k < chunks.size(); ++k) {
        const int c1 = c0 + chunks[k];
        const int need = std::min(nframes, c1 + r);
        for (; uploaded < need; ++uploaded) {
            for (int i = 0; i < nplanes; ++i)
                CUDA_TRY(cudaMemcpy2DAsync(dsrc + src_off[i] + frame[i] * uploaded, row[i],
                                           (const uint8_t*)hp[i].src + hp[i].src_frame_bytes * uploaded,
                                           hp[i].src_stride, row[i], hp[i].height, cudaMemcpyHostToDevice, s.up));
        }
        CUDA_TRY(cudaEventRecord(s.ev_up[k & 1], s.up));
        uint8_t* ob = dout[k & 1];
        std::vector<dfttest2_b200_plane> planes;
        planes.reserve((size_t)(c1 - c0) * nplanes);
        for (int i = 0; i < nplanes; ++i) {
            for (int n = c0; n < c1; ++n) {
                dfttest2_b200_plane p;
                std::memset(&p, 0, sizeof(p));
                for (int t = 0; t < f->T; ++t) {
                    const int fi = std::min(std::max(n - r + t, 0), nframes - 1);
                    p.src[t] = dsrc + src_off[i] + frame[i] * fi;
                }
                p.src_stride = row[i];
                p.dst = ob + kMaxChunk * out_off[i] + frame[i] * (n - c0);
                p.dst_stride = row[i];
                p.width = hp[i].width;
                p.height = hp[i].height;
                planes.push_back(p);
            }
        }
        Plan plan;
        if (int rc = make_plan(f, planes.data(), (int)planes.size(), bps, plan)) return rc;
        CUDA_TRY(cudaStreamWaitEvent(s.stream, s.ev_up[k & 1], 0));
        if (k >= 2) CUDA_TRY(cudaStreamWaitEvent(s.stream, s.ev_down[k & 1], 0));  // output buffer free
        if (int rc = launch(f, s, plan, kind, scale, peak, s.stream)) return rc;
        CUDA_TRY(cudaEventRecord(s.ev_comp[k & 1], s.stream));
        CUDA_TRY(cudaStreamWaitEvent(s.down, s.ev_comp[k & 1], 0));
        for (int i = 0; i < nplanes; ++i)
            for (int n = c0; n < c1; ++n)
                CUDA_TRY(cudaMemcpy2DAsync((uint8_t*)hp[i].dst + hp[i].dst_frame_bytes * n, hp[i].dst_stride,
                                           ob + kMaxChunk * out_off[i] + frame[i] * (n - c0), row[i], row[i],
                                           hp[i].height, cudaMemcpyDeviceToHost, s.down));
        CUDA_TRY(cudaEventRecord(s.ev_down[k & 1], s.down));
        c0 = c1;
    }
    CUDA_TRY(cudaMemcpyAsync(s.h_error, s.d_error, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
    CUDA_TRY(cudaStreamSynchronize(s.down));
    CUDA_TRY(cudaStreamSynchronize(s.stream));
    CUDA_TRY(cudaEventRecord(s.done, s.stream));
    return slot_status(s);
}

int dfttest2_b200_process_clip_host(dfttest2_b200_filter* f, const void* src, ptrdiff_t src_stride,
                                    ptrdiff_t src_frame_bytes, void* dst, ptrdiff_t dst_stride,
                                    ptrdiff_t dst_frame_bytes, int nframes, int width, int height, int sample_type,
                                    int bits_per_sample) {
    if (!f || !src || !dst || nframes <= 0) return fail(DFTTEST2_B200_EINVAL, "invalid argument");
    dfttest2_b200_host_plane p;
    p.src = src;
    p.src_stride = src_stride;
    p.src_frame_bytes = src_frame_bytes;
    p.dst = dst;
    p.dst_stride = dst_stride;
    p.dst_frame_bytes = dst_frame_bytes;
    p.width = width;
    p.height = height;
    return dfttest2_b200_process_clip_planes_host(f, &p, 1, nframes, sample_type, bits_per_sample);
}

int dfttest2_b200_process_planes_sigma(dfttest2_b200_filter* f, const dfttest2_b200_plane* planes, int nplanes,
                                       int sample_type, int bits_per_sample, const float* sigma, void* stream) {
    if (!f) return fail(DFTTEST2_B200_EINVAL, "null filter");
    if (!sigma) return fail(DFTTEST2_B200_EINVAL, "null sigma");
    if (nplanes < 0 || (nplanes > 0 && !planes)) return fail(DFTTEST2_B200_EINVAL, "invalid plane list");
    if (int rc = check_format(sample_type, bits_per_sample)) return rc;
    DeviceGuard dg(f->device);
    Plan plan;
    if (int rc = make_plan(f, planes, nplanes, bytes_of(sample_type, bits_per_sample), plan)) return rc;
    float scale, peak;
    int kind;
    scale_peak(sample_type, bits_per_sample, scale, peak, kind);
    SlotGuard sg(f);
    Slot& s = sg.slot();
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaStreamWaitEvent(st, s.done, 0));
    if (int rc = ensure(s.d_sigtab, s.sigtab_cap, (size_t)2 * f->n_slots, s.done)) return rc;
    if (int rc = launch_sigma_tables(sigma, f->d_sig_idx, f->d_sig2_idx, s.d_sigtab, s.d_sigtab + f->n_slots,
                                     f->n_slots, st))
        return rc;
    return launch(f, s, plan, kind, scale, peak, st, s.d_sigtab, s.d_sigtab + f->n_slots);
}

int dfttest2_b200_backward_planes(dfttest2_b200_filter* f, const dfttest2_b200_grad_plane* planes, int nplanes,
                                  const float* sigma, float* grad_sigma, void* stream) {
    if (!f) return fail(DFTTEST2_B200_EINVAL, "null filter");
    if (nplanes < 0 || (nplanes > 0 && !planes)) return fail(DFTTEST2_B200_EINVAL, "invalid plane list");
    if (nplanes == 0) return 0;
    DeviceGuard dg(f->device);
    const int B = f->B, S = f->S, T = f->T;
    int tbx, tby;
    if (int rc = adjoint_tile_dims(B, T, tbx, tby)) return rc;
    std::vector<dft2::GradJob> jobs(nplanes);
    long long ntiles = 0;
    for (int i = 0; i < nplanes; ++i) {
        const dfttest2_b200_grad_plane& p = planes[i];
        const int pw = dft2::pad_size(p.width, B, S), ph = dft2::pad_size(p.height, B, S);
        const int ox = (pw - p.width) / 2, oy = (ph - p.height) / 2;
        if (p.width <= std::max(ox, pw - p.width - ox) || p.height <= std::max(oy, ph - p.height - oy))
            return fail(DFTTEST2_B200_EINVAL, "plane too small for the block size");
        if (!p.grad_dst) return fail(DFTTEST2_B200_EINVAL, "null output gradient");
        if (p.src_stride % 4 || p.grad_src_stride % 4 || p.grad_dst_stride % 4)
            return fail(DFTTEST2_B200_EINVAL, "invalid stride");
        dft2::GradJob& j = jobs[i];
        std::memset(&j, 0, sizeof(j));
        for (int t = 0; t < T; ++t) {
            if (!p.src[t] || !p.grad_src[t]) return fail(DFTTEST2_B200_EINVAL, "null source plane");
            j.src[t] = (const float*)p.src[t];
            j.gsrc[t] = p.grad_src[t];
        }
        j.gdst = p.grad_dst;
        j.src_stride = p.src_stride / 4;
        j.gsrc_stride = p.grad_src_stride / 4;
        j.gdst_stride = p.grad_dst_stride / 4;
        j.width = p.width;
        j.height = p.height;
        j.tile_base = (int)ntiles;
        j.ntx = (dft2::pad_num(p.width, B, S) + tbx - 1) / tbx;
        ntiles += (long long)j.ntx * ((dft2::pad_num(p.height, B, S) + tby - 1) / tby);
        if (ntiles > INT_MAX) return fail(DFTTEST2_B200_EINVAL, "too many planes in one call");
    }
    SlotGuard sg(f);
    Slot& s = sg.slot();
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaStreamWaitEvent(st, s.done, 0));
    if (int rc = ensure(s.d_gjobs, s.gjobs_cap, jobs.size(), s.done)) return rc;
    CUDA_TRY(cudaMemcpyAsync(s.d_gjobs, jobs.data(), jobs.size() * sizeof(dft2::GradJob), cudaMemcpyHostToDevice, st));
    dft2::AdjointArgs a{};
    a.jobs = s.d_gjobs;
    a.njobs = nplanes;
    a.ntiles = (int)ntiles;
    a.scale = 255.0f;
    a.block_step = S;
    a.filter_type = f->filter_type;
    a.sigma2 = f->sigma2;
    a.pmin = f->pmin;
    a.pmax = f->pmax;
    a.zero_mean = f->zero_mean ? 1 : 0;
    a.win = f->d_win;
    a.wsyn = f->d_wsyn;
    a.sigma = sigma ? sigma : f->d_sigma_full;
    a.wf = f->d_wf_full;
    a.gsigma = grad_sigma;
    if (int rc = launch_adjoint(B, T, a, f->num_sms, st)) return rc;
    CUDA_TRY(cudaEventRecord(s.done, st));
    return 0;
}

int dfttest2_b200_rdft(const double* data, int data_len, const int* shape, int ndim, double* out, int out_len) {
    if (ndim != 1 && ndim != 2 && ndim != 3)
        return fail(DFTTEST2_B200_EINVAL, "\"shape\" must be an array of ints with 1, 2 or 3 values");
    if (!data || !shape || !out) return fail(DFTTEST2_B200_EINVAL, "null argument");
    long long size = 1;
    for (int i = 0; i < ndim; ++i) {
        if (shape[i] <= 0) return fail(DFTTEST2_B200_EINVAL, "cannot reshape array");
        size *= shape[i];
    }
    if (size != data_len) return fail(DFTTEST2_B200_EINVAL, "cannot reshape array");
    const int nx = shape[ndim - 1], xo = nx / 2 + 1;
    long long outer = size / nx;
    if ((long long)out_len != outer * xo * 2) return fail(DFTTEST2_B200_EINVAL, "invalid output size");
    using C = std::complex<double>;
    const double pi = 3.14159265358979323846;
    // real last axis first, then the remaining axes from the innermost out
    std::vector<C> buf(outer * xo);
    for (long long o = 0; o < outer; ++o) {
        for (int k = 0; k < xo; ++k) {
            C sum = 0.0;
            for (int j = 0; j < nx; ++j) {
                const double ang = -2.0 * pi * (double)k * j / nx;
                sum += data[o * nx + j] * C(std::cos(ang), std::sin(ang));
            }
            buf[o * xo + k] = sum;
        }
    }
    long long inner = xo;  // stride of the axis being transformed
    for (int ax = ndim - 2; ax >= 0; --ax) {
        const int n = shape[ax];
        const long long block = inner * n;
        std::vector<C> tmp(buf.size());
        for (long long base = 0; base < (long long)buf.size(); base += block) {
            for (long long in = 0; in < inner; ++in) {
                for (int k = 0; k < n; ++k) {
                    C sum = 0.0;
                    for (int j = 0; j < n; ++j) {
                        const double ang = -2.0 * pi * (double)k * j / n;
                        sum += buf[base + j * inner + in] * C(std::cos(ang), std::sin(ang));
                    }
                    tmp[base + k * inner + in] = sum;
                }
            }
        }
        buf.swap(tmp);
        inner = block;
    }
    for (long long i = 0; i < outer * xo; ++i) {
        out[2 * i] = buf[i].real();
        out[2 * i + 1] = buf[i].imag();
    }
    return 0;
}

const char* dfttest2_b200_version(void) {
    return "dfttest2_b200 " DFTTEST2_B200_VERSION " (sm_100a; fused unit kernel, FP32 register codelets)";
}

const char* dfttest2_b200_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point (dfttest2_b200_process_plane_noalloc)
//
// For hosts that cannot allocate GPU memory: everything the kernels need
// besides the caller's planes (tables, the plane descriptor, the error flag
// and the per-unit overlap bands) is placed in one file-scope device array.
// In host code `g_noalloc_scratch` is only a stand-in symbol; its device
// address comes from cudaGetSymbolAddress, once per device.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocBytes = DFTTEST2_B200_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_lock;
unsigned char* g_noalloc_addr[kNoAllocMaxDevices] = {};

// device address of the array on the current device `dev` (set-up on first use)
int noalloc_address(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(DFTTEST2_B200_EINVAL, "invalid device_id");
    std::lock_guard<std::mutex> lk(g_noalloc_lock);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(DFTTEST2_B200_ECUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                                 cudaGetErrorString(e));
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_addr[dev];
    return 0;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Fixed-capacity host tables (T <= 7, B <= 32, about 97 KB): one buffer for
// the process, not the caller's stack (frame-server worker threads may have
// small stacks).  g_noalloc_tables_lock is held from the table build until the
// copies out of the buffer have been queued; copies from pageable memory are
// staged before cudaMemcpyAsync returns, so the next call may reuse it.
struct NoAllocTables {
    float win[7 * 32 * 32];
    float wsyn[32 * 32];
    float sig[7 * 18 * 32];
    float sig2[7 * 18 * 32];
    float wfe[2 * 7 * 18 * 32];
};
NoAllocTables g_noalloc_tables;
std::mutex g_noalloc_tables_lock;

// byte offset of the error word in the array
constexpr size_t kNoAllocErrorOffset = 0;

}  // namespace

extern "C" int dfttest2_b200_process_plane_noalloc(const dfttest2_b200_params* p, const dfttest2_b200_plane* plane,
                                                   int sample_type, int bits_per_sample, void* stream) {
    if (!p || !plane) return fail(DFTTEST2_B200_EINVAL, "null argument");
    // argument checks of DFTTestCreate (nvrtc_source/source.cpp:650-760)
    const int radius = p->radius < 0 ? 0 : p->radius;
    if (p->radius > 3) return fail(DFTTEST2_B200_EINVAL, "\"radius\" must be in [0, 1, 2, 3]");
    const int B = p->block_size < 0 ? 16 : p->block_size;
    if (B != 8 && B != 16 && B != 32) return fail(DFTTEST2_B200_EINVAL, "\"block_size\" must be 8, 16 or 32");
    const int S = p->block_step < 0 ? B : p->block_step;
    if (S < 1 || S > B) return fail(DFTTEST2_B200_EINVAL, "\"block_step\" must be in [1, block_size]");
    const int T = 2 * radius + 1, X = B / 2 + 1, NS = B / 2 + 2, O = B - S;
    const int zero_mean = p->zero_mean < 0 ? 1 : !!p->zero_mean;
    const int device_id = p->device_id < 0 ? 0 : p->device_id;
    if (p->filter_type < 0 || p->filter_type > 6) return fail(DFTTEST2_B200_EINVAL, "\"filter_type\" must be in [0, 6]");
    if (p->window_len != T * B * B || !p->window) return fail(DFTTEST2_B200_EINVAL, "invalid window size");
    if (p->sigma_len <= 0 || !p->sigma) return fail(DFTTEST2_B200_EINVAL, "sigma must not be empty");
    if (p->sigma_len != 1 && p->sigma_len != T * B * X) return fail(DFTTEST2_B200_EINVAL, "invalid sigma array size");
    if (zero_mean && (p->window_freq_len != T * B * X * 2 || !p->window_freq))
        return fail(DFTTEST2_B200_EINVAL, "invalid window_freq size");
    const int syn = p->synthesis_slice < 0 ? radius : p->synthesis_slice;
    if (syn >= T) return fail(DFTTEST2_B200_EINVAL, "\"synthesis_slice\" out of range");
    if (int rc = check_format(sample_type, bits_per_sample)) return rc;
    const Variant var = select_variant(B, T, S);
    if (!var.main) return fail(DFTTEST2_B200_EINVAL, "unsupported block_size / radius");

    const float g_div = zero_mean ? (float)p->window_freq[0] : 0.0f;
    if (zero_mean && g_div == 0.0f) return fail(DFTTEST2_B200_EINVAL, "window_freq[0] must be non-zero");

    // -- the plane and its unit split ------------------------------------------
    const int bps = bytes_of(sample_type, bits_per_sample);
    const int pw = dft2::pad_size(plane->width, B, S), ph = dft2::pad_size(plane->height, B, S);
    const int ox = (pw - plane->width) / 2, oy = (ph - plane->height) / 2;
    if (plane->width <= std::max(ox, pw - plane->width - ox) || plane->height <= std::max(oy, ph - plane->height - oy))
        return fail(DFTTEST2_B200_EINVAL, "plane too small for the block size");
    for (int t = 0; t < T; ++t)
        if (!plane->src[t]) return fail(DFTTEST2_B200_EINVAL, "null source plane");
    if (!plane->dst) return fail(DFTTEST2_B200_EINVAL, "null destination plane");
    if (plane->src_stride % bps || plane->dst_stride % bps || plane->src_stride < (ptrdiff_t)plane->width * bps ||
        plane->dst_stride < (ptrdiff_t)plane->width * bps)
        return fail(DFTTEST2_B200_EINVAL, "invalid stride");

    DeviceGuard dg(device_id);
    int dev = -1, num_sms = 148;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != device_id) return fail(DFTTEST2_B200_EINVAL, "invalid device_id");
    CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    {
        // the plane descriptor is copied from this call's stack frame and the tables from a
        // process-wide host buffer that the next call rewrites: a captured copy would read them
        // again at every replay, after the frame is gone and the buffer has changed
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        const cudaError_t e = cudaStreamIsCapturing((cudaStream_t)stream, &cs);
        if (e != cudaSuccess) cudaGetLastError();
        if (e != cudaSuccess || cs != cudaStreamCaptureStatusNone)
            return fail(DFTTEST2_B200_EINVAL,
                        "dfttest2_b200_process_plane_noalloc cannot run inside a stream capture (its table and "
                        "descriptor copies come from host memory that the call does not keep)");
    }

    const int BPS = strip_blocks(var, B, S);
    const int pnx = dft2::pad_num(plane->width, B, S), pny = dft2::pad_num(plane->height, B, S);
    bool narrow = false;
    const int nsx = strip_count(pnx, B, S, BPS, narrow);
    const int min_seg = std::max((O + S - 1) / S, 4);
    const size_t off_err = kNoAllocErrorOffset, off_job = 256;
    const size_t off_win = align256(off_job + sizeof(dft2::PlaneJob));
    const size_t off_wsyn = align256(off_win + sizeof(float) * T * B * B);
    const size_t off_sig = align256(off_wsyn + sizeof(float) * B * B);
    const size_t off_sig2 = align256(off_sig + sizeof(float) * T * NS * B);
    const size_t off_wfe = align256(off_sig2 + sizeof(float) * T * NS * B);
    const size_t off_band = align256(off_wfe + sizeof(float) * 2 * T * NS * B);
    auto band_bytes = [&](int nsy, int& rec) {
        const int wmax = (pnx + nsx - 1) / nsx, hmax = (pny + nsy - 1) / nsy;
        rec = std::max(dft2::band_record_size(wmax * S + O, hmax * S + O, O), 1);
        return sizeof(float) * (size_t)nsx * nsy * rec;
    };
    // as many segments as fill the GPU, fewer if the overlap bands must fit the array
    int nsy = std::max(1, std::min((4 * num_sms + nsx - 1) / nsx, pny / min_seg));
    int rec = 0;
    while (nsy > 1 && off_band + band_bytes(nsy, rec) > kNoAllocBytes) --nsy;
    const size_t need = off_band + band_bytes(nsy, rec);
    if (need > kNoAllocBytes)
        return fail(DFTTEST2_B200_EINVAL, "plane too large for the allocation-free path: needs " +
                                              std::to_string(need) + " bytes of scratch, the array holds " +
                                              std::to_string(kNoAllocBytes));

    dft2::PlaneJob job;
    std::memset(&job, 0, sizeof(job));
    for (int t = 0; t < 7; ++t) job.tmap[t] = -1;  // staged by plain loads
    for (int t = 0; t < T; ++t) job.src[t] = plane->src[t];
    job.dst = plane->dst;
    job.src_stride = plane->src_stride / bps;
    job.dst_stride = plane->dst_stride / bps;
    job.width = plane->width;
    job.height = plane->height;
    job.nsx = nsx;
    job.nsy = nsy;
    job.unit_base = 0;
    job.fix_base = 0;

    unsigned char* base = nullptr;
    if (int rc = noalloc_address(dev, &base)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    bool asym = false;
    int wmask = 0;
    {
        // tables as dfttest2_b200_create builds them, in the process-wide host
        // buffer; the error word must start at zero; tables and descriptor are
        // copied in (pageable sources are staged before these calls return)
        std::lock_guard<std::mutex> lk(g_noalloc_tables_lock);
        NoAllocTables& tb = g_noalloc_tables;
        build_tables(p, B, radius, zero_mean, syn, TableSpans{tb.win, tb.wsyn, tb.sig, tb.sig2, tb.wfe, nullptr, nullptr},
                     asym, wmask);
        CUDA_TRY(cudaMemsetAsync(base + off_err, 0, sizeof(int), st));
        CUDA_TRY(cudaMemcpyAsync(base + off_job, &job, sizeof(job), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(base + off_win, tb.win, sizeof(float) * T * B * B, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(base + off_wsyn, tb.wsyn, sizeof(float) * B * B, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(base + off_sig, tb.sig, sizeof(float) * T * NS * B, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(base + off_sig2, tb.sig2, sizeof(float) * T * NS * B, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(base + off_wfe, tb.wfe, sizeof(float) * 2 * T * NS * B, cudaMemcpyHostToDevice, st));
    }

    float scale, peak;
    int kind;
    scale_peak(sample_type, bits_per_sample, scale, peak, kind);
    dft2::KernelArgs a{};
    a.jobs = reinterpret_cast<const dft2::PlaneJob*>(base + off_job);
    a.njobs = 1;
    a.nunits = nsx * nsy;
    a.nfix = (nsx - 1) * O * plane->height + (nsy - 1) * O * plane->width;
    a.p.kind = kind;
    a.p.scale = scale;
    a.p.peak = peak;
    a.block_step = S;
    a.p.filter_type = p->filter_type;
    a.p.sigma2 = (float)p->sigma2;
    a.p.pmin = (float)p->pmin;
    a.p.pmax = (float)p->pmax;
    a.p.g_div = g_div;
    a.p.win = reinterpret_cast<const float*>(base + off_win);
    a.p.wsyn = reinterpret_cast<const float*>(base + off_wsyn);
    a.p.sig = reinterpret_cast<const float*>(base + off_sig);
    a.p.sig2 = asym ? reinterpret_cast<const float*>(base + off_sig2) : nullptr;
    a.p.wfe = reinterpret_cast<const float*>(base + off_wfe);
    a.p.wmask = zero_mean ? wmask : 0;
    a.scratch = reinterpret_cast<float*>(base + off_band);
    a.rec_stride = rec;
    a.ring_pitch = ((BPS * S + O) + 3) & ~3;
    a.error_flag = reinterpret_cast<int*>(base + off_err);

    const size_t smem = var.smem(a.ring_pitch);
    KernelFn kern = (p->filter_type == 0 && !asym) ? var.main : var.generic;
    if (int rc = prepare_kernel((const void*)kern, smem, var.nw * 32, nullptr)) return rc;
    kern<<<a.nunits, var.nw * 32, smem, st>>>(a);
    CUDA_TRY(cudaGetLastError());
    if (a.nfix > 0) {
        const int threads = 256;
        const int blocks = std::min((a.nfix + threads - 1) / threads, num_sms * 8);
        var.fixup<<<blocks, threads, 0, st>>>(a);
        CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

extern "C" int dfttest2_b200_noalloc_check(int device_id, void* stream) {
    const int dev_id = device_id < 0 ? 0 : device_id;
    DeviceGuard dg(dev_id);
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != dev_id) return fail(DFTTEST2_B200_EINVAL, "invalid device_id");
    unsigned char* base = nullptr;
    if (int rc = noalloc_address(dev, &base)) return rc;
    CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    int code = 0;
    CUDA_TRY(cudaMemcpy(&code, base + kNoAllocErrorOffset, sizeof(int), cudaMemcpyDeviceToHost));
    if (code != 0) return fail(DFTTEST2_B200_EKERNEL, kernel_error_text(code));
    return 0;
}

#include "dfttest_batch.cuh"
