// Multi-clip batches: work-lists of plane jobs with per-job formats and
// filters, grouped by kernel, tuned on the batch itself and captured into one
// CUDA graph.  Included at the end of dfttest_capi.cu (same translation unit:
// it uses the planning and launch helpers there).
//
// The reference has no batch: each DFTTest instance filters one clip, one
// frame per DFTTestGetFrame call (nvrtc_source/source.cpp:356-605), and its
// runtime specialisation cache keys compiled kernels by their parameters
// (hiprtc_source/source.cpp:248-309).  Here every kernel shape is compiled
// ahead of time for sm_100a; what is chosen per batch is the shape and the
// unit split of every group.
#pragma once

struct dfttest2_b200_batch {
    struct Group {
        int B = 16, S = 16, T = 1;
        bool generic = false;
        std::vector<PlaneRef> planes;  // cost-ordered work-list
        long long blocks = 0;          // blocks per run (all planes)
        std::vector<Variant> cands;
        int var_idx = 0;
        int target_mult = 4;           // units ~ target_mult x SMs
        Plan plan;
        dft2::PlaneJob* d_jobs = nullptr;
        float* d_scratch = nullptr;
        int* d_seams = nullptr;        // seam counters when every unit is a full-height strip
        void* d_tmaps = nullptr;       // tensor maps of the TMA row staging (null: plain loads)
        int stage_bw = 0;
        size_t smem = 0;               // dynamic shared memory of the group's launch
        std::string trials;            // "shape:ms ..." of the tuning runs
        bool cached = false;
    };
    int device = 0;
    int num_sms = 148;
    std::vector<Group> groups;
    std::vector<int> kinds;            // sample format per clip (FilterParams index)
    dft2::FilterParams* d_params = nullptr;
    int* d_error = nullptr;
    cudaStream_t cap = nullptr;        // capture origin
    std::vector<cudaStream_t> branch;  // one per group
    std::vector<cudaEvent_t> ev;       // fork + one join per group
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

std::mutex g_tune_lock;
std::vector<std::pair<std::string, std::pair<int, int>>> g_tune_cache;  // signature -> (variant, target)

void free_batch(dfttest2_b200_batch* b) {
    if (!b) return;
    DeviceGuard g(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto& gr : b->groups) {
        if (gr.d_jobs) cudaFree(gr.d_jobs);
        if (gr.d_scratch) cudaFree(gr.d_scratch);
        if (gr.d_seams) cudaFree(gr.d_seams);
        if (gr.d_tmaps) cudaFree(gr.d_tmaps);
    }
    for (cudaStream_t s : b->branch) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->d_params) cudaFree(b->d_params);
    if (b->d_error) cudaFree(b->d_error);
    delete b;
}

int launch_group(const dfttest2_b200_batch* b, const dfttest2_b200_batch::Group& g, cudaStream_t st) {
    const Variant& var = g.cands[g.var_idx];
    dft2::KernelArgs a{};
    a.jobs = g.d_jobs;
    a.njobs = (int)g.plan.jobs.size();
    a.nunits = g.plan.nunits;
    a.nfix = g.plan.nfix;
    a.block_step = g.S;
    a.params = b->d_params;
    a.scratch = g.d_scratch;
    a.rec_stride = g.plan.rec_stride;
    a.ring_pitch = g.plan.pitch;
    a.error_flag = b->d_error;
    if (g.d_seams) {  // full-height strips: seams summed in the unit kernel
        CUDA_TRY(cudaMemsetAsync(g.d_seams, 0, (size_t)g.plan.nseams * sizeof(int), st));
        a.seam_count = g.d_seams;
    }
    if (g.d_tmaps) {
        a.tmaps = g.d_tmaps;
        a.stage_bw = g.stage_bw;
        a.stage_off = (int)((var.smem(g.plan.pitch) + 127) & ~(size_t)127);
    }
    KernelFn kern = g.generic ? var.generic : var.main;
    kern<<<g.plan.nunits, var.nw * 32, g.smem, st>>>(a);
    CUDA_TRY(cudaGetLastError());
    if (g.plan.nfix > 0 && !g.d_seams) {
        const int threads = 256;
        const int blocks = std::min((g.plan.nfix + threads - 1) / threads, b->num_sms * 8);
        var.fixup<<<blocks, threads, 0, st>>>(a);
        CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

// plan a group for (variant, target), size its buffers and upload its work-list
int prepare_group(dfttest2_b200_batch* b, dfttest2_b200_batch::Group& g, int var_idx, int target_mult) {
    const Variant& var = g.cands[var_idx];
    g.var_idx = var_idx;
    g.target_mult = target_mult;
    if (int rc = plan_units(g.B, g.S, strip_blocks(var, g.B, g.S), g.planes, (long long)target_mult * b->num_sms,
                            g.plan))
        return rc;
    size_t smem = var.smem(g.plan.pitch);
    if (smem > 227 * 1024) return fail(DFTTEST2_B200_EINVAL, "block step too large for the kernel's shared memory");
    // TMA staging of the input rows where the planes allow it
    std::vector<int> kinds(g.plan.jobs.size());
    for (size_t i = 0; i < kinds.size(); ++i) kinds[i] = b->kinds[g.plan.jobs[i].param];
    std::vector<CUtensorMap> maps;
    size_t stage = 0;
    build_stage_maps(g.plan.jobs, kinds, g.B, g.S, g.T, g.plan.pitch, maps, g.stage_bw, stage);
    if (g.stage_bw > 0 && ((smem + 127) & ~(size_t)127) + stage <= 227 * 1024) {
        smem = ((smem + 127) & ~(size_t)127) + stage;
    } else {
        g.stage_bw = 0;
        maps.clear();
        for (auto& j : g.plan.jobs)
            for (int t = 0; t < 7; ++t) j.tmap[t] = -1;
    }
    g.smem = smem;
    KernelFn kern = g.generic ? var.generic : var.main;
    if (int rc = prepare_kernel((const void*)kern, smem, var.nw * 32, nullptr)) return rc;
    if (g.d_jobs) CUDA_TRY(cudaFree(g.d_jobs));
    if (g.d_scratch) CUDA_TRY(cudaFree(g.d_scratch));
    if (g.d_seams) CUDA_TRY(cudaFree(g.d_seams));
    if (g.d_tmaps) CUDA_TRY(cudaFree(g.d_tmaps));
    g.d_jobs = nullptr;
    g.d_scratch = nullptr;
    g.d_seams = nullptr;
    g.d_tmaps = nullptr;
    if (!maps.empty()) {
        CUDA_TRY(cudaMalloc(&g.d_tmaps, maps.size() * sizeof(CUtensorMap)));
        CUDA_TRY(cudaMemcpy(g.d_tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    }
    if (g.plan.nfix > 0 && g.plan.full_strips && g.plan.nseams > 0)
        CUDA_TRY(cudaMalloc((void**)&g.d_seams, (size_t)g.plan.nseams * sizeof(int)));
    CUDA_TRY(cudaMalloc((void**)&g.d_jobs, g.plan.jobs.size() * sizeof(dft2::PlaneJob)));
    CUDA_TRY(cudaMalloc((void**)&g.d_scratch, (size_t)g.plan.nunits * g.plan.rec_stride * sizeof(float)));
    CUDA_TRY(cudaMemcpy(g.d_jobs, g.plan.jobs.data(), g.plan.jobs.size() * sizeof(dft2::PlaneJob),
                        cudaMemcpyHostToDevice));
    return 0;
}

std::string group_signature(const dfttest2_b200_batch::Group& g, int num_sms) {
    // kernel and the multiset of plane sizes decide the best shape
    std::vector<std::pair<int, int>> dims;
    for (const PlaneRef& p : g.planes) dims.emplace_back(p.width, p.height);
    std::sort(dims.begin(), dims.end());
    std::string s = std::to_string(g.B) + "/" + std::to_string(g.S) + "/" + std::to_string(g.T) + "/" +
                    (g.generic ? "g" : "w") + "/" + std::to_string(num_sms) + ":";
    for (size_t i = 0; i < dims.size();) {
        size_t j = i;
        while (j < dims.size() && dims[j] == dims[i]) ++j;
        s += std::to_string(dims[i].first) + "x" + std::to_string(dims[i].second) + "*" + std::to_string(j - i) + ",";
        i = j;
    }
    return s;
}

// time every candidate (shape x unit target) on the batch itself; keep the fastest
int tune_group(dfttest2_b200_batch* b, dfttest2_b200_batch::Group& g, cudaStream_t st) {
    static const int kTargets[] = {2, 4, 8, 16};
    const std::string sig = group_signature(g, b->num_sms);
    {
        std::lock_guard<std::mutex> lk(g_tune_lock);
        for (const auto& e : g_tune_cache)
            if (e.first == sig) {
                g.cached = true;
                return prepare_group(b, g, e.second.first, e.second.second);
            }
    }
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_v = 0, best_t = 4;
    int last_units = -1, last_v = -1;
    int rc = 0;
    for (int v = 0; v < (int)g.cands.size() && rc == 0; ++v) {
        for (int t : kTargets) {
            if ((rc = prepare_group(b, g, v, t)) != 0) {
                if (v > 0 && rc == DFTTEST2_B200_EINVAL) rc = 0;  // an alternative shape that cannot split these planes
                break;
            }
            if (v == last_v && g.plan.nunits == last_units) continue;  // same split as the previous target
            last_v = v;
            last_units = g.plan.nunits;
            const int reps = 3;
            if ((rc = launch_group(b, g, st)) != 0) break;  // warm-up
            if (cudaEventRecord(e0, st) != cudaSuccess) { rc = fail(DFTTEST2_B200_ECUDA, "event record failed"); break; }
            for (int r = 0; r < reps && rc == 0; ++r) rc = launch_group(b, g, st);
            if (rc) break;
            if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
                rc = fail(DFTTEST2_B200_ECUDA, "tuning run failed");
                break;
            }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= reps;
            char buf[96];
            std::snprintf(buf, sizeof buf, "%dw/%dx:%.3fms ", g.cands[v].nw, t, ms);
            g.trials += buf;
            if (ms < best) {
                best = ms;
                best_v = v;
                best_t = t;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(g_tune_lock);
        g_tune_cache.emplace_back(sig, std::make_pair(best_v, best_t));
    }
    return prepare_group(b, g, best_v, best_t);
}

}  // namespace

extern "C" {

int dfttest2_b200_batch_create(const dfttest2_b200_clip* clips, int nclips, int flags, dfttest2_b200_batch** out) {
    if (!out) return fail(DFTTEST2_B200_EINVAL, "null output");
    *out = nullptr;
    if (nclips <= 0 || !clips) return fail(DFTTEST2_B200_EINVAL, "empty clip list");
    const int device = clips[0].filter ? clips[0].filter->device : 0;
    std::vector<dft2::FilterParams> params(nclips);
    std::unique_ptr<dfttest2_b200_batch, void (*)(dfttest2_b200_batch*)> b(new dfttest2_b200_batch, free_batch);
    b->device = device;
    for (int c = 0; c < nclips; ++c) {
        const dfttest2_b200_clip& k = clips[c];
        const dfttest2_b200_filter* f = k.filter;
        if (!f) return fail(DFTTEST2_B200_EINVAL, "clip " + std::to_string(c) + ": null filter");
        if (f->device != device) return fail(DFTTEST2_B200_EINVAL, "all clips of a batch must be on one device");
        if (int rc = check_format(k.sample_type, k.bits_per_sample)) return rc;
        const int bps = bytes_of(k.sample_type, k.bits_per_sample);
        if (k.nframes <= 0 || !k.src || !k.dst)
            return fail(DFTTEST2_B200_EINVAL, "clip " + std::to_string(c) + ": no frames");
        if (!plane_fits(k.width, k.height, f->B, f->S))
            return fail(DFTTEST2_B200_EINVAL, "clip " + std::to_string(c) + ": plane too small for the block size");
        if (k.src_stride % bps || k.dst_stride % bps || k.src_stride < (ptrdiff_t)k.width * bps ||
            k.dst_stride < (ptrdiff_t)k.width * bps || k.src_frame_bytes < k.src_stride * k.height ||
            k.dst_frame_bytes < k.dst_stride * k.height)
            return fail(DFTTEST2_B200_EINVAL, "clip " + std::to_string(c) + ": invalid stride");
        float scale, peak;
        int kind;
        scale_peak(k.sample_type, k.bits_per_sample, scale, peak, kind);
        dft2::FilterParams& p = params[c];
        std::memset(&p, 0, sizeof(p));
        p.kind = kind;
        b->kinds.push_back(kind);
        p.scale = scale;
        p.peak = peak;
        p.filter_type = f->filter_type;
        p.sigma2 = f->sigma2;
        p.pmin = f->pmin;
        p.pmax = f->pmax;
        p.g_div = f->zero_mean ? f->g_div : 0.0f;
        p.win = f->d_win;
        p.wsyn = f->d_wsyn;
        p.sig = f->d_sig;
        p.sig2 = f->asym ? f->d_sig2 : nullptr;
        p.wfe = f->d_wfe;
        p.wmask = f->zero_mean ? f->wmask : 0;

        const bool generic = !(f->filter_type == 0 && !f->asym);
        dfttest2_b200_batch::Group* g = nullptr;
        for (auto& gr : b->groups)
            if (gr.B == f->B && gr.S == f->S && gr.T == f->T && gr.generic == generic) g = &gr;
        if (!g) {
            b->groups.emplace_back();
            g = &b->groups.back();
            g->B = f->B;
            g->S = f->S;
            g->T = f->T;
            g->generic = generic;
            g->cands = candidate_variants(f->B, f->T, f->S);
            if (g->cands.empty()) return fail(DFTTEST2_B200_EINVAL, "unsupported block_size / radius");
        }
        const int r = f->radius;
        const char* src = static_cast<const char*>(k.src);
        char* dst = static_cast<char*>(k.dst);
        for (int n = 0; n < k.nframes; ++n) {
            PlaneRef pr;
            std::memset(&pr, 0, sizeof(pr));
            for (int t = 0; t < f->T; ++t) {
                const int fi = std::min(std::max(n - r + t, 0), k.nframes - 1);
                pr.src[t] = src + (ptrdiff_t)fi * k.src_frame_bytes;
            }
            pr.dst = dst + (ptrdiff_t)n * k.dst_frame_bytes;
            pr.src_stride = k.src_stride / bps;
            pr.dst_stride = k.dst_stride / bps;
            pr.width = k.width;
            pr.height = k.height;
            pr.param = c;
            g->planes.push_back(pr);
            g->blocks += (long long)dft2::pad_num(k.width, f->B, f->S) * dft2::pad_num(k.height, f->B, f->S);
        }
    }
    // largest planes first, so that the block scheduler ends on small units
    for (auto& g : b->groups)
        std::stable_sort(g.planes.begin(), g.planes.end(), [](const PlaneRef& x, const PlaneRef& y) {
            return (long long)x.width * x.height > (long long)y.width * y.height;
        });
    // biggest groups first in the graph
    std::stable_sort(b->groups.begin(), b->groups.end(),
                     [](const dfttest2_b200_batch::Group& x, const dfttest2_b200_batch::Group& y) {
                         return x.blocks * x.T > y.blocks * y.T;
                     });

    DeviceGuard dg(device);
    b->num_sms = clips[0].filter->num_sms;
    CUDA_TRY(cudaMalloc((void**)&b->d_params, params.size() * sizeof(dft2::FilterParams)));
    CUDA_TRY(cudaMemcpy(b->d_params, params.data(), params.size() * sizeof(dft2::FilterParams),
                        cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMalloc((void**)&b->d_error, sizeof(int)));
    CUDA_TRY(cudaMemset(b->d_error, 0, sizeof(int)));
    CUDA_TRY(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    for (auto& g : b->groups) {
        if (flags & DFTTEST2_B200_BATCH_TUNE) {
            if (int rc = tune_group(b.get(), g, b->cap)) return rc;
        } else {
            if (int rc = prepare_group(b.get(), g, 0, 4)) return rc;
        }
    }
    CUDA_TRY(cudaStreamSynchronize(b->cap));
    int err = 0;
    CUDA_TRY(cudaMemcpy(&err, b->d_error, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(DFTTEST2_B200_EKERNEL, "kernel consistency check failed while tuning");

    // the graph: fork from the origin stream, one branch per group, join
    const int ng = (int)b->groups.size();
    b->branch.resize(ng);
    b->ev.resize(ng + 1);
    for (int i = 0; i < ng; ++i) CUDA_TRY(cudaStreamCreateWithFlags(&b->branch[i], cudaStreamNonBlocking));
    for (int i = 0; i <= ng; ++i) CUDA_TRY(cudaEventCreateWithFlags(&b->ev[i], cudaEventDisableTiming));
    CUDA_TRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    if (cudaEventRecord(b->ev[0], b->cap) != cudaSuccess) rc = fail(DFTTEST2_B200_ECUDA, "graph fork failed");
    for (int i = 0; i < ng && rc == 0; ++i) {
        if (cudaStreamWaitEvent(b->branch[i], b->ev[0], 0) != cudaSuccess) {
            rc = fail(DFTTEST2_B200_ECUDA, "graph fork failed");
            break;
        }
        if ((rc = launch_group(b.get(), b->groups[i], b->branch[i])) != 0) break;
        if (cudaEventRecord(b->ev[i + 1], b->branch[i]) != cudaSuccess ||
            cudaStreamWaitEvent(b->cap, b->ev[i + 1], 0) != cudaSuccess)
            rc = fail(DFTTEST2_B200_ECUDA, "graph join failed");
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(b->cap, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    CUDA_TRY(ce);
    b->graph = graph;
    CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    *out = b.release();
    return 0;
}

int dfttest2_b200_batch_run(dfttest2_b200_batch* b, void* stream) {
    if (!b) return fail(DFTTEST2_B200_EINVAL, "null batch");
    DeviceGuard dg(b->device);
    CUDA_TRY(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
    return 0;
}

int dfttest2_b200_batch_describe(const dfttest2_b200_batch* b, char* buf, int len) {
    if (!b) return -fail(DFTTEST2_B200_EINVAL, "null batch");
    std::string s;
    int launches = 0;
    for (const auto& g : b->groups) {
        const Variant& v = g.cands[g.var_idx];
        char line[256];
        std::snprintf(line, sizeof line, "B%d S%d T%d %s: %d warps x %d units, %zu jobs, %lld blocks, %s %d%s | ",
                      g.B, g.S, g.T, g.generic ? "general" : "wiener", v.nw, g.plan.nunits, g.plan.jobs.size(),
                      g.blocks, g.d_seams ? "in-kernel seams" : "fixup", g.plan.nfix, g.cached ? ", cached" : "");
        s += line;
        s += g.trials.empty() ? "untuned" : g.trials;
        s += "\n";
        launches += 1 + (g.plan.nfix > 0 && !g.d_seams ? 1 : 0);
    }
    if (buf && len > 0) {
        const size_t n = std::min(s.size(), (size_t)len - 1);
        std::memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    return launches;
}

void dfttest2_b200_batch_free(dfttest2_b200_batch* b) { free_batch(b); }

}  // extern "C"
