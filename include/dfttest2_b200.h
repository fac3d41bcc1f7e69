/*
 * dfttest2_b200 -- C ABI of the B200 (sm_100a) DFTTest per-plane hot path.
 *
 * The entry points replace the VapourSynth plugin functions of the
 * reference's GPU backends (vs-dfttest2):
 *
 *   DFTTest  -> dfttest2_b200_create / dfttest2_b200_process_* / dfttest2_b200_free
 *               (nvrtc_source/source.cpp:629-858 DFTTestCreate,
 *                nvrtc_source/source.cpp:356-605 DFTTestGetFrame,
 *                nvrtc_source/source.cpp:607-627 DFTTestFree,
 *                signature registered at nvrtc_source/source.cpp:951-972)
 *   RDFT     -> dfttest2_b200_rdft   (nvrtc_source/source.cpp:862-933,
 *                                      cpu_source/source.cpp:269-340)
 *   Version  -> dfttest2_b200_version (nvrtc_source/source.cpp:935-938)
 *
 * Only plain C types cross this boundary.  Every function that can fail
 * returns 0 on success and a non-zero status otherwise; the message is
 * available from dfttest2_b200_last_error() (thread-local) and uses the
 * reference's wording where the reference has one.
 *
 * Array layouts are those of the plugin arguments: row-major (t, y, x),
 * t in [0, 2*radius], y in [0, block_size), x in [0, block_size) for the
 * window and x in [0, block_size/2] for sigma / window_freq; window_freq
 * interleaves (re, im).
 */
#ifndef DFTTEST2_B200_H
#define DFTTEST2_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DFTTEST2_B200_OK 0
#define DFTTEST2_B200_EINVAL 1   /* invalid argument (same checks as the reference's Create) */
#define DFTTEST2_B200_ECUDA 2    /* CUDA runtime error */
#define DFTTEST2_B200_ENOMEM 3   /* allocation failure */
#define DFTTEST2_B200_EKERNEL 4  /* the kernel reported an internal consistency failure */

/* sample types, as VapourSynth's stInteger / stFloat */
#define DFTTEST2_B200_INTEGER 0
#define DFTTEST2_B200_FLOAT 1

typedef struct dfttest2_b200_filter dfttest2_b200_filter;

/* Arguments of DFTTest (nvrtc_source/source.cpp:951-972).  Integer options
 * that the reference marks ":opt" take their reference default when set to
 * -1 (radius 0, block_size 16, block_step block_size, zero_mean 1,
 * device_id 0, num_streams 1). */
typedef struct dfttest2_b200_params {
    const double* window;      /* (2r+1)*B*B values */
    int window_len;
    const double* sigma;       /* 1 value (flat) or (2r+1)*B*(B/2+1) values */
    int sigma_len;
    double sigma2;
    double pmin;
    double pmax;
    int filter_type;           /* 0..6 as translated by python/dfttest2.py:263-271 */
    int radius;                /* 0..3 */
    int block_size;            /* 8, 16 or 32 */
    int block_step;
    int zero_mean;
    const double* window_freq; /* (2r+1)*B*(B/2+1)*2 values, required when zero_mean */
    int window_freq_len;
    int device_id;
    int num_streams;
    /* Temporal slice of `window` used as the synthesis window.  -1 selects the
     * centre slice r, as dfttest2_nvrtc / dfttest2_cuda do
     * (cuda_source/kernels.cu:240); dfttest2_cpu uses slice 2r
     * (cpu_source/getframe_impl.cpp:383).  They agree for a rectangular
     * temporal window or r = 0. */
    int synthesis_slice;
} dfttest2_b200_params;

/* One output plane: 2r+1 source planes (frames n-r..n+r, already clamped to
 * the clip as in nvrtc_source/source.cpp:427-431) and the destination.
 * Strides are in bytes. */
typedef struct dfttest2_b200_plane {
    const void* src[7];
    ptrdiff_t src_stride;
    void* dst;
    ptrdiff_t dst_stride;
    int width;
    int height;
} dfttest2_b200_plane;

/* Fills *p with the reference defaults (all optional fields -1). */
void dfttest2_b200_params_init(dfttest2_b200_params* p);

/* DFTTestCreate: validates the arguments, selects the device and uploads the
 * constant tables.  On failure *out is NULL and the message is the
 * reference's (e.g. "\"radius\" must be in [0, 1, 2, 3]"). */
int dfttest2_b200_create(const dfttest2_b200_params* params, dfttest2_b200_filter** out);

/* DFTTestFree */
void dfttest2_b200_free(dfttest2_b200_filter* f);

/* Batched device-resident path: every plane's pointers are device memory on
 * the filter's device; all planes share the sample format.  The work is
 * queued on `stream` (a cudaStream_t, NULL = legacy default stream) and the
 * call returns without waiting.  This is the hot path that
 * DFTTestGetFrame's kernel launches (nvrtc_source/source.cpp:487-551)
 * correspond to, for any number of planes and frames at once. */
int dfttest2_b200_process_planes(dfttest2_b200_filter* f, const dfttest2_b200_plane* planes, int nplanes,
                                 int sample_type, int bits_per_sample, void* stream);

/* Kernel status of the asynchronous calls (process_planes,
 * process_planes_sigma, the tensor-core form).  The kernels record an
 * internal failure (a unit wider than the kernel's strip, a bounded wait for
 * the tensor cores that ran out) in an error word of the stream slot instead
 * of trapping; this waits for the filter's queued work, clears the words and
 * returns DFTTEST2_B200_EKERNEL with the failure's text if any was set.  The
 * host-memory calls below (process_plane_host, the cached and clip paths)
 * read the word after their own wait and return DFTTEST2_B200_EKERNEL
 * themselves.  The reference reports every CUDA failure through
 * setFilterError (cuda_source/source.cpp:124-138, 418-421). */
int dfttest2_b200_check(dfttest2_b200_filter* f);

/* Iteration limit of the filter's bounded device waits (the tensor-core
 * form's waits for its products); a negative value restores the default
 * (2^22 polls).  A limit of 0 makes every such wait give up at once: the
 * kernel then drains the products in flight with the default limit, frees
 * its tensor memory, returns early and the call reports
 * DFTTEST2_B200_EKERNEL.  Meant for failure-path tests; no counterpart in
 * the reference. */
int dfttest2_b200_set_wait_limit(dfttest2_b200_filter* f, int iterations);

/* Host-memory path with the semantics of DFTTestGetFrame for one plane:
 * copies the 2r+1 source planes in, filters, copies the result out and
 * waits for completion.  Concurrent calls are spread over num_streams
 * stream slots (nvrtc_source/source.cpp:471-584). */
int dfttest2_b200_process_plane_host(dfttest2_b200_filter* f, const dfttest2_b200_plane* plane, int sample_type,
                                     int bits_per_sample);

/* As dfttest2_b200_process_plane_host, for hosts that filter a clip frame by
 * frame (a VapourSynth GetFrame): src_frame_ids[t] is the clip frame number of
 * plane->src[t] (after the clip-end clamp) and plane_index the plane of the
 * format.  Source planes are kept on the device keyed by (frame number,
 * plane index), so consecutive frames upload each source frame once instead
 * of 2r+1 times (the reference uploads a padded stack of 2r+1 frames per
 * output frame, nvrtc_source/source.cpp:456-551).  The key must identify the
 * plane's contents for the life of the filter (true for the frames of one
 * clip).  Thread-safe; at most 64 planes are cached per filter. */
int dfttest2_b200_process_plane_host_cached(dfttest2_b200_filter* f, const dfttest2_b200_plane* plane,
                                            const int* src_frame_ids, int plane_index, int sample_type,
                                            int bits_per_sample);

/* The same for several planes of one output frame (the planes of a YUV
 * frame, one sample format): every plane in one launch and one wait.
 * plane_indices[i] is the plane index of planes[i]; src_frame_ids as above
 * (shared by the planes).  nplanes <= 4. */
int dfttest2_b200_process_frame_host_cached(dfttest2_b200_filter* f, const dfttest2_b200_plane* planes, int nplanes,
                                            const int* plane_indices, const int* src_frame_ids, int sample_type,
                                            int bits_per_sample);

/* Whole-clip host path: filters `nframes` frames of one plane stored
 * contiguously in host memory (frame i at src + i*frame_bytes, rows
 * src_stride bytes apart) into dst.  Each source frame is uploaded once
 * and reused by the 2r+1 outputs that need it; the temporal window is
 * clamped at the clip ends (cpu_source/getframe_impl.cpp:296-298). */
int dfttest2_b200_process_clip_host(dfttest2_b200_filter* f, const void* src, ptrdiff_t src_stride,
                                    ptrdiff_t src_frame_bytes, void* dst, ptrdiff_t dst_stride,
                                    ptrdiff_t dst_frame_bytes, int nframes, int width, int height, int sample_type,
                                    int bits_per_sample);

/* One plane of a clip in host memory: frame i at src + i*src_frame_bytes,
 * rows src_stride bytes apart (likewise dst). */
typedef struct dfttest2_b200_host_plane {
    const void* src;
    ptrdiff_t src_stride;
    ptrdiff_t src_frame_bytes;
    void* dst;
    ptrdiff_t dst_stride;
    ptrdiff_t dst_frame_bytes;
    int width;
    int height;
} dfttest2_b200_host_plane;

/* Whole-clip host path over several planes of one sample format (the planes
 * of a YUV clip): one upload / filter / download pipeline for all of them, so
 * it fills and drains once; each chunk of frames filters every plane's
 * frames in one launch.  Same semantics per plane as
 * dfttest2_b200_process_clip_host, which is this call with one plane. */
int dfttest2_b200_process_clip_planes_host(dfttest2_b200_filter* f, const dfttest2_b200_host_plane* planes,
                                           int nplanes, int nframes, int sample_type, int bits_per_sample);

/* Differentiable path (float planes).  The reference has no gradient; these
 * serve training the sigma array and backpropagating through the filter.
 *
 * dfttest2_b200_process_planes_sigma: as dfttest2_b200_process_planes, with
 * the per-bin sigma array taken from device memory (float,
 * (2r+1)*B*(B/2+1), layout of the `sigma` argument), so it can change
 * between calls without host round trips.
 *
 * dfttest2_b200_backward_planes: adjoint of the same filter.  For every
 * plane, grad_dst is dL/d(output plane); dL/d(source planes) is ADDED to
 * grad_src[t] (the caller zeroes them; planes that alias the same frame
 * accumulate) and dL/d(sigma) is ADDED to grad_sigma (may be NULL).  sigma
 * NULL means the array given at create time.  Block spectra are recomputed,
 * nothing is kept from the forward call. */
typedef struct dfttest2_b200_grad_plane {
    const void* src[7];
    float* grad_src[7];
    const float* grad_dst;
    ptrdiff_t src_stride;
    ptrdiff_t grad_src_stride;
    ptrdiff_t grad_dst_stride;
    int width;
    int height;
} dfttest2_b200_grad_plane;

int dfttest2_b200_process_planes_sigma(dfttest2_b200_filter* f, const dfttest2_b200_plane* planes, int nplanes,
                                       int sample_type, int bits_per_sample, const float* sigma, void* stream);

int dfttest2_b200_backward_planes(dfttest2_b200_filter* f, const dfttest2_b200_grad_plane* planes, int nplanes,
                                  const float* sigma, float* grad_sigma, void* stream);

/* Arithmetic of the per-block transforms.  FP32 (the default) runs them as
 * FP32 FFT codelets on the CUDA cores, like the reference's kernels
 * (nvrtc_source/kernels.cu:86-295).  The TC modes run them as dense products
 * on the tensor cores (tcgen05.mma, FP32 accumulation): TC_FP16X3 and
 * TC_BF16X3 split every operand into 16-bit hi + lo parts and sum three
 * products (about 22 and 16 significant bits), TC_TF32 and TC_BF16 use one
 * product (10 and 7 bits); the gain, zero-mean and overlap-add stay in FP32.
 * TC_FP16X3, and TC_BF16X3 where the arguments allow it, use the strip form
 * (block_size 16, radius 0 or 1, block_step 1, 2 or 4, a separable window
 * and sigma symmetric in the x-bins 0 and block_size/2, as the Python front
 * end produces; the x products run over 8 blocks at once); TC_FP16X3 fails
 * with DFTTEST2_B200_EINVAL outside it.  The other modes use the tile form
 * (block_size 16 with radius 0 or 1, block_size 32 with radius 0).  No
 * counterpart in the reference.  Applies to the process_* paths of the
 * filter (not to the differentiable and batch paths, which stay FP32). */
#define DFTTEST2_B200_FP32 0
#define DFTTEST2_B200_TC_BF16X3 1
#define DFTTEST2_B200_TC_TF32 2
#define DFTTEST2_B200_TC_BF16 3
#define DFTTEST2_B200_TC_FP16X3 4

int dfttest2_b200_set_precision(dfttest2_b200_filter* f, int mode);

/* Multi-clip batches.  The reference filters one clip per filter instance,
 * one frame per DFTTestGetFrame call (nvrtc_source/source.cpp:356-605); a
 * batch filters many device-resident clips, each with its own DFTTest
 * arguments (its filter), size, length and sample format, in one CUDA graph
 * launch.
 *
 * At creation every frame of every clip becomes a plane job of a work-list.
 * Jobs are grouped by kernel (block size, block step, temporal size, Wiener
 * or general gain); each group is one kernel over its cost-ordered
 * work-list (largest planes first) plus its overlap fix-up, and the groups
 * run as parallel branches of one graph.  With DFTTEST2_B200_BATCH_TUNE the
 * kernel shape (warps per CTA) and unit split of every group are chosen by
 * timing the candidates on the batch itself (the timed runs write the same
 * outputs as a normal run); choices are cached per process by group
 * signature.  Without it the single-call heuristics are used. */
typedef struct dfttest2_b200_batch dfttest2_b200_batch;

typedef struct dfttest2_b200_clip {
    dfttest2_b200_filter* filter;  /* DFTTest arguments of this clip; must outlive the batch */
    const void* src;               /* device memory: frame i at src + i*src_frame_bytes */
    ptrdiff_t src_stride;          /* bytes between rows */
    ptrdiff_t src_frame_bytes;
    void* dst;                     /* device memory, same layout rules */
    ptrdiff_t dst_stride;
    ptrdiff_t dst_frame_bytes;
    int nframes;                   /* the temporal window is clamped at the clip ends */
    int width;
    int height;
    int sample_type;
    int bits_per_sample;
} dfttest2_b200_clip;

#define DFTTEST2_B200_BATCH_TUNE 1

/* Validates the clips (all filters on one device), builds the work-lists,
 * tunes when asked, allocates the scratch and captures the graph.  The
 * clip memory must stay valid for the life of the batch. */
int dfttest2_b200_batch_create(const dfttest2_b200_clip* clips, int nclips, int flags, dfttest2_b200_batch** out);

/* Launches the batch's graph on `stream` (asynchronous). */
int dfttest2_b200_batch_run(dfttest2_b200_batch* b, void* stream);

/* Writes a one-line-per-group description (kernel, shape, units, jobs, tuning
 * times) into buf (NUL-terminated, truncated to len).  Returns the number of
 * kernel launches per run, or a negative status. */
int dfttest2_b200_batch_describe(const dfttest2_b200_batch* b, char* buf, int len);

void dfttest2_b200_batch_free(dfttest2_b200_batch* b);

/* Size of the device array that dfttest2_b200_process_plane_noalloc works
 * in (bytes, per GPU, held from library load until process exit). */
#define DFTTEST2_B200_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)

/* Allocation-free single-plane filter.  No counterpart in the reference:
 * this is an addition for callers that cannot allocate GPU memory, such as
 * a host that hands the filter frames from a memory pool it has already
 * reserved and that must not see cudaMalloc / cudaFree (which can claim
 * memory outside its budget and implicitly synchronise the device in the
 * middle of its pipeline).
 *
 * It takes the DFTTest arguments (as dfttest2_b200_create) and one plane
 * whose pointers are device memory on params->device_id, and queues the
 * same kernels as dfttest2_b200_process_planes on `stream`, asynchronously.
 * It allocates nothing: its tables, plane descriptor and overlap scratch
 * live in one statically sized device array of
 * DFTTEST2_B200_NOALLOC_SCRATCH_BYTES; a plane whose scratch needs more is
 * rejected with an error that states both sizes.
 *
 * The first call on a device resolves the array's device address.  A call
 * inside a stream capture is rejected (DFTTEST2_B200_EINVAL): the plane
 * descriptor (from the call's stack frame) and the tables (from a
 * process-wide host buffer that the next call rewrites) are copied with
 * cudaMemcpyAsync from pageable host memory, which a replayed graph would
 * read again after the call has returned (pageable copies may also wait for
 * the stream).  All calls on a device share the array, so calls that overlap on
 * the GPU (different streams, or concurrent host threads) race: serialise
 * them on one stream. */
int dfttest2_b200_process_plane_noalloc(const dfttest2_b200_params* params, const dfttest2_b200_plane* plane,
                                        int sample_type, int bits_per_sample, void* stream);

/* Kernel status of the last dfttest2_b200_process_plane_noalloc call on
 * device_id: waits for `stream`, then reads the error word in the same static
 * array (allocates nothing) and returns DFTTEST2_B200_EKERNEL with the
 * failure's text if the kernels reported one.  No reference counterpart. */
int dfttest2_b200_noalloc_check(int device_id, void* stream);

/* RDFT: FP64 direct real DFT over 1, 2 or 3 axes, real last axis first
 * (cpu_source/source.cpp:269-340).  `out` receives
 * prod(shape[:-1]) * (shape[-1]/2+1) interleaved (re, im) values. */
int dfttest2_b200_rdft(const double* data, int data_len, const int* shape, int ndim, double* out, int out_len);

/* Version string (version, build architecture, kernel variant). */
const char* dfttest2_b200_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* dfttest2_b200_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* DFTTEST2_B200_H */
