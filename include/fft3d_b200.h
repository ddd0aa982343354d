/*
 * fft3d_b200.h — C ABI of the B200 (sm_100a) FFT3D filtering core.
 *
 * This is the drop-in boundary for the per-plane engine of neo_fft3d:
 * one fft3d_plane replaces one FFT3DEngine (reference src/fft3d_engine.h:22-741),
 * which the plugin filter creates per processed plane (src/fft3d.hpp:186-198)
 * and calls once per output frame (src/fft3d.hpp:241). Everything below takes
 * plain pointers and sizes; no CUDA or torch types appear in the signatures
 * (a CUDA stream is passed as void*).
 *
 * All functions return FFT3D_OK (0) or a negative FFT3D_E_* status; the
 * message of the last failure on the calling thread is fft3d_last_error().
 * Parameter errors carry the reference's own messages
 * (src/fft3d_engine.h:105-126, src/fft3d.hpp:143-147).
 *
 * Threading: a plane handle is internally locked, so concurrent calls on one
 * handle are serialised (like the reference's cache mutex). Distinct handles
 * run concurrently; each owns one CUDA stream.
 */
#ifndef FFT3D_B200_H
#define FFT3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFT3D_OK 0
#define FFT3D_E_PARAM (-1)       /* invalid parameter (reference-compatible message) */
#define FFT3D_E_CUDA (-2)        /* CUDA runtime or launch failure */
#define FFT3D_E_UNSUPPORTED (-3) /* valid for the reference, not built here (see message) */
#define FFT3D_E_NOMEM (-4)       /* device allocation failed */
#define FFT3D_E_FRAME (-5)       /* a frame the call needs was not supplied */
#define FFT3D_E_NOLIB (-6)       /* no CUDA device / driver */

/* Filter parameters: the parameter surface of neo_fft3d (src/fft3d.hpp:29-73)
 * with the reference's meanings. Defaults: fft3d_params_default()
 * (src/fft3d.hpp:77-106). Field names follow EngineParams
 * (src/fft3d_common.h:61-100). Booleans are ints. */
typedef struct fft3d_params {
  float sigma, beta;
  int bw, bh, bt, ow, oh;
  float kratio, sharpen, scutoff, svr, smin, smax;
  int measure, interlaced, wintype;
  int pframe, px, py, pshow;
  float pcutoff, pfactor;
  float sigma2, sigma3, sigma4;
  float degrid, dehalo, hr, ht;
  int l, t, r, b;
  int opt, ncpu, mt;
} fft3d_params;

/* One plane of a clip, as the engine sees it (src/fft3d.hpp:186-192). */
typedef struct fft3d_plane_desc {
  int width, height;   /* plane size in pixels (already subsampled for chroma) */
  int bits;            /* bits per sample: 8 (uint8), 9..16 (uint16), 32 (float) */
  int is_chroma;       /* YUV chroma plane: integer samples are centred on 2^(bits-1) */
  int ssw, ssh;        /* subsampling shifts applied to the crop l/r and t/b */
  int num_frames;      /* clip length; frames near either end use bt = 1 */
  int rgb;             /* plane of an RGB clip (pshow's display offset; 0 for YUV and Gray) */
} fft3d_plane_desc;

typedef struct fft3d_plane fft3d_plane;

/* Reference defaults (src/fft3d.hpp:77-106): sigma 2, beta 1, bw=bh=32, bt=3,
 * ow=oh=-1 (-> bw/3), kratio 2, sharpen 0, scutoff 0.3, svr 1, smin 4,
 * smax 20, measure 1, wintype 0, pcutoff 0.1, pfactor 0, sigma2..4 = sigma,
 * degrid 1, dehalo 0, hr 2, ht 50, ncpu 2. */
void fft3d_params_default(fft3d_params* p);

/* Create a plane engine on CUDA device `device`.
 * Replaces FFT3DEngine::FFT3DEngine (src/fft3d_engine.h:87-408). */
int fft3d_plane_create(const fft3d_params* p, const fft3d_plane_desc* d, int device, fft3d_plane** out);

/* Filter output frame n of this plane from HOST memory.
 * Replaces FFT3DEngine::GetFrame (src/fft3d_engine.h:452-734).
 * src[2+d] is frame n+d for d in [-2, 2] (the reference's apply_in[] slots,
 * src/fft3d_engine.h:634-644); only d in [-bt/2, (bt-1)/2] is read, and a slot
 * may be NULL when that frame's spectrum is already cached on the device
 * (query with fft3d_plane_cached). src_stride / dst_stride are in bytes.
 * The whole plane is written to dst: the crop borders (l, t, r, b) are copied
 * from src[2], as the plugin filter does (src/fft3d.hpp:292-352). */
int fft3d_plane_filter(fft3d_plane* h, int n, const void* const src[5], const int src_stride[5], void* dst,
                       int dst_stride);

/* Same as fft3d_plane_filter, but src/dst are DEVICE pointers and the work is
 * queued on `stream` (a cudaStream_t; NULL = the handle's own stream) without
 * a host synchronisation. A plane's calls are queued one at a time (its lock);
 * their GPU work is ordered when they use one stream, as the spectrum ring and
 * the Kalman state carry over from call to call: a caller that switches
 * streams orders them itself (an event). */
int fft3d_plane_filter_device(fft3d_plane* h, int n, const void* const src[5], const int src_stride[5], void* dst,
                              int dst_stride, void* stream);

/* Frame group (no counterpart in the reference, whose engine filters one
 * output frame per GetFrame, src/fft3d_engine.h:452-734): output frames
 * n0 .. n0 + count - 1 of one plane in one call, 1 <= count <=
 * FFT3D_MAX_FRAME_GROUP. DEVICE pointers: src[j] is frame n0 - 2 + j for
 * j in [0, count + 4) with stride src_stride[j] (NULL outside the clip, or
 * where the frame's spectrum is cached); frame n0 + j is written to dst[j]
 * (stride dst_stride[j]); all work is queued on `stream` (NULL = the
 * handle's own stream). On the default and tensor-core paths, the group's
 * new frames are transformed by one launch and its overlap-adds are one
 * launch; Wiener 3D
 * planes (bt = 2..5) filter the group's frames with one filter/inverse launch
 * whose CTAs interleave the frames block range by block range, so that a
 * window spectrum shared by up to bt frames is read from HBM about once
 * (Kalman, Wiener 2D and sharpen-only planes: one filter/inverse launch per
 * frame, in frame order). The ring keeps every spectrum the group needs and
 * there is one time-domain buffer per frame (both grow on first use:
 * count + bt spectra and count - 1 buffers). Planes on the other paths
 * (fused, learned PSD, bulk-staged) filter the frames one after another.
 * Outputs are those of count calls of fft3d_plane_filter_device. */
#define FFT3D_MAX_FRAME_GROUP 16
int fft3d_plane_filter_frames_device(fft3d_plane* h, int n0, int count, const void* const* src,
                                     const int* src_stride, void* const* dst, const int* dst_stride, void* stream);

/* Same as fft3d_plane_filter_frames_device with HOST frames (as in
 * fft3d_plane_filter): the frames the group needs and the device does not
 * hold are uploaded, the outputs downloaded, and the call returns when they
 * are in dst. Calls from several threads overlap one call's copies with
 * another's kernels; each call owns one of the plane's 4 group staging sets
 * until it returns (a fifth concurrent call waits for a free one). Planes
 * with crop borders, and planes that are not grouped, go through
 * fft3d_plane_filter frame by frame. */
int fft3d_plane_filter_frames(fft3d_plane* h, int n0, int count, const void* const* src, const int* src_stride,
                              void* const* dst, const int* dst_stride);

/* 1 if the spectrum of frame n is held in the device spectrum cache. */
int fft3d_plane_cached(fft3d_plane* h, int n);

/* Copy the forward spectrum of frame n (which must be cached) to host memory
 * as blocks x bh x (bw/2+1) complex floats (interleaved re, im; no padding). */
int fft3d_plane_spectrum(fft3d_plane* h, int n, float* out);

/* Geometry: out[0..7] = nox, noy, cover width, cover height, bw/2+1, blocks,
 * ow, oh (after the ow/oh = bw/3 default is applied). */
int fft3d_plane_geometry(fft3d_plane* h, int out[8]);

/* Estimate the noise pattern (pfactor != 0) from one frame in HOST memory, as
 * the reference does from frame pframe on its first GetFrame
 * (src/fft3d_engine.h:485-504, src/helper.cpp:46-132): block (px, py), or the
 * quietest block when px = py = 0. Required before the first filter call of a
 * pattern-mode plane; a no-op otherwise, and for pshow planes, which find the
 * block on every frame. */
int fft3d_plane_set_pattern_frame(fft3d_plane* h, const void* src, int src_stride);

/* Drop all cached spectra and reset the Kalman state to its initial values.
 * Waits first for the work already queued for this plane, on whatever stream
 * it was queued (device-buffer calls and batch steps included). */
int fft3d_plane_reset(fft3d_plane* h);

void fft3d_plane_destroy(fft3d_plane* h);

/* Device memory this plane holds, in bytes (tables, spectrum ring, Kalman
 * state, time-domain blocks, staging planes; frame groups grow it). No
 * counterpart in the reference. When the environment variable
 * NEO_FFT3D_DEVICE_ALLOC_CAP is set at fft3d_plane_create, the plane's device
 * allocations stop at that many bytes and fail with FFT3D_E_NOMEM, as on an
 * exhausted device (a host-side fault injection for the out-of-memory paths). */
int fft3d_plane_device_bytes(fft3d_plane* h, uint64_t* out);

/* Wait for all work queued for this plane (on any stream) and report what the
 * device-buffer calls cannot: a bounded device-side wait of one of the
 * plane's kernels that ran out (FFT3D_E_CUDA with "... timed out"; the flag is
 * cleared, so the next call starts clean). Host-buffer calls report it
 * themselves. No counterpart in the reference, whose filter runs on the host. */
int fft3d_plane_synchronize(fft3d_plane* h);

/* Test hook (host-side fault injection, no counterpart in the reference): sets
 * the plane's device error flag to `bits`, as a kernel does when a bounded
 * wait runs out (bit 0: tensor-core MMA completion, bit 1: bulk copy
 * completion), after the work already queued for the plane. The next
 * host-buffer call, or fft3d_plane_synchronize, then reports the error and
 * clears the flag. Lets the device error path be tested without a real
 * device fault. */
int fft3d_plane_debug_set_error_flag(fft3d_plane* h, int bits);

/* Per-kernel timing of this handle: when enabled, every launch is bracketed
 * by CUDA events on the stream it runs on. */
int fft3d_plane_set_timing(fft3d_plane* h, int enable);

/* Read and reset the timing counters: out[3k+0] launches, out[3k+1] summed
 * event milliseconds, out[3k+2] summed algorithmic bytes (what the launch's
 * interface must read and write once), for k = 0 forward (gather + window +
 * r2c), 1 filter + inverse (spectra in, time-domain blocks out), 2 overlap-add
 * (time-domain blocks in, pixels out), 3 fused (newest frame's pixels and the
 * older spectra in; newest spectrum and time-domain blocks out), 4 streaming
 * filter (the window's spectra in, filtered spectrum out). Waits for the
 * recorded launches. */
int fft3d_plane_timing(fft3d_plane* h, double out[15]);

/* Allocation-free filtering of ONE frame of one plane (DEVICE pointers),
 * queued on `stream` (a cudaStream_t; NULL = the legacy default stream).
 * No counterpart in the reference: it exists for callers that cannot allocate
 * device memory while frames flow -- applications whose device memory is all
 * owned by their own pool allocator, and real-time pipelines that must not pay
 * the implicit synchronisation and latency of cudaMalloc/cudaFree. The call
 * allocates and frees nothing: the plane's tables, the frame's spectrum and
 * its time-domain blocks live in one fixed 32 MiB device array that every GPU
 * loading this library holds until the process exits. Spatial modes only
 * (bt = 1 Wiener with sharpen/dehalo, bt = -1 sharpen/dehalo); no noise
 * patterns, no interlacing. A plane needing more scratch than 32 MiB (e.g.
 * 1080p luma at bw=bh=32, ow=oh=16; 720p luma and 1080p chroma fit) returns
 * FFT3D_E_UNSUPPORTED. All calls on a device share the array and find the
 * previous call's contents in it (each call writes everything it reads), so
 * calls whose GPU work overlaps race: keep them on one stream. The first call
 * on a device resolves the array's address and uploads the FFT twiddle tables;
 * make it before any stream capture. Later calls only queue kernels on
 * `stream` (the plane's tables travel as kernel parameters) and never wait on
 * it from the host. Not for use across a cudaDeviceReset of a device it has
 * run on (the address and tables are kept per device for the process's life).
 * Output equals fft3d_plane_filter_device's with the same parameters, byte
 * for byte (the same kernels). */
int fft3d_filter2d_static(const fft3d_params* p, const fft3d_plane_desc* d, const void* src, int src_stride,
                          void* dst, int dst_stride, void* stream);

/* ------------------------------------------------------------------------
 * Batched multi-plane scheduler. No counterpart in the reference, which runs
 * one FFT3DEngine per plane per clip (src/fft3d.hpp:186-198, 241). One step
 * filters one output frame of each of `count` planes -- luma and chroma of
 * many clips, of mixed sizes, block sizes, bt and sample types -- with one
 * batched persistent launch per kernel variant, phase (forward,
 * filter/inverse, overlap-add) and wave instead of three launches per plane.
 * A wave is a run of planes whose new spectra and time-domain blocks fit a
 * byte budget, so that they can stay in L2 from one phase to the next. The
 * first steps of a new step shape are timed under candidate wave budgets
 * and then under candidate schedules per launch (persistent grid size,
 * work-item order), keeping the fastest (autotuner); the tuned step is
 * captured into a CUDA graph and replayed on later steps of that shape.
 * ------------------------------------------------------------------------ */
typedef struct fft3d_batch fft3d_batch;

int fft3d_batch_create(int device, fft3d_batch** out);
void fft3d_batch_destroy(fft3d_batch* b);

/* 1 (default): tune new step shapes; 0: use the default schedule (all
 * resident CTAs per SM, plane-major work items). */
int fft3d_batch_set_tuning(fft3d_batch* b, int enable);

/* One step: plane i filters its output frame n[i] from DEVICE frames
 * src[5*i + k] (frame n[i] + k - 2, strides src_stride[5*i + k] in bytes, as
 * in fft3d_plane_filter_device) into dst[i] (stride dst_stride[i]); all work
 * is queued on `stream` (a cudaStream_t) without a host synchronisation
 * (except while a new step shape is tuned). Successive steps of one batch
 * must use one stream. Planes must be on the batch's device, on the default
 * (unfused) path, without a learned PSD.
 * Frame groups: a Wiener/sharpen plane (bt != 0) may appear several times in
 * one step with consecutive frames n, n + 1, ... (in item order). The
 * group's filter/inverse work items then run together, interleaved frame by
 * frame over the same blocks, so that each block's window spectra are read
 * from HBM about once per group instead of once per frame (the rest hit L2);
 * the plane keeps every spectrum the group needs (its ring and time-domain
 * buffers grow on first use). Outputs are those of one-frame-at-a-time
 * filtering. A Kalman plane (bt = 0) appears at most once per step. */
int fft3d_batch_step(fft3d_batch* b, int count, fft3d_plane* const* planes, const int* n, const void* const* src,
                     const int* src_stride, void* const* dst, const int* dst_stride, void* stream);

/* out[0] steps, [1] graph launches, [2] tuning steps, [3] host milliseconds
 * spent planning the steps' planes (summed), [4] kernels of the last step,
 * [5] step shapes seen, [6] wave budget (MiB, 0 = one wave) of the last
 * tuned step, [7] host milliseconds of the steps (summed). */
int fft3d_batch_stats(fft3d_batch* b, double out[8]);

/* Per-phase kernel timing (1 = on). While on, tuned steps run without their
 * CUDA graph, with events around every launch. fft3d_batch_timing waits for
 * the timed launches and returns, cumulated since the batch was created,
 * out[3*k + 0] launches, [3*k + 1] milliseconds and [3*k + 2] algorithmic
 * bytes (each distinct input read once, outputs written once) for k = 0
 * forward, 1 filter/inverse, 2 plane copies, 3 overlap-add. */
int fft3d_batch_set_timing(fft3d_batch* b, int enable);
int fft3d_batch_timing(fft3d_batch* b, double out[12]);

/* ------------------------------------------------------------------------
 * Learned noise PSD. No counterpart in the reference, whose per-frequency
 * noise comes from sigma..sigma4 (src/helper.cpp:14-44) or from one measured
 * block (src/helper.cpp:46-132) and enters the Wiener gain through the
 * `pattern` slot (pattern2d, and pattern3d = bt x pattern2d,
 * src/helper.cpp:171-178, src/fft3d_engine.h:625-630). This model predicts,
 * for every 32x32 block, that slot's per-frequency noise power from the
 * block's own log power spectrum: a 3-layer MLP (544 -> 512 -> 512 -> 544 bins,
 * GELU, BF16 weights and activations, FP32 accumulation on the tensor cores,
 * FP32 master weights, Adam), trained on the device from noisy/clean block
 * pairs that the device generates (coloured Gaussian noise shaped by a random
 * radially symmetric transfer function over seeded sinusoid-field frames).
 * Units: |X|^2 of the plane's windowed, unnormalised block FFT.
 * ------------------------------------------------------------------------ */
typedef struct fft3d_psd fft3d_psd;

#define FFT3D_PSD_BINS 544     /* 32 rows x 17 columns of a 32x32 block's half spectrum */
#define FFT3D_PSD_FEATURES 576 /* model input width: BINS padded to a multiple of 64 */
#define FFT3D_PSD_HIDDEN 512
#define FFT3D_PSD_OUTPUTS 640  /* model output width: BINS padded to a multiple of 128 */
#define FFT3D_PSD_INFO 12      /* floats of generator record per block, see fft3d_psd_generate */

typedef struct fft3d_psd_train_cfg {
  long long blocks;            /* training blocks generated on the device (default 2^21) */
  int batch;                   /* rows per Adam step, a multiple of 128 (default 4096) */
  int epochs;                  /* passes over the generated blocks (default 3) */
  float lr, lr_final;          /* Adam step size, decayed linearly to lr_final */
  unsigned long long seed;     /* data seed (weights are seeded at creation) */
  int clean_frames;            /* clean frames generated at width x height (default 16) */
  int width, height;           /* default 1920 x 1080 */
  float sigma_min, sigma_max;  /* total noise sigma range in 8-bit codes (default 2, 10) */
  float knot_min;              /* smallest transfer-function knot amplitude (default 0.1) */
} fft3d_psd_train_cfg;

void fft3d_psd_train_default(fft3d_psd_train_cfg* cfg);

/* A model for 32x32 blocks with the analysis window of (ow, oh, wintype),
 * weights initialised from `seed` (normal, std 1/sqrt(fan-in); zero biases). */
int fft3d_psd_create(int device, unsigned long long seed, int ow, int oh, int wintype, fft3d_psd** out);
void fft3d_psd_destroy(fft3d_psd* m);

/* Parameters as FP32: W1 [512][576], b1 [512], W2 [512][512], b2 [512],
 * W3 [640][512], b3 [640] (row = output unit), in that order. Input and output
 * columns past 544 are padding (zero features; ignored outputs). */
long long fft3d_psd_param_count(void);
int fft3d_psd_get_params(fft3d_psd* m, float* host, long long n);
int fft3d_psd_set_params(fft3d_psd* m, const float* host, long long n);

/* Generate cfg->blocks training blocks on the device and train for
 * cfg->epochs. loss_curve (may be NULL) receives the mean training loss of
 * curve_len equal stretches of the run; val_loss (may be NULL) the loss on
 * 32768 held-out blocks after training. */
int fft3d_psd_train(fft3d_psd* m, const fft3d_psd_train_cfg* cfg, float* loss_curve, int curve_len, float* val_loss);

/* Device timing of the last fft3d_psd_train: out[0] ms generating the blocks,
 * out[1] ms of the training steps, out[2] steps, out[3] GEMM flops per step
 * (forward + backward). */
int fft3d_psd_train_stats(fft3d_psd* m, double out[4]);

/* The generator's blocks first .. first+count-1 of a training run with cfg,
 * copied to HOST arrays (each may be NULL): features [count][576] (the BF16
 * model input as float), target [count][544] (log noise power minus 7),
 * info [count][12] (total sigma, knot amplitudes a0..a3 at radius 0, 1/3,
 * 2/3, 1, direction (0 falling, 1 rising), noise gain s, clean frame, x0, y0,
 * sum of FIR taps squared, 0), clean [count][1024] (unrounded clean pixels),
 * noisy [count][1024] (8-bit noisy pixels). */
int fft3d_psd_generate(fft3d_psd* m, const fft3d_psd_train_cfg* cfg, long long first, long long count,
                       float* features, float* target, float* info, float* clean, unsigned char* noisy);

/* One forward and backward pass on HOST rows (rows a multiple of 128):
 * features [rows][576], target [rows][544]; writes the loss (mean squared
 * error of the 544 outputs) and the gradients in the parameter layout. */
int fft3d_psd_gradients(fft3d_psd* m, const float* features, const float* target, int rows, float* grads,
                        float* loss);

/* Model output for HOST feature rows: out [rows][544] (log noise power minus 7). */
int fft3d_psd_forward(fft3d_psd* m, const float* features, int rows, float* out);

/* Use the model's prediction in place of sigma for this plane: every output
 * frame, the current frame's block spectra go through the model and the
 * Wiener (or Kalman) noise power of block b, bin k becomes strength x its
 * prediction (x bt for Wiener 3D, like pattern3d). The limited Wiener gain
 * max(1 - noise/|F|^2, lowlimit) leaves part of every pure-noise bin when
 * given the exact noise power; over-subtraction by strength ~3 maximises
 * PSNR on the generator's noise (as the best scalar sigma does for white
 * noise, whose sigma^2 / norm is ~3.4x the windowed noise power at bw = 32,
 * ow = 16). pooled = 1 uses the mean log prediction of all blocks of the
 * frame for every block. The plane must have bw = bh = 32 and the model's
 * window; the model must outlive the plane's use of it. m = NULL returns to
 * sigma. */
int fft3d_plane_set_psd(fft3d_plane* h, fft3d_psd* m, int pooled, float strength);

/* Message of the last failure on this thread ("" if none). */
const char* fft3d_last_error(void);

/* Number of kernels this library has launched in this process (all handles). */
uint64_t fft3d_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif /* FFT3D_B200_H */
