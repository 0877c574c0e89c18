/*
 * kbsrc_gpu.h - the C ABI between the host C++ library (planning, staging, kernel taps, LPC edges, WAV I/O)
 * and the sm_100a block engine. Plain pointers and sizes, integer status codes, nothing throws.
 *
 * It replaces, in HongYue1/KBSRC 1.3.0:
 *   run_engine<T,W,C>()          src/resampler.cpp:34-88   -> kbsrc_gpu_engine_create / _run_host / _run_device
 *   kernel_spectrum()            src/design.cpp:40-49      -> kbsrc_gpu_kernel_spectrum
 * The whole conversion kbsrc::resample() (include/kbsrc/kbsrc.hpp:41-43) is also exported in C form by
 * libkbsrc.so as kbsrc_resample_c (include/kbsrc/kbsrc_c.h).
 *
 * Output is byte-identical to the reference CPU engines: the kernels execute the reference's IEEE operation
 * sequence (f64 for fast, double-double for exact) in round-to-nearest.
 */
#ifndef KBSRC_GPU_H
#define KBSRC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define KBSRC_GPU_OK 0
#define KBSRC_GPU_E_ARG (-1)         /* invalid argument */
#define KBSRC_GPU_E_NOMEM (-2)       /* device or host allocation failed */
#define KBSRC_GPU_E_CUDA (-3)        /* a CUDA call failed; kbsrc_gpu_last_error() has the text */
#define KBSRC_GPU_E_UNSUPPORTED (-4) /* a plan this build does not run on the GPU */
#define KBSRC_GPU_E_NODEVICE (-5)    /* no CUDA device */

#define KBSRC_GPU_FAST 0  /* float64 pipeline (reference Precision::Fast) */
#define KBSRC_GPU_EXACT 1 /* double-double pipeline (reference Precision::Exact) */
#define KBSRC_GPU_LD 2    /* x87 extended pipeline, emulated in integers (reference Precision::LongDouble) */
#define KBSRC_GPU_SPLIT 3 /* split-precision form: tensor-core DFT contractions of 8-bit digit slices as int8
                             (int32 accumulators), float64 elsewhere; not byte-identical, within float64 rounding
                             of exact (no reference counterpart) */
#define KBSRC_GPU_SPLIT_F16 4 /* the same split-precision form with the digit slices as f16 (f32 accumulators):
                                 the same products, exact in both, so the same output bytes as KBSRC_GPU_SPLIT */

/* Sample formats of the interleaved input (kbsrc_gpu_desc.in_format). The GPU reads each sample as the
 * reference's WAV reader decodes it (src/io/wav.cpp:299-362): float64 as stored, float32 widened, integer PCM
 * little-endian times 2^-(8B-1) (8-bit unsigned, offset by 128), all exact. Callers of every run function pass
 * `in` (or d_in) pointing at samples of this format, cast to the declared pointer type. */
#define KBSRC_GPU_IN_F64 0
#define KBSRC_GPU_IN_F32 1
#define KBSRC_GPU_IN_S32 2
#define KBSRC_GPU_IN_S24 3 /* 3 bytes per sample */
#define KBSRC_GPU_IN_S16 4
#define KBSRC_GPU_IN_U8 5

typedef struct kbsrc_gpu_engine kbsrc_gpu_engine;

/* One device's share of a conversion split across GPUs by contiguous block ranges (the reference's tasks are
 * independent: each reads its own input span and writes a disjoint output range, src/resampler.cpp:48-50,80-84).
 * All zero: the whole conversion. Otherwise the engine runs blocks [blk0, blk1) of every channel; its input buffer
 * holds frames [frame0, frame0 + frames) (the blocks' spans, their 2*marg*Q halo included, clipped to the signal;
 * the LPC edge buffers stay whole) and its output buffer holds output samples [out0, out0 + nout) of each channel,
 * channel after channel (out[c*nout + i]). kbsrc_gpu_shard_plan computes the shares. */
typedef struct {
    long long blk0, blk1;
    long long frame0, frames;
    long long out0, nout;
} kbsrc_gpu_shard;

/* One conversion plan, as computed by the host planner (reference src/resampler.cpp:98-209).
 * Block b of channel c reads staged samples [b*hop*Q, b*hop*Q + nb*Q) where the staged channel holds
 * `lead` zeros/edge samples before input frame 0 (lead = marg*Q + pre), and writes output samples
 * [b*hop*P - o, (b+1)*hop*P - o) clipped to [0, nout). */
typedef struct {
    int precision;      /* KBSRC_GPU_FAST, KBSRC_GPU_EXACT, KBSRC_GPU_LD, KBSRC_GPU_SPLIT or KBSRC_GPU_SPLIT_F16 */
    int channels;       /* >= 1 */
    long long P, Q;     /* reduced rate ratio rate_out/rate_in = P/Q */
    int nb;             /* block size factor: forward FFT nb*Q points, inverse nb*P */
    int marg;           /* margin in units of Q (input) or P (output) */
    long long nblk;     /* blocks per channel */
    long long lead;     /* staged-sample index of input frame 0 */
    long long o;        /* output offset (pre/Q*P) */
    long long frames;   /* input frames per channel */
    long long nout;     /* output samples per channel */
    int up;             /* rate_out > rate_in: periodic spectrum extension instead of folding */
    int Jg;             /* general-fold bin limit (near-unity ratios), 0 otherwise */
    long long edge_len; /* LPC samples predicted before and after the signal per channel (0: zero padding) */
    const double* H;    /* kernel spectrum, H_len (hi, lo) pairs, host memory; copied at create */
    long long H_len;
    int in_format;      /* KBSRC_GPU_IN_*: the input's sample format (0, float64, when zero-initialised) */
    kbsrc_gpu_shard shard; /* this engine's share of a multi-GPU conversion (zero-initialised: all of it) */
} kbsrc_gpu_desc;

/* Splits the conversion `d` (its shard ignored) into `count` shares of contiguous block ranges, as even as the
 * block count allows: share k gets blocks [nblk*k/count, nblk*(k+1)/count), the input frames those blocks read and
 * the output samples they write; the output ranges partition [0, nout) in order (the last share also owns samples
 * past the last block, which are zero). Host arithmetic only, no device needed. Run share k with
 * kbsrc_gpu_engine_create on a descriptor whose `shard` is shards[k], passing that share's input span (interleaved
 * frames from frame0) and an output buffer of channels * shards[k].nout samples. No data crosses between devices.
 * Not in the reference (its block loop runs on one host). */
int kbsrc_gpu_shard_plan(const kbsrc_gpu_desc* d, int count, kbsrc_gpu_shard* shards);

/* Initialises the current CUDA device for the engine (context, kernel attributes). Optional: the first engine
 * or spectrum call does it otherwise. A caller may run it on another thread while it does host work, since
 * creating a CUDA context takes a good fraction of a second. Not in the reference (no GPU). */
int kbsrc_gpu_init(void);

/* Makes `device` (a CUDA device index) the calling thread's current device: engines, batches and spectra the
 * thread creates afterwards live there. For multi-GPU callers that run one host thread per device. Not in the
 * reference (no GPU). */
int kbsrc_gpu_use_device(int device);

/* Creates an engine on the current CUDA device: FFT plans, twiddle tables and the kernel spectrum on the
 * device. Replaces the set-up half of run_engine (src/resampler.cpp:38-40). */
int kbsrc_gpu_engine_create(const kbsrc_gpu_desc* desc, kbsrc_gpu_engine** out);

/* Runs every (channel, block) task of the plan. Host buffers:
 *   in    interleaved input, frames * channels doubles (pinned memory gives full copy bandwidth)
 *   head  channels * edge_len doubles: head[c*edge_len + i] is the sample i+1 frames before frame 0
 *   tail  channels * edge_len doubles: tail[c*edge_len + i] is the sample i frames after the last frame
 *   out   planar output, channels * nout doubles (out[c*nout + i])
 * head/tail may be NULL when edge_len is 0. An engine created for a share (desc.shard) reads `in` as that share's
 * span, shard.frames * channels doubles from frame shard.frame0, and writes channels * shard.nout samples to `out`
 * (out[c*shard.nout + i] is output sample shard.out0 + i). Replaces the block loop of run_engine
 * (src/resampler.cpp:41-87). */
int kbsrc_gpu_engine_run_host(kbsrc_gpu_engine* e, const double* in, const double* head, const double* tail,
                              double* out);

/* Same with device buffers (a share's span and output range as above), asynchronous on `stream` (a cudaStream_t;
 * NULL = the engine's own stream). The caller keeps the buffers alive until the stream reaches this point. */
int kbsrc_gpu_engine_run_device(kbsrc_gpu_engine* e, const double* d_in, const double* d_head,
                                const double* d_tail, double* d_out, void* stream);

/* kbsrc_gpu_engine_run_device, recording an event after every launch; waits for the run, then returns the
 * summed device time of each pass kind in pass_ms[6] (forward column or direct, forward row, spectrum split,
 * multiply+merge, inverse column or direct, inverse row + output) and their launch counts (may be NULL). */
int kbsrc_gpu_engine_run_device_timed(kbsrc_gpu_engine* e, const double* d_in, const double* d_head,
                                      const double* d_tail, double* d_out, void* stream, float* pass_ms,
                                      int* pass_launches);

/* Output step on the GPU (src/io/wav.cpp:242-255,371-418): the interleaved little-endian data section of a WAV
 * file in `format` (0 f64, 1 f32, 2 s32, 3 s24, 4 s16). Integer formats are scaled by 2^(8B-1), TPDF-dithered
 * when `dither` (two uniform(-0.5, 0.5) draws per sample from std::mt19937_64 seeded 12345, frame-major order,
 * generated on the GPU), rounded to nearest, clipped; *clipped receives the number of clipped samples.
 * kbsrc_gpu_engine_run_host_packed: the block loop on host input followed by the packing; out_bytes is
 *   host memory of channels * nout * bytes-per-sample (whole conversions only: a share returns
 *   KBSRC_GPU_E_UNSUPPORTED, since the dither stream runs from the file's first sample).
 * kbsrc_gpu_pack: packs planar device samples (ch x frames, row stride `stride`) into device memory d_out on
 *   `stream`, synchronous. */
int kbsrc_gpu_engine_run_host_packed(kbsrc_gpu_engine* e, const double* in, const double* head,
                                     const double* tail, int format, int dither, unsigned char* out_bytes,
                                     long long* clipped);
int kbsrc_gpu_pack(const double* d_planar, int channels, long long frames, long long stride, int format, int dither,
                   unsigned char* d_out, long long* clipped, void* stream);

/* Autotuner: picks the launch shape (sequences per CTA, threads per CTA, and for double-double and extended
 * passes whether the stage twiddles are staged in shared memory; see kbsrc_gpu_engine_staging) of each
 * four-step pass (forward column and row, inverse column and row) by timing whole device-resident runs on the
 * given buffers: every candidate shape is applied to all passes at once, each pass keeps its fastest. The radix
 * order and the block size are never changed, so the output bytes are the same under every shape. Runs the
 * conversion many times (d_out holds a valid result afterwards); synchronous. shapes: 8 ints out, F and T of the
 * four passes (0 for a pass that is not a four-step pass: direct, Bluestein or split-precision transforms).
 * Not in the reference (its engines have no launch shapes). */
int kbsrc_gpu_engine_tune(kbsrc_gpu_engine* e, const double* d_in, const double* d_head, const double* d_tail,
                          double* d_out, void* stream, int* shapes);

/* Where the four four-step passes (forward column and row, inverse column and row) read their stage twiddles:
 * 4 ints out, 1 = a copy in each CTA's shared memory, 0 = the global table through the read-only cache, -1 = not a
 * four-step pass. Float64 passes always read the global table; the double-double and extended passes stage by
 * default unless a CTA holds a single sequence (KBSRC_GPU_TW_GLOBAL=1 reads the table in every pass, =0 stages in
 * every pass), and the autotuner chooses per pass. The bytes do not depend on it.
 * Not in the reference (its engines run on the CPU). */
int kbsrc_gpu_engine_staging(const kbsrc_gpu_engine* e, int* staged);

/* Number of (channel, block) tasks, kernel launches per run, and the engine's device bytes. */
int kbsrc_gpu_engine_info(const kbsrc_gpu_engine* e, long long* tasks, long long* launches,
                          long long* device_bytes);

void kbsrc_gpu_engine_destroy(kbsrc_gpu_engine* e);

/* Batches: many conversions at once (the uneven multi-file queue). Conversions whose plans are equal (precision,
 * P/Q, block, margin, fold, kernel spectrum) form one group and share FFT tables. A group with enough work to fill
 * the GPU on every pass runs on its own launches; the other groups of the batch's arithmetic (exact or fast, with
 * four-step 7-smooth transforms: the common rates) run together as one work queue: waves of tasks of any of them,
 * largest transform first, and per wave one persistent launch per pass whose CTAs take units of work (a column or
 * row group of a task, a range of spectrum bins) from an atomic counter, like the reference's workers take tasks
 * (src/resampler.cpp:42-49). KBSRC_GPU_QUEUE=0 runs every group on its own launches. The first run records the whole launch sequence in a CUDA graph and later runs replay it: every buffer
 * pointer is read from a small per-run table, so new buffers need no new recording. Replaces running run_engine
 * once per file (src/resampler.cpp:34-88). descs[i] as for kbsrc_gpu_engine_create (H copied at create; shards are
 * not accepted). */
typedef struct kbsrc_gpu_batch kbsrc_gpu_batch;
int kbsrc_gpu_batch_create(const kbsrc_gpu_desc* descs, int count, kbsrc_gpu_batch** out);
/* Device buffers per conversion (arrays of count pointers; head/tail may be NULL when no conversion has edges).
 * Asynchronous on `stream` (NULL: the batch's own stream); a run waits for the previous one to have started. */
int kbsrc_gpu_batch_run_device(kbsrc_gpu_batch* b, const double* const* d_in, const double* const* d_head,
                               const double* const* d_tail, double* const* d_out, void* stream);
/* Host buffers per conversion, synchronous (device buffers allocated on the first call). */
int kbsrc_gpu_batch_run_host(kbsrc_gpu_batch* b, const double* const* in, const double* const* head,
                             const double* const* tail, double* const* out);
int kbsrc_gpu_batch_info(const kbsrc_gpu_batch* b, long long* groups, long long* tasks, long long* launches);
void kbsrc_gpu_batch_destroy(kbsrc_gpu_batch* b);

/* Real spectrum of the symmetric kernel h[0..L] placed circularly in n points, divided by scale, computed on
 * the GPU with the reference's scalar double-double real FFT (src/design.cpp:40-49, RFFT<dd,dd,dd>).
 * taps: (L+1) (hi, lo) pairs; H: (n/2+1) (hi, lo) pairs out. n must be even. */
int kbsrc_gpu_kernel_spectrum(const double* taps, int L, int n, double scale, double* H);

/* The same kernel spectrum for callers that cannot let a library allocate GPU memory. No counterpart in the
 * reference: it exists for such callers only. Examples: an application that reserves the device's memory up front
 * for its own pool (a framework's caching allocator, an audio host that budgets the GPU at start-up) and has nothing
 * left for cudaMalloc, or one whose other streams must not stall, which they would at the device-wide wait inside
 * cudaFree.
 *   d_taps  (L+1) (hi, lo) pairs in device memory; d_H  (n/2+1) (hi, lo) pairs out, device memory
 *   stream  cudaStream_t to run on (NULL: the CUDA default stream); the call returns once its kernels are queued
 * It calls no cudaMalloc, cudaFree or other allocating routine, and builds and copies no host table: its scratch
 * (work buffers and every twiddle table, computed on the GPU) is one 24 MiB device array inside the library, present
 * on every GPU that loads the library until the process exits. So n is limited to about 300,000 points (80 bytes
 * per point); a larger n returns KBSRC_GPU_E_ARG with the sizes in the message. The n/2-point transform must also
 * have a plan without Bluestein's chirp-z (n/2 7-smooth) whose four-step sub-FFTs have at most 32768 points;
 * otherwise the call returns KBSRC_GPU_E_UNSUPPORTED (use kbsrc_gpu_kernel_spectrum for such n). The array's device
 * address is looked up on every call (cudaGetSymbolAddress, in the current device's context); the first call on a
 * device also sets kernel attributes, so make it before any stream capture. All calls share the one array and it
 * keeps the previous call's contents (each call rewrites all it reads), so calls that can overlap on the GPU (other
 * streams, other threads) race: serialise them. */
int kbsrc_gpu_kernel_spectrum_static(const double* d_taps, int L, int n, double scale, double* d_H, void* stream);

/* Text of the last error on this thread ("" if none). */
const char* kbsrc_gpu_last_error(void);

/* Engine name for Stats::isa, e.g. "sm_100a". */
const char* kbsrc_gpu_engine_name(void);

#ifdef __cplusplus
}
#endif
#endif
