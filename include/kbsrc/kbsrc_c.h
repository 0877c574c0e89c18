/* C form of kbsrc::resample (include/kbsrc/kbsrc.hpp), for FFI callers (ctypes, cgo, JNI).
 * The reference (HongYue1/KBSRC 1.3.0) has only the C++ entry include/kbsrc/kbsrc.hpp:41-45; this wraps it
 * with plain pointers and sizes. Nothing throws across it. */
#ifndef KBSRC_C_H
#define KBSRC_C_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int precision; /* 0 fast, 1 exact, 2 long double (x87 extended, emulated on the GPU), 3 split-precision
                      tensor-core form with int8 digit slices, 4 the same with f16 digit slices (no reference
                      counterpart; float64-level accuracy) */
    double length; /* one-sided kernel length, seconds (reference default 0.2) */
    double beta;   /* Kaiser beta (default 40) */
    int threads;   /* host threads, 0 = automatic */
    int block;     /* block size factor, 0 = automatic */
    int lpc_edges; /* nonzero: Burg LPC edges (default) */
} kbsrc_options_c;

typedef struct {
    long long p, q, taps;
    int block, threads, general_fold;
    double design_seconds, process_seconds, passband, stopband;
    const char* isa;
} kbsrc_stats_c;

/* Output frames per channel for a conversion: ceil(frames * P / Q), or -1 on bad arguments. */
long long kbsrc_output_frames(long long frames, int rate_in, int rate_out);

/* Converts. out: planar, channels * out_cap doubles (out[c*out_cap + i]). Returns the output frames per
 * channel (>= 0), or -1 invalid argument, -2 out_cap too small, -3 runtime (GPU) error, -4 out of memory;
 * err (if not NULL) receives the message. */
long long kbsrc_resample_c(const double* in, long long frames, int channels, int rate_in, int rate_out,
                           const kbsrc_options_c* opt, double* out, long long out_cap, kbsrc_stats_c* stats,
                           char* err, int err_len);

const char* kbsrc_version_c(void);

/* A planned conversion: block plan, LPC edges and the GPU engine with the kernel spectrum, built once for
 * input of one shape (frames, channels, rates, options) and run any number of times on such input. */
typedef struct kbsrc_conversion kbsrc_conversion;
struct kbsrc_gpu_engine;

/* Plans a conversion for `in` (its edges feed the LPC prediction). Returns 0, or -1 invalid argument,
 * -3 runtime (GPU) error, -4 out of memory. */
int kbsrc_prepare_c(const double* in, long long frames, int channels, int rate_in, int rate_out,
                    const kbsrc_options_c* opt, kbsrc_conversion** out, char* err, int err_len);
/* Runs it: in as given to kbsrc_prepare_c (interleaved), out planar channels * nout. */
int kbsrc_conversion_run_c(kbsrc_conversion* cv, const double* in, double* out, char* err, int err_len);
/* Output frames, LPC edge arrays (channels * edge_len each) and the engine (NULL for equal rates). */
int kbsrc_conversion_info_c(const kbsrc_conversion* cv, long long* nout, long long* edge_len, const double** head,
                            const double** tail, struct kbsrc_gpu_engine** engine, kbsrc_stats_c* stats);
void kbsrc_conversion_free_c(kbsrc_conversion* cv);

/* Multi-GPU (not in the reference): the block loop split into contiguous block ranges, one per device
 * (kbsrc_gpu_shard_plan in include/kbsrc_gpu.h); each device receives only its input span and returns its output
 * range, nothing moves between devices, and the output equals kbsrc_resample_c's.
 * kbsrc_resample_devices_c: the whole conversion over devices[0..ndevices) (a device may appear more than once),
 *   one host thread per share; arguments and return values as kbsrc_resample_c.
 * kbsrc_prepare_share_c: a conversion whose engine runs share `index` of `count` on the calling thread's current
 *   device (one process per GPU). kbsrc_conversion_run_c then takes the whole interleaved input and writes that
 *   share's output, channels * share.nout doubles; kbsrc_conversion_share_c returns the share (blocks, input
 *   frames, output samples) as six long longs: blk0 blk1 frame0 frames out0 nout (all zero for equal rates). */
long long kbsrc_resample_devices_c(const double* in, long long frames, int channels, int rate_in, int rate_out,
                                   const int* devices, int ndevices, const kbsrc_options_c* opt, double* out,
                                   long long out_cap, kbsrc_stats_c* stats, char* err, int err_len);
int kbsrc_prepare_share_c(const double* in, long long frames, int channels, int rate_in, int rate_out,
                          const kbsrc_options_c* opt, int index, int count, kbsrc_conversion** out, char* err,
                          int err_len);
int kbsrc_conversion_share_c(const kbsrc_conversion* cv, long long* share6);

/* Batches: many conversions (files) of any lengths, channel counts and rate pairs, planned together and run
 * on the GPU as one recorded launch sequence (kbsrc_gpu_batch in include/kbsrc_gpu.h); conversions with equal
 * plans share their kernel design and launches. Each output equals that of kbsrc_resample_c for the item. */
typedef struct {
    const double* in; /* interleaved frames x channels (used for the LPC edges at prepare) */
    long long frames;
    int channels, rate_in, rate_out;
} kbsrc_batch_item_c;
typedef struct kbsrc_batch kbsrc_batch;
int kbsrc_batch_prepare_c(const kbsrc_batch_item_c* items, int count, const kbsrc_options_c* opt,
                          kbsrc_batch** out, char* err, int err_len);
/* in[i]: interleaved input of item i; out[i]: planar output, channels * nout doubles. */
int kbsrc_batch_run_c(kbsrc_batch* b, const double* const* in, double* const* out, char* err, int err_len);
/* Item i: output frames, LPC edges (channels * edge_len each) and its index in the GPU batch (-1: equal rates). */
int kbsrc_batch_info_c(const kbsrc_batch* b, int i, long long* nout, long long* edge_len, const double** head,
                       const double** tail, int* gpu_index);
struct kbsrc_gpu_batch* kbsrc_batch_gpu_c(kbsrc_batch* b);
void kbsrc_batch_free_c(kbsrc_batch* b);

/* Diagnostics: the host-side steps on their own (no GPU needed).
 * kbsrc_plan_c: the block plan of src/resampler.cpp:98-167, info[16] = P Q taps nb marg hop nblk Nb Mb pre o E
 *   lead general up nout; returns 0, 1 (equal rates: copy) or -1 (invalid argument).
 * kbsrc_kernel_taps_c: Kaiser taps h[0..L] of src/design.cpp:17-37 as (hi, lo) pairs.
 * kbsrc_burg_c: the Burg LPC prediction of src/lpc.cpp:13-42. */
int kbsrc_plan_c(long long frames, int channels, int rate_in, int rate_out, const kbsrc_options_c* opt,
                 long long* info, char* err, int err_len);
int kbsrc_kernel_taps_c(int L, long long a, long long b, double beta, int threads, double* out);
int kbsrc_burg_c(const double* x, long long len, long long n, double* out);

#ifdef __cplusplus
}
#endif
#endif
