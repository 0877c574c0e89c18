// sm_100a block engine of the DFT-domain resampler, and its C ABI (include/kbsrc_gpu.h).
//
// One run processes every (channel, block) task of a conversion plan: the overlap-save loop of the
// reference's run_engine (HongYue1/KBSRC src/resampler.cpp:34-88). Per task:
//   forward real FFT of nb*Q points  = gather (staged input + LPC edges) -> complex FFT of h = nb*Q/2 points
//                                      -> split into h+1 real-spectrum bins          (fft.hpp:362-409)
//   spectrum multiply with the kernel, fold (down) or periodic extension (up)        (resampler.cpp:53-78)
//   inverse real FFT of nb*P points  = merge into h' = nb*P/2 complex points -> complex FFT (fft.hpp:411-461)
//   discard the margins and write hop*P output samples                               (resampler.cpp:80-84)
// Complex FFTs of more than 2048 points use the reference's four-step split n = N1*N2 (fft.hpp:267-313):
// a column pass (N2 sequences of N1, stride N2, then the w_n^{k1 n2} twiddle) and a row pass (N1 sequences
// of N2, stored transposed). Each pass is one launch over all tasks of a wave; the sub-FFTs run in shared
// memory (fft.cuh). Smaller FFTs run whole in one CTA.
//
// Arithmetic (dd.cuh): fast = f64; exact = short-add dd in the four-step sub-FFTs and accurate-add dd
// elsewhere; long double = x87 extended emulated in integers (x80.cuh) everywhere, exactly as the reference
// instantiates its templates, so the output is byte-identical.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../host/ddh.hpp"
#include "dd.cuh"
#include "fft.cuh"
#include "kbsrc_gpu.h"
#include "tcfft.cuh"

using namespace kbsrc::dev;
namespace hd = kbsrc::host;

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

#define KB_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t err_ = (call);                                                                      \
        if (err_ != cudaSuccess) return fail(KBSRC_GPU_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(err_)); \
    } while (0)

// ------------------------------------------------------------------------------------------------------
// kernel parameter blocks
// ------------------------------------------------------------------------------------------------------

// One conversion's buffers and placement; a single engine runs one, a batch many.
// The staged channel of the reference (resampler.cpp:168-186) is read without being materialised: zeros, the
// LPC head, the interleaved input, the LPC tail, zeros; frame t of the signal is staged sample t + lead.
// A multi-GPU share holds only part of the input and of the output: `in` starts at frame f0, and `out` holds
// output samples [d0, d0 + ostride) of each channel (a whole conversion: f0 = d0 = 0, ostride = nout).
struct Item {
    const void* in;      // interleaved input, frames [f0, ...) x ch, samples in format `fmt` (KBSRC_GPU_IN_*)
    const double* head;  // ch x edge: head[c*edge + i] is frame -1-i
    const double* tail;  // ch x edge: tail[c*edge + i] is frame frames+i
    double* out;         // planar output, ch x ostride: out[c*ostride + (d - d0)] is output sample d
    long long frames, edge, lead, nout, o;
    int ch;
    int fmt;
    long long f0, d0, ostride;
};

// Which conversion, channel and block a task is.
struct TaskRef {
    int item, c;
    long long b;
};

// The tasks of one launch group: a single conversion (refs == nullptr; task = b * ch + c, so the channels of
// one block run side by side and share the sectors of the interleaved input) or a batch (device tables). The
// order of tasks does not affect any value.
struct Work {
    Item item0;
    const Item* items;
    const TaskRef* refs;
    long long hopQ, hopP, margP;  // block hop in staged samples and output samples, output margin
};

__device__ __forceinline__ TaskRef task_ref(const Work& w, long long task) {
    if (w.refs) return w.refs[task];
    return TaskRef{0, (int)(task % w.item0.ch), task / w.item0.ch};
}
__device__ __forceinline__ Item item_of(const Work& w, const TaskRef& r) { return w.refs ? w.items[r.item] : w.item0; }

// Input sample i (= frame * ch + channel) as the WAV reader delivers it (src/io/wav.cpp:299-362): float64 as
// stored, float32 widened, integer PCM times 2^-(8B-1) (8-bit offset by 128), all exact.
__device__ __forceinline__ double input_at(const Item& s, long long i) {
    switch (s.fmt) {
        case KBSRC_GPU_IN_F64: return __ldg(static_cast<const double*>(s.in) + i);
        case KBSRC_GPU_IN_F32: return (double)__ldg(static_cast<const float*>(s.in) + i);
        case KBSRC_GPU_IN_S32: return __dmul_rn((double)__ldg(static_cast<const int*>(s.in) + i), 0x1p-31);
        case KBSRC_GPU_IN_S24: {
            const unsigned char* p = static_cast<const unsigned char*>(s.in) + 3 * i;
            const int v = (int)__ldg(p) | (int)__ldg(p + 1) << 8 | (int)(signed char)__ldg(p + 2) << 16;
            return __dmul_rn((double)v, 0x1p-23);
        }
        case KBSRC_GPU_IN_S16: return __dmul_rn((double)__ldg(static_cast<const short*>(s.in) + i), 0x1p-15);
        default: return __dmul_rn((double)((int)__ldg(static_cast<const unsigned char*>(s.in) + i) - 128), 0x1p-7);
    }
}

__device__ __forceinline__ double signal_at(const Item& s, int c, long long t) {
    if (t >= 0 && t < s.frames) return input_at(s, (t - s.f0) * s.ch + c);
    if (t < 0 && t >= -s.edge) return __ldg(s.head + c * s.edge + (-1 - t));
    if (t >= s.frames && t < s.frames + s.edge) return __ldg(s.tail + c * s.edge + (t - s.frames));
    return 0.0;
}

// Discard and copy (resampler.cpp:80-84): sample e of block b's inverse FFT lands at b*hopP + e - margP - o
__device__ __forceinline__ void emit(const Work& w, const Item& it, int c, long long b, long long e, double v) {
    const long long k = e - w.margP;
    if (k < 0 || k >= w.hopP) return;
    const long long d = b * w.hopP + k - it.o, j = d - it.d0;
    if (d >= 0 && d < it.nout && j >= 0 && j < it.ostride) it.out[c * it.ostride + j] = v;
}

enum Src { kSrcSignal = 0, kSrcComplex = 1, kSrcDDReal = 2 };
enum Dst { kDstComplex = 0, kDstOutput = 1 };

template <class Ar>
struct PassParams {
    SubPlan sp;                   // the sub-FFT
    int N1, N2, F;                // four-step shape; F sequences per CTA
    const CxW<Ar>* tw_stage;      // stage twiddles of sp
    const CxW<Ar>* tw4;           // four-step twiddles [k1*N2 + n2] (column pass)
    OddRoots<typename Ar::W> odd; // radix 3/5/7 constants
    CxR<Ar>* src;                 // complex input (or output of the column pass), per task `stride`
    CxR<Ar>* dst;
    long long stride;             // complex elements between task slots
    long long task0;              // first task of this launch (blockIdx.y adds)
    Work work;                    // kSrcSignal / kDstOutput: the conversions and their buffers
    const double* ddreal;         // kSrcDDReal: (hi, lo) pairs
    const CxW<Ar>* bc;            // Bluestein chirp (bn entries) and kernel spectrum (bm entries)
    const CxW<Ar>* vf;
    int bn, bm;
};

// Where a task's first pass reads the staged signal: its conversion, channel and the signal frame of real
// sample 0 of the block; interior when no sample of the block needs the edge or padding tests.
struct TaskSource {
    Item it;
    int c;
    long long g0;
    bool interior;
};

__device__ __forceinline__ TaskSource task_source(const Work& w, long long task, long long nreal) {
    const TaskRef r = task_ref(w, task);
    TaskSource t;
    t.it = item_of(w, r);
    t.c = r.c;
    t.g0 = r.b * w.hopQ - t.it.lead;
    t.interior = t.g0 >= 0 && t.g0 + nreal <= t.it.frames;
    return t;
}

// Complex input value i of a task: (x[2i], x[2i+1]) of the staged signal (fft.hpp:363), a buffer value, or a
// dd real pair (kernel design).
template <class Ar, int SRC>
__device__ __forceinline__ CxR<Ar> load_input(const double* ddreal, const TaskSource& ts, const CxR<Ar>* src,
                                              long long i) {
    using R = typename Ar::R;
    if constexpr (SRC == kSrcSignal) {
        const long long t = ts.g0 + 2 * i;
        double x0, x1;
        if (ts.interior) {
            x0 = input_at(ts.it, (t - ts.it.f0) * ts.it.ch + ts.c);
            x1 = input_at(ts.it, (t + 1 - ts.it.f0) * ts.it.ch + ts.c);
        } else {
            x0 = signal_at(ts.it, ts.c, t);
            x1 = signal_at(ts.it, ts.c, t + 1);
        }
        return CxR<Ar>{Ar::from_f64(x0), Ar::from_f64(x1)};
    } else if constexpr (SRC == kSrcComplex) {
        return src[i];
    } else if constexpr (Ar::kWide) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(ddreal) + 2 * i);
        const double2 b = __ldg(reinterpret_cast<const double2*>(ddreal) + 2 * i + 1);
        return CxR<Ar>{R{a.x, a.y}, R{b.x, b.y}};
    } else {
        return CxR<Ar>{ddreal[4 * i], ddreal[4 * i + 2]};
    }
}
template <class Ar, int SRC>
__device__ __forceinline__ CxR<Ar> load_input(const PassParams<Ar>& P, const TaskSource& ts, const CxR<Ar>* src,
                                              long long i) {
    return load_input<Ar, SRC>(P.ddreal, ts, src, i);
}

template <class Ar>
__device__ __forceinline__ CxR<Ar> czero() {
    return CxR<Ar>{Ar::zero(), Ar::zero()};
}

// Loads per thread issued together before their shared-memory stores (memory-level parallelism), for the wide
// types (double-double, extended) and for float64
#ifndef KB_LOAD_BATCH
#define KB_LOAD_BATCH 4
#endif
#ifndef KB_LOAD_BATCH_F64
#define KB_LOAD_BATCH_F64 4
#endif
template <class Ar>
constexpr int kLoadBatch = Ar::kWide ? KB_LOAD_BATCH : KB_LOAD_BATCH_F64;

// Shared memory of a pass: two plane pairs of n*F values, then (double-double) the sub-FFT's stage twiddles.
template <class Ar>
__device__ __forceinline__ CxW<Ar>* twiddle_smem(unsigned char* after_planes) {
    return reinterpret_cast<CxW<Ar>*>(after_planes);
}

// Column pass: sequences n2 in [c0, c0+F) of length N1 (stride N2), twiddle, store in place
// (fft.hpp:283-299). blockIdx.x: column group; blockIdx.y: task slot. Reading the staged signal, the two are
// swapped (task slot fastest): the channels of a block are consecutive tasks, and their CTAs for one column group
// then run side by side and share the interleaved input's sectors in L2.
// One column-pass unit for the batch queue: sequences n2 in [c0, c0+F) of length N1 (stride N2) of one task's slot
// (src, dst), or of the staged signal `ts` (SRC), through the sub-plan sp (in global memory), then the four-step
// twiddle, stored in place (fft.hpp:283-299).
template <class Ar, int SRC>
__device__ __forceinline__ void column_unit(const SubPlan& sp, int N1, int N2, int F, int c0,
                                            const CxW<Ar>* tw_stage, const CxW<Ar>* tw4,
                                            const OddRoots<typename Ar::W>& odd, const CxR<Ar>* src, CxR<Ar>* dst,
                                            const TaskSource& ts, const double* ddreal, unsigned char* smem) {
    using C = CxR<Ar>;
    const int total = N1 * F;
    const FastDiv dF = fast_div(F);
    Planes<Ar> A, B;
    unsigned char* rest = carve<Ar>(smem, total, A, B);
    const auto tws = stage_twiddles<Ar>(sp, tw_stage, twiddle_smem<Ar>(rest));
    for (int e0 = threadIdx.x; e0 < total; e0 += kLoadBatch<Ar> * blockDim.x) {
        C v[kLoadBatch<Ar>];
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, r = (int)fdiv(e, dF), n2 = c0 + (e - r * F);
            if (e < total) v[j] = n2 < N2 ? load_input<Ar, SRC>(ddreal, ts, src, (long long)r * N2 + n2) : czero<Ar>();
        }
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++)
            if (e0 + j * blockDim.x < total) A.st(e0 + j * blockDim.x, v[j]);
    }
    __syncthreads();
    const Planes<Ar> res = stockham<Ar>(sp, A, B, F, tws, odd);
    // four-step twiddle and store; the table loads of a batch are issued before any of its products
    for (int e0 = threadIdx.x; e0 < total; e0 += kLoadBatch<Ar> * blockDim.x) {
        CxW<Ar> w[kLoadBatch<Ar>];
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, k1 = (int)fdiv(e, dF), n2 = c0 + (e - k1 * F);
            if (e < total && n2 < N2 && k1 && (Ar::kLanes || n2)) w[j] = ld_tw(tw4 + (long long)k1 * N2 + n2);
        }
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, k1 = (int)fdiv(e, dF), n2 = c0 + (e - k1 * F);
            if (e >= total || n2 >= N2) continue;
            C v = res.ld(e);
            if (k1 && (Ar::kLanes || n2)) v = c_mulw<Ar>(v, w[j]);
            if (Ar::kLaneRenorm) v = c_renorm<Ar>(v);
            dst[(long long)k1 * N2 + n2] = v;
        }
    }
}

// The per-plan grid kernel runs the same loop as column_unit with every plan value read straight from its
// parameters: a reference to the parameter block would turn those reads into generic loads (C2 exact: forward
// column 1.05 -> 1.10 ms). TWG (double-double and extended): read the stage twiddles from the global table instead
// of a shared-memory copy (the launch shape's choice).
template <class Ar, int SRC, bool TWG>
__global__ void __launch_bounds__(Ar::kColMaxThreads, Ar::kColMinBlocks) k_column(const __grid_constant__ PassParams<Ar> P) {
    extern __shared__ __align__(16) unsigned char smem[];
    using C = CxR<Ar>;
    const int F = P.F, N1 = P.N1, N2 = P.N2, total = N1 * F;
    const FastDiv dF = fast_div(F);
    Planes<Ar> A, B;
    unsigned char* rest = carve<Ar>(smem, total, A, B);
    const unsigned slot = SRC == kSrcSignal ? blockIdx.x : blockIdx.y, group = SRC == kSrcSignal ? blockIdx.y : blockIdx.x;
    const long long task = P.task0 + slot;
    const int c0 = group * F;
    const C* src = P.src + slot * P.stride;
    C* dst = P.dst + slot * P.stride;
    const TaskSource ts = SRC == kSrcSignal ? task_source(P.work, task, 2LL * N1 * N2) : TaskSource{};
    const auto tws = stage_twiddles<Ar, TWG || !Ar::kWide>(P.sp, P.tw_stage, twiddle_smem<Ar>(rest));
    for (int e0 = threadIdx.x; e0 < total; e0 += kLoadBatch<Ar> * blockDim.x) {
        C v[kLoadBatch<Ar>];
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, r = (int)fdiv(e, dF), n2 = c0 + (e - r * F);
            if (e < total) v[j] = n2 < N2 ? load_input<Ar, SRC>(P, ts, src, (long long)r * N2 + n2) : czero<Ar>();
        }
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++)
            if (e0 + j * blockDim.x < total) A.st(e0 + j * blockDim.x, v[j]);
    }
    __syncthreads();
    const Planes<Ar> res = stockham<Ar>(P.sp, A, B, F, tws, P.odd);
    for (int e0 = threadIdx.x; e0 < total; e0 += kLoadBatch<Ar> * blockDim.x) {
        CxW<Ar> w[kLoadBatch<Ar>];
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, k1 = (int)fdiv(e, dF), n2 = c0 + (e - k1 * F);
            if (e < total && n2 < N2 && k1 && (Ar::kLanes || n2)) w[j] = ld_tw(P.tw4 + (long long)k1 * N2 + n2);
        }
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, k1 = (int)fdiv(e, dF), n2 = c0 + (e - k1 * F);
            if (e >= total || n2 >= N2) continue;
            C v = res.ld(e);
            if (k1 && (Ar::kLanes || n2)) v = c_mulw<Ar>(v, w[j]);
            if (Ar::kLaneRenorm) v = c_renorm<Ar>(v);
            dst[(long long)k1 * N2 + n2] = v;
        }
    }
}

// Row pass: rows r in [r0, r0+F) of length N2 (contiguous), stored transposed to [N1*k2 + r]
// (fft.hpp:300-311), or written straight to the output as real samples (fft.hpp:459-460).
// One row-pass unit for the batch queue: rows r in [r0, r0+F) of length N2 of one task's slot through sp, stored
// transposed to dst[N1*k2 + r], or written to the output as real samples (DST; `work` and the task place them)
// (fft.hpp:300-311,459-460).
template <class Ar, int DST>
__device__ __forceinline__ void row_unit(const SubPlan& sp, int N1, int N2, int F, int r0, const CxW<Ar>* tw_stage,
                                         const OddRoots<typename Ar::W>& odd, const CxR<Ar>* src, CxR<Ar>* dst,
                                         const Work& work, long long task, unsigned char* smem) {
    using C = CxR<Ar>;
    const int total = N2 * F;
    const FastDiv dF = fast_div(F), dN2 = fast_div(N2);
    Planes<Ar> A, B;
    unsigned char* rest = carve<Ar>(smem, total, A, B);
    const auto tws = stage_twiddles<Ar>(sp, tw_stage, twiddle_smem<Ar>(rest));
    for (int e0 = threadIdx.x; e0 < total; e0 += kLoadBatch<Ar> * blockDim.x) {
        C v[kLoadBatch<Ar>];
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, f = (int)fdiv(e, dN2), i = e - f * N2, row = r0 + f;
            if (e < total) v[j] = row < N1 ? src[(long long)row * N2 + i] : czero<Ar>();
        }
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, f = (int)fdiv(e, dN2), i = e - f * N2;
            if (e < total) A.st(i * F + f, v[j]);
        }
    }
    __syncthreads();
    const Planes<Ar> res = stockham<Ar>(sp, A, B, F, tws, odd);
    const TaskRef tr = DST == kDstOutput ? task_ref(work, task) : TaskRef{0, 0, 0};
    const Item it = DST == kDstOutput ? item_of(work, tr) : Item{};
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int k2 = (int)fdiv(e, dF), f = e - k2 * F, row = r0 + f;
        if (row >= N1) continue;
        C v = res.ld(e);
        if (Ar::kLaneRenorm) v = c_renorm<Ar>(v);
        const long long iz = (long long)N1 * k2 + row;
        if (DST == kDstComplex) {
            dst[iz] = v;
        } else {
            emit(work, it, tr.c, tr.b, 2 * iz, Ar::to_f64(v.re));
            emit(work, it, tr.c, tr.b, 2 * iz + 1, Ar::to_f64(Ar::neg(v.im)));
        }
    }
}

// The per-plan grid kernel: row_unit's loop with the plan read straight from the parameters (see k_column).
template <class Ar, int DST, bool TWG>
__global__ void __launch_bounds__(Ar::kMaxThreads, Ar::kMinBlocks) k_row(const __grid_constant__ PassParams<Ar> P) {
    extern __shared__ __align__(16) unsigned char smem[];
    using C = CxR<Ar>;
    const int F = P.F, N1 = P.N1, N2 = P.N2, total = N2 * F;
    const FastDiv dF = fast_div(F), dN2 = fast_div(N2);
    Planes<Ar> A, B;
    unsigned char* rest = carve<Ar>(smem, total, A, B);
    const long long task = P.task0 + blockIdx.y;
    const int r0 = blockIdx.x * F;
    const C* src = P.src + blockIdx.y * P.stride;
    const auto tws = stage_twiddles<Ar, TWG || !Ar::kWide>(P.sp, P.tw_stage, twiddle_smem<Ar>(rest));
    for (int e0 = threadIdx.x; e0 < total; e0 += kLoadBatch<Ar> * blockDim.x) {
        C v[kLoadBatch<Ar>];
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, f = (int)fdiv(e, dN2), i = e - f * N2, row = r0 + f;
            if (e < total) v[j] = row < N1 ? src[(long long)row * N2 + i] : czero<Ar>();
        }
#pragma unroll
        for (int j = 0; j < kLoadBatch<Ar>; j++) {
            const int e = e0 + j * blockDim.x, f = (int)fdiv(e, dN2), i = e - f * N2;
            if (e < total) A.st(i * F + f, v[j]);
        }
    }
    __syncthreads();
    const Planes<Ar> res = stockham<Ar>(P.sp, A, B, F, tws, P.odd);
    C* dst = P.dst + blockIdx.y * P.stride;
    const TaskRef tr = DST == kDstOutput ? task_ref(P.work, task) : TaskRef{0, 0, 0};
    const Item it = DST == kDstOutput ? item_of(P.work, tr) : Item{};
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int k2 = (int)fdiv(e, dF), f = e - k2 * F, row = r0 + f;
        if (row >= N1) continue;
        C v = res.ld(e);
        if (Ar::kLaneRenorm) v = c_renorm<Ar>(v);
        const long long iz = (long long)N1 * k2 + row;
        if (DST == kDstComplex) {
            dst[iz] = v;
        } else {
            emit(P.work, it, tr.c, tr.b, 2 * iz, Ar::to_f64(v.re));
            emit(P.work, it, tr.c, tr.b, 2 * iz + 1, Ar::to_f64(Ar::neg(v.im)));
        }
    }
}

// Whole FFT of n <= 2048 points in one CTA (the reference's direct SFFT path, fft.hpp:241-244,279).
template <class Ar, int SRC, int DST>
__global__ void __launch_bounds__(Ar::kMaxThreads, Ar::kMinBlocks) k_direct(const __grid_constant__ PassParams<Ar> P) {
    extern __shared__ __align__(16) unsigned char smem[];
    using C = CxR<Ar>;
    const int n = P.sp.n;
    Planes<Ar> A, B;
    unsigned char* rest = carve<Ar>(smem, n, A, B);
    const long long task = P.task0 + blockIdx.y;
    const C* src = P.src + blockIdx.y * P.stride;
    const TaskSource ts = SRC == kSrcSignal ? task_source(P.work, task, 2LL * n) : TaskSource{};
    const auto tws = stage_twiddles<Ar>(P.sp, P.tw_stage, twiddle_smem<Ar>(rest));
    for (int i = threadIdx.x; i < n; i += blockDim.x) A.st(i, load_input<Ar, SRC>(P, ts, src, i));
    __syncthreads();
    const Planes<Ar> res = stockham<Ar>(P.sp, A, B, 1, tws, P.odd);
    C* dst = P.dst + blockIdx.y * P.stride;
    const TaskRef tr = DST == kDstOutput ? task_ref(P.work, task) : TaskRef{0, 0, 0};
    const Item it = DST == kDstOutput ? item_of(P.work, tr) : Item{};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const C v = res.ld(i);
        if (DST == kDstComplex) {
            dst[i] = v;
        } else {
            emit(P.work, it, tr.c, tr.b, 2LL * i, Ar::to_f64(v.re));
            emit(P.work, it, tr.c, tr.b, 2LL * i + 1, Ar::to_f64(Ar::neg(v.im)));
        }
    }
}

// Bluestein (chirp-z) steps for lengths that are not 7-smooth (fft.hpp:268-277), n points through an m-point
// smooth transform: u = x conj(b) zero-padded to m; U = FFT(u); A = conj(U Vf); C = FFT(A); y = conj(C) conj(b).
// Scalar arithmetic (accurate dd in exact).
template <class Ar, int SRC>
__global__ void k_blue_pre(const __grid_constant__ PassParams<Ar> P) {
    using C = CxR<Ar>;
    const long long task = P.task0 + blockIdx.y;
    const C* src = P.src + blockIdx.y * P.stride;
    C* dst = P.dst + blockIdx.y * P.stride;
    const TaskSource ts = SRC == kSrcSignal ? task_source(P.work, task, 2LL * P.bn) : TaskSource{};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < P.bm; j += gridDim.x * blockDim.x) {
        if (j < P.bn) {
            const CxW<Ar> b = ld_tw(P.bc + j);
            dst[j] = c_mulw<Ar>(load_input<Ar, SRC>(P, ts, src, j), CxW<Ar>{b.re, w_neg(b.im)});
        } else {
            dst[j] = czero<Ar>();
        }
    }
}

template <class Ar>
__global__ void k_blue_mid(const __grid_constant__ PassParams<Ar> P) {
    const CxR<Ar>* src = P.src + blockIdx.y * P.stride;
    CxR<Ar>* dst = P.dst + blockIdx.y * P.stride;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P.bm; k += gridDim.x * blockDim.x)
        dst[k] = c_conj<Ar>(c_mulw<Ar>(src[k], ld_tw(P.vf + k)));
}

template <class Ar, int DST>
__global__ void k_blue_post(const __grid_constant__ PassParams<Ar> P) {
    using C = CxR<Ar>;
    const long long task = P.task0 + blockIdx.y;
    const C* src = P.src + blockIdx.y * P.stride;
    C* dst = P.dst + blockIdx.y * P.stride;
    const TaskRef tr = DST == kDstOutput ? task_ref(P.work, task) : TaskRef{0, 0, 0};
    const Item it = DST == kDstOutput ? item_of(P.work, tr) : Item{};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P.bn; k += gridDim.x * blockDim.x) {
        const CxW<Ar> w = ld_tw(P.bc + k);
        const C y = c_mulw<Ar>(c_conj<Ar>(src[k]), CxW<Ar>{w.re, w_neg(w.im)});
        if (DST == kDstComplex) {
            dst[k] = y;
        } else {
            emit(P.work, it, tr.c, tr.b, 2LL * k, Ar::to_f64(y.re));
            emit(P.work, it, tr.c, tr.b, 2LL * k + 1, Ar::to_f64(Ar::neg(y.im)));
        }
    }
}

// ------------------------------------------------------------------------------------------------------
// real-FFT split, spectrum, real-FFT merge
// ------------------------------------------------------------------------------------------------------
template <class Ar>
struct SpecParams {
    const CxR<Ar>* Z;    // forward complex FFT output, h per task
    CxR<Ar>* X;          // forward spectrum, h+1 per task
    CxR<Ar>* Zi;         // inverse complex FFT input, hi per task
    long long stride;
    const CxW<Ar>* w_fw; // e^{-2 pi i k/Nb}, k <= h
    const CxW<Ar>* w_iv; // e^{-2 pi i k/Mb}, k <= hi
    const typename Ar::W* H;
    int h, hi;           // Nb/2 and Mb/2
    int Nb, Mb, up;
    int Jg;              // general-fold bin limit, 0 otherwise
    double scale;        // kernel design: H = X.re / scale
    typename Ar::W* Hout;
};

// X[k] = (E + O w[k]) / 2 with E = z[k] + conj z[h-k], O = -i (z[k] - conj z[h-k]) (fft.hpp:365-408).
// Double-double computes conjugate pairs together (one E, O for k and h-k); f64 computes each k alone.
// Bins k = k0, k0 + step, ... <= k_end of one task's split (Z -> X); the last bin a task needs is split_last.
template <class Ar>
__device__ __forceinline__ int split_last(int h) {
    return Ar::kWide ? h / 2 : h - 1;
}
template <class Ar>
__device__ __forceinline__ void split_range(const SpecParams<Ar>& P, const CxR<Ar>* Z, CxR<Ar>* X, int k0, int k_end,
                                            int step) {
    using C = CxR<Ar>;
    const int h = P.h;
    const typename Ar::R half = Ar::from_f64(0.5);
    for (int k = k0; k <= k_end; k += step) {
        if (k == 0) {
            const C z0 = Z[0];
            X[0] = C{Ar::add(z0.re, z0.im), Ar::zero()};
            X[h] = C{Ar::sub(z0.re, z0.im), Ar::zero()};
            continue;
        }
        const int j = h - k;
        const C a = Z[k], bb = c_conj<Ar>(Z[j]);
        const C E = c_add<Ar>(a, bb), O = c_mul_mi<Ar>(c_sub<Ar>(a, bb));
        const C v = c_add<Ar>(E, c_mulw<Ar>(O, ld_tw(P.w_fw + k)));
        X[k] = c_scale<Ar>(v, half);
        if (Ar::kWide && j != k) {
            const C u = c_add<Ar>(c_conj<Ar>(E), c_mulw<Ar>(c_conj<Ar>(O), ld_tw(P.w_fw + j)));
            X[j] = c_scale<Ar>(u, half);
        }
    }
}

template <class Ar>
__global__ void k_split(const __grid_constant__ SpecParams<Ar> P) {
    split_range<Ar>(P, P.Z + blockIdx.y * P.stride, P.X + blockIdx.y * P.stride, blockIdx.x * blockDim.x + threadIdx.x,
                    split_last<Ar>(P.h), gridDim.x * blockDim.x);
}

template <class W>
__device__ __forceinline__ W ld_w(const W* p) {
    return __ldg(p);
}
template <>
__device__ __forceinline__ dd ld_w<dd>(const dd* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    return dd{a.x, a.y};
}
template <>
__device__ __forceinline__ x80 ld_w<x80>(const x80* p) {
    const longlong2 a = __ldg(reinterpret_cast<const longlong2*>(p));
    return x80{(unsigned long long)a.x, (int)a.y, 0};
}

// The forward spectrum X[j] (j <= h) as the spectrum step reads it: from the split pass's output buffer ...
template <class Ar>
struct SpectrumBuf {
    const CxR<Ar>* X;
    __device__ __forceinline__ CxR<Ar> operator()(int j) const { return X[j]; }
};

// ... or, in float64, computed from the complex spectrum Z where it is needed: the float64 split computes every bin
// alone by the same operations (fft.hpp:377-407), so a bin's value does not depend on the pass that computes it,
// and the spectrum step can read Z directly instead of a stored copy of X (one pass and 2 x (h+1) values of HBM
// traffic per task fewer).
template <class Ar>
struct SpectrumFromZ {
    static_assert(!Ar::kWide, "the wide types split conjugate pairs together");
    const CxR<Ar>* Z;
    const CxW<Ar>* w_fw;
    int h;
    __device__ __forceinline__ CxR<Ar> operator()(int k) const {
        using C = CxR<Ar>;
        if (k == 0 || k == h) {
            const C z0 = Z[0];
            return C{k ? Ar::sub(z0.re, z0.im) : Ar::add(z0.re, z0.im), Ar::zero()};
        }
        const C a = Z[k], bb = c_conj<Ar>(Z[h - k]);
        const C E = c_add<Ar>(a, bb), O = c_mul_mi<Ar>(c_sub<Ar>(a, bb));
        const C v = c_add<Ar>(E, c_mulw<Ar>(O, ld_tw(w_fw + k)));
        return c_scale<Ar>(v, Ar::from_f64(0.5));
    }
};

// Y[k]: spectrum multiply with fold (down) or periodic extension (up) (resampler.cpp:64-78); X(j) is the forward
// spectrum (SpectrumBuf or SpectrumFromZ).
template <class Ar, class XS>
__device__ __forceinline__ CxR<Ar> spectrum_bin(const SpecParams<Ar>& P, const XS& X, int k) {
    using C = CxR<Ar>;
    const int Nb = P.Nb, Mb = P.Mb;
    if (P.Jg) {
        // General fold (resampler.cpp:53-63): bin j <= Jg of the true kernel response lands on j mod Mb, on
        // Mb - (j mod Mb) conjugated when above Mb/2, and bins 0 and Mb/2 take twice the real part (bin j = 0
        // whole). Bin k collects j = k, Mb-k, Mb+k, 2Mb-k, ... in that (increasing) order, as the loop over j did.
        const bool edge = k == 0 || 2 * k == Mb;
        C y = czero<Ar>();
        auto take = [&](long long j, bool mirrored) {
            const int jj = (int)(j % Nb);
            const C x = jj <= Nb / 2 ? X(jj) : c_conj<Ar>(X(Nb - jj));
            const C v = c_scale<Ar>(x, Ar::from_w(ld_w(P.H + j)));
            if (j == 0) y = c_add<Ar>(y, v);
            else if (edge) y.re = Ar::add(y.re, Ar::mul(Ar::from_f64(2.0), v.re));
            else y = c_add<Ar>(y, mirrored ? c_conj<Ar>(v) : v);
        };
        for (long long base = 0; base + k <= P.Jg; base += Mb) {
            take(base + k, false);
            if (!edge && base + Mb - k <= P.Jg) take(base + Mb - k, true);
        }
        if (edge) y.im = Ar::zero();
        return y;
    }
    if (P.up) {
        const int kk = k % Nb;
        const C v = kk <= Nb / 2 ? X(kk) : c_conj<Ar>(X(Nb - kk));
        C y = c_scale<Ar>(v, Ar::from_w(ld_w(P.H + k)));
        if (2 * k == Mb) y.im = Ar::zero();
        return y;
    }
    if (2 * k == Mb)
        return C{Ar::mul(Ar::mul(Ar::from_f64(2.0), X(k).re), Ar::from_w(ld_w(P.H + k))), Ar::zero()};
    C y = c_scale<Ar>(X(k), Ar::from_w(ld_w(P.H + k)));
    const int j = Mb - k, jmax = min(Nb / 2, Mb - 1);
    if (k >= 1 && j <= jmax) {  // j >= Mb/2 + 1 = K holds for every k < Mb/2
        const C v = c_scale<Ar>(X(j), Ar::from_w(ld_w(P.H + j)));
        y = c_add<Ar>(y, c_conj<Ar>(v));
    }
    return y;
}

// Inverse merge z[k] = conj(E + i D), E = Y[k] + conj Y[hi-k], D = (Y[k] - conj Y[hi-k]) conj w[k]
// (fft.hpp:411-458); pairs in dd, each k alone in f64.
template <class Ar, class XS>
__device__ __forceinline__ void merge_range(const SpecParams<Ar>& P, const XS& X, CxR<Ar>* Zi, int k0, int k_end,
                                            int step) {
    using C = CxR<Ar>;
    const int hi = P.hi;
    for (int k = k0; k <= k_end; k += step) {
        const int j = hi - k;
        const C a = spectrum_bin<Ar>(P, X, k), bb = c_conj<Ar>(spectrum_bin<Ar>(P, X, j));
        const C E = c_add<Ar>(a, bb), split = c_sub<Ar>(a, bb);
        const CxW<Ar> wk = ld_tw(P.w_iv + k);
        const C D = c_mulw<Ar>(split, CxW<Ar>{wk.re, w_neg(wk.im)});
        const C v = {Ar::sub(E.re, D.im), Ar::add(E.im, D.re)};
        Zi[k] = c_conj<Ar>(v);
        if (Ar::kWide && k && j != k) {
            const C Ej = c_conj<Ar>(E);
            const CxW<Ar> wj = ld_tw(P.w_iv + j);
            const C Dj = c_mulw<Ar>(C{Ar::neg(split.re), split.im}, CxW<Ar>{wj.re, w_neg(wj.im)});
            const C u = {Ar::sub(Ej.re, Dj.im), Ar::add(Ej.im, Dj.re)};
            Zi[j] = c_conj<Ar>(u);
        }
    }
}

template <class Ar>
__global__ void k_merge(const __grid_constant__ SpecParams<Ar> P) {
    merge_range<Ar>(P, SpectrumBuf<Ar>{P.X + blockIdx.y * P.stride}, P.Zi + blockIdx.y * P.stride,
                    blockIdx.x * blockDim.x + threadIdx.x, split_last<Ar>(P.hi), gridDim.x * blockDim.x);
}

// Float64 split, spectrum multiply and merge in one pass: Z (forward complex FFT) -> Zi (inverse input), with the
// forward spectrum computed from Z bin by bin as the spectrum step needs it. Zi must not alias Z.
template <class Ar>
__global__ void k_spectrum_z(const __grid_constant__ SpecParams<Ar> P) {
    merge_range<Ar>(P, SpectrumFromZ<Ar>{P.Z + blockIdx.y * P.stride, P.w_fw, P.h}, P.Zi + blockIdx.y * P.stride,
                    blockIdx.x * blockDim.x + threadIdx.x, split_last<Ar>(P.hi), gridDim.x * blockDim.x);
}

// dd / double (double_double.hpp:80-84) with IEEE division
__device__ __forceinline__ dd div_dd_f64(dd a, double b) {
    auto mul_f64 = [](dd x, double y) {
        const double p = __dmul_rn(x.hi, y);
        double e = __fma_rn(x.hi, y, -p);
        e = __dadd_rn(e, __dmul_rn(x.lo, y));
        return qts(p, e);
    };
    const double q1 = __ddiv_rn(a.hi, b);
    dd r = add_accurate(a, dd_neg(mul_f64(dd{b, 0.0}, q1)));
    const double q2 = __ddiv_rn(r.hi, b);
    r = add_accurate(r, dd_neg(mul_f64(dd{b, 0.0}, q2)));
    const double q3 = __ddiv_rn(r.hi, b);
    return add_accurate(qts(q1, q2), dd{q3, 0.0});
}

// Kernel design: H[k] = X[k].re / scale (design.cpp:46-47)
__global__ void k_design_out(const __grid_constant__ SpecParams<ArDDAccurate> P) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= P.h; k += gridDim.x * blockDim.x)
        P.Hout[k] = div_dd_f64(P.X[k].re, P.scale);
}

// ------------------------------------------------------------------------------------------------------
// batch queue: the tasks of every plan group of a batch wave through one persistent launch per pass
// ------------------------------------------------------------------------------------------------------
// The reference hands (channel, block) tasks to its workers through one atomic counter (src/resampler.cpp:42-49,
// src/parallel.cpp:9-32). Here each pass of a batch wave is one persistent launch whose CTAs take work units from
// an atomic counter: a unit is one column or row group of one task, or a range of spectrum bins, of any plan group.
// Units are listed largest transform first, so the long units start early and the short ones fill in at the end.

// One plan group as the queue kernels read it (four-step forward and inverse transforms, split/merge roots,
// kernel spectrum, block hop); W: the table type.
struct QueueGroup {
    SubPlan fs1, fs2, is1, is2;
    int fN1, fN2, iN1, iN2;
    int fcF, frF, icF, irF;  // sequences per unit: forward column, forward row, inverse column, inverse row
    const void* ftw_stage;
    const void* ftw4;
    const void* itw_stage;
    const void* itw4;
    const void* w_fw;
    const void* w_iv;
    const void* H;
    int h, hi, Nb, Mb, up, Jg;
    long long hopQ, hopP, margP;
};
// One task of a wave: its conversion, channel and block, its plan group, and its slot in the wave buffers (the
// first complex element of its slot; slots of different groups have different sizes).
struct QueueTask {
    TaskRef ref;
    int group;
    long long slot;
};
struct QueueUnit {
    int task, unit;
};
constexpr int kQueueBins = 1024;      // spectrum bins per split or merge unit
constexpr int kQueueBinThreads = 256;

template <class W>
struct QueueParams {
    const QueueGroup* groups;
    const QueueTask* tasks;
    const QueueUnit* units;
    int nunits;
    int* counter;       // next unit (zero before the launch)
    const Item* items;  // the batch's conversions
    void* A;            // wave buffers
    void* B;
    OddRoots<W> odd;
};

// A CTA's place in a queue pass: the unit it works on (in shared memory, so that the whole CTA agrees on it) and
// the next one, claimed from the counter and fetched by thread 0 while the CTA works on the current one, so that
// the dependent loads of the unit and task descriptors overlap the work instead of preceding it.
struct QueueSlot {
    int u;
    QueueUnit qu;
    QueueTask t;
};
template <class W>
struct QueueCursor {
    const QueueParams<W>& Q;
    QueueSlot& cur;  // shared memory
    QueueSlot nxt;   // thread 0
    __device__ __forceinline__ void claim() {
        nxt.u = atomicAdd(Q.counter, 1);
        if (nxt.u < Q.nunits) {
            nxt.qu = Q.units[nxt.u];
            nxt.t = Q.tasks[nxt.qu.task];
        }
    }
    // the first unit; ends with the CTA synchronised
    __device__ __forceinline__ void start() {
        if (threadIdx.x == 0) {
            claim();
            cur = nxt;
        }
        __syncthreads();
    }
    // claim and fetch the unit after the current one (thread 0; the loads complete while the CTA works)
    __device__ __forceinline__ void prefetch() {
        if (threadIdx.x == 0) claim();
    }
    // the current unit is done: move to the prefetched one; ends with the CTA synchronised
    __device__ __forceinline__ void advance() {
        __syncthreads();
        if (threadIdx.x == 0) cur = nxt;
        __syncthreads();
    }
};

// Copies a unit's sub-FFT plan from the group table to shared memory, where the pass's stage loops read it (from
// the group table in global memory every read of the plan would be a load; the per-plan kernels have it in their
// parameters). Ends with the CTA synchronised.
__device__ __forceinline__ void queue_plan(const SubPlan& from, SubPlan& to) {
    static_assert(sizeof(SubPlan) % 4 == 0, "SubPlan is copied as 32-bit words");
    constexpr int kWords = (int)(sizeof(SubPlan) / 4);
    const int* src = reinterpret_cast<const int*>(&from);
    int* dst = reinterpret_cast<int*>(&to);
    for (int i = threadIdx.x; i < kWords; i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
}

// The Work view of one queue task: its conversion as the only item (task = b * ch + c), the group's hop.
__device__ __forceinline__ Work queue_work(const QueueGroup& g, const Item* items, const QueueTask& t, long long& task) {
    Work w{};
    w.item0 = items[t.ref.item];
    w.hopQ = g.hopQ;
    w.hopP = g.hopP;
    w.margP = g.margP;
    task = t.ref.b * w.item0.ch + t.ref.c;
    return w;
}

// Column pass: forward (reads the signal, writes buffer A in place) or inverse (buffer B in place).
template <class Ar, int SRC, bool FWD>
__global__ void __launch_bounds__(Ar::kColMaxThreads, Ar::kColMinBlocks)
    k_column_q(const __grid_constant__ QueueParams<typename Ar::W> Q) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ QueueSlot slot;
    __shared__ SubPlan sp;
    using C = CxR<Ar>;
    QueueCursor<typename Ar::W> qc{Q, slot};
    for (qc.start(); slot.u < Q.nunits; qc.advance()) {
        const QueueUnit qu = slot.qu;
        const QueueTask t = slot.t;
        qc.prefetch();
        const QueueGroup& g = Q.groups[t.group];
        queue_plan(FWD ? g.fs1 : g.is1, sp);
        const int N1 = FWD ? g.fN1 : g.iN1, N2 = FWD ? g.fN2 : g.iN2, F = FWD ? g.fcF : g.icF;
        C* x = static_cast<C*>(FWD ? Q.A : Q.B) + t.slot;
        long long task;
        const Work w = queue_work(g, Q.items, t, task);
        const TaskSource ts = SRC == kSrcSignal ? task_source(w, task, 2LL * N1 * N2) : TaskSource{};
        column_unit<Ar, SRC>(sp, N1, N2, F, qu.unit * F,
                             static_cast<const CxW<Ar>*>(FWD ? g.ftw_stage : g.itw_stage),
                             static_cast<const CxW<Ar>*>(FWD ? g.ftw4 : g.itw4), Q.odd, x, x, ts, nullptr, smem);
    }
}

// Row pass: forward (buffer A to B, natural order) or inverse (buffer B to the output samples).
template <class Ar, int DST, bool FWD>
__global__ void __launch_bounds__(Ar::kMaxThreads, Ar::kMinBlocks)
    k_row_q(const __grid_constant__ QueueParams<typename Ar::W> Q) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ QueueSlot slot;
    __shared__ SubPlan sp;
    using C = CxR<Ar>;
    QueueCursor<typename Ar::W> qc{Q, slot};
    for (qc.start(); slot.u < Q.nunits; qc.advance()) {
        const QueueUnit qu = slot.qu;
        const QueueTask t = slot.t;
        qc.prefetch();
        const QueueGroup& g = Q.groups[t.group];
        queue_plan(FWD ? g.fs2 : g.is2, sp);
        const int N1 = FWD ? g.fN1 : g.iN1, N2 = FWD ? g.fN2 : g.iN2, F = FWD ? g.frF : g.irF;
        long long task;
        const Work w = queue_work(g, Q.items, t, task);
        const C* src = static_cast<const C*>(FWD ? Q.A : Q.B) + t.slot;
        C* dst = static_cast<C*>(Q.B) + t.slot;
        row_unit<Ar, DST>(sp, N1, N2, F, qu.unit * F,
                          static_cast<const CxW<Ar>*>(FWD ? g.ftw_stage : g.itw_stage), Q.odd, src, dst, w, task, smem);
    }
}

template <class Ar>
__device__ __forceinline__ SpecParams<Ar> queue_spec(const QueueGroup& g) {
    SpecParams<Ar> s{};
    s.w_fw = static_cast<const CxW<Ar>*>(g.w_fw);
    s.w_iv = static_cast<const CxW<Ar>*>(g.w_iv);
    s.H = static_cast<const typename Ar::W*>(g.H);
    s.h = g.h; s.hi = g.hi; s.Nb = g.Nb; s.Mb = g.Mb; s.up = g.up; s.Jg = g.Jg;
    return s;
}

// Real-FFT split (buffer B to A, bins of one unit) or spectrum multiply and merge (buffer A to B).
template <class Ar, bool SPLIT>
__global__ void __launch_bounds__(kQueueBinThreads) k_bins_q(const __grid_constant__ QueueParams<typename Ar::W> Q) {
    __shared__ QueueSlot slot;
    using C = CxR<Ar>;
    QueueCursor<typename Ar::W> qc{Q, slot};
    for (qc.start(); slot.u < Q.nunits; qc.advance()) {
        const QueueUnit qu = slot.qu;
        const QueueTask t = slot.t;
        qc.prefetch();
        const QueueGroup& g = Q.groups[t.group];
        const SpecParams<Ar> sp = queue_spec<Ar>(g);
        const int k0 = qu.unit * kQueueBins, last = split_last<Ar>(SPLIT ? g.h : g.hi);
        const int k_end = min(last, k0 + kQueueBins - 1);
        if (SPLIT)
            split_range<Ar>(sp, static_cast<const C*>(Q.B) + t.slot, static_cast<C*>(Q.A) + t.slot,
                            k0 + (int)threadIdx.x, k_end, blockDim.x);
        else
            merge_range<Ar>(sp, SpectrumBuf<Ar>{static_cast<const C*>(Q.A) + t.slot}, static_cast<C*>(Q.B) + t.slot,
                            k0 + (int)threadIdx.x, k_end, blockDim.x);
    }
}

// ------------------------------------------------------------------------------------------------------
// split-precision form: the four-step passes with tensor-core sub-FFTs (tcfft.cuh), float64 everywhere else
// ------------------------------------------------------------------------------------------------------
struct TcParams {
    TcSub sub;
    const double2* tw4;  // four-step twiddles [k1 * N2 + n2] of the column pass (null: none)
    int N1, N2;
    int slots;           // task slots of the launch (items = groups x slots)
    int* err;            // set when a tensor-core stage timed out
};

// Column pass, persistent: each CTA sets up its tensor memory and tables once, then takes items (column group
// g, task slot y) in turn, item = y * groups + g (reading the signal: item = g * slots + y). An item: sequences
// n2 in [c0, c0+F) of length N1 (stride N2) through the sub-FFT, its first stage reading the input straight from
// global memory and its last stage storing, with the four-step twiddle, straight to global memory (in place);
// with N2 == 1 the single column is the whole transform and DST may write it as output samples. S: the digit
// slices' element kind (TcI8 or TcF16). H: items in flight per CTA (1, or 2: one per half of the CTA, which take
// alternate items of the CTA's share).
template <class S, int SRC, int DST, int H>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_tc_column(const __grid_constant__ PassParams<ArF64> P, const __grid_constant__ TcParams T) {
    extern __shared__ __align__(16) unsigned char smem[];
    using C = CxR<ArF64>;
    constexpr int kT = kTcThreads / H;
    const int F = T.sub.F, N1 = T.N1, N2 = T.N2, groups = (N2 + F - 1) / F;
    const TcSmem m = tc_carve(smem, T.sub);
    const uint32_t tmem = tc_setup(m, T.sub);
    const TcHalf hf = tc_half(m, T.sub, H == 2 ? (int)(threadIdx.x >> 8) : 0, tmem);
    uint32_t phase = 0;
    for (long long item = blockIdx.x + (long long)hf.id * gridDim.x; item < (long long)groups * T.slots;
         item += (long long)H * gridDim.x) {
        // reading the signal, the task slot varies fastest: the channels of a block share input sectors in L2
        const int slot = SRC == kSrcSignal ? (int)(item % T.slots) : (int)(item / groups);
        const int c0 = (SRC == kSrcSignal ? (int)(item / T.slots) : (int)(item - (long long)slot * groups)) * F;
        const long long task = P.task0 + slot;
        const C* src = P.src + slot * P.stride;
        C* dst = P.dst + slot * P.stride;
        const TaskSource ts = SRC == kSrcSignal ? task_source(P.work, task, 2LL * N1 * N2) : TaskSource{};
        const TaskRef tr = DST == kDstOutput ? task_ref(P.work, task) : TaskRef{0, 0, 0};
        const Item it = DST == kDstOutput ? item_of(P.work, tr) : Item{};
        tc_subfft<S, kT>(
            T.sub, true, hf, phase, T.err,
            [&](int n, int f) {
                const int n2 = c0 + f;
                if (n2 >= N2) return make_double2(0.0, 0.0);
                const C v = load_input<ArF64, SRC>(P, ts, src, (long long)n * N2 + n2);
                return make_double2(v.re, v.im);
            },
            [&](int k1, int f, double re, double im) {
                const int n2 = c0 + f;
                if (n2 >= N2) return;
                if (DST == kDstComplex) {
                    const long long i = (long long)k1 * N2 + n2;
                    double2 y = make_double2(re, im);
                    if (T.tw4) y = tc_cmul(re, im, __ldg(T.tw4 + i));
                    dst[i] = C{y.x, y.y};
                } else {
                    emit(P.work, it, tr.c, tr.b, 2LL * k1, re);
                    emit(P.work, it, tr.c, tr.b, 2LL * k1 + 1, -im);
                }
            });
    }
    tc_teardown(tmem);
}

// Row pass, persistent like the column pass: items (row group g, task slot y); an item transforms rows r in
// [r0, r0+F) of length N2 (its first stage reading them from global memory, neighbouring rows of the MMA taking
// neighbouring inputs) and stores them transposed to [N1*k2 + r], or writes them as output samples.
template <class S, int DST, int H>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_tc_row(const __grid_constant__ PassParams<ArF64> P, const __grid_constant__ TcParams T) {
    extern __shared__ __align__(16) unsigned char smem[];
    using C = CxR<ArF64>;
    constexpr int kT = kTcThreads / H;
    const int F = T.sub.F, N1 = T.N1, N2 = T.N2, groups = (N1 + F - 1) / F;
    const TcSmem m = tc_carve(smem, T.sub);
    const uint32_t tmem = tc_setup(m, T.sub);
    const TcHalf hf = tc_half(m, T.sub, H == 2 ? (int)(threadIdx.x >> 8) : 0, tmem);
    uint32_t phase = 0;
    for (long long item = blockIdx.x + (long long)hf.id * gridDim.x; item < (long long)groups * T.slots;
         item += (long long)H * gridDim.x) {
        const int slot = (int)(item / groups), r0 = (int)(item - (long long)slot * groups) * F;
        const long long task = P.task0 + slot;
        const C* src = P.src + slot * P.stride;
        C* dst = P.dst + slot * P.stride;
        const TaskRef tr = DST == kDstOutput ? task_ref(P.work, task) : TaskRef{0, 0, 0};
        const Item it = DST == kDstOutput ? item_of(P.work, tr) : Item{};
        tc_subfft<S, kT>(
            T.sub, false, hf, phase, T.err,
            [&](int n, int f) {
                const int row = r0 + f;
                if (row >= N1) return make_double2(0.0, 0.0);
                const C v = src[(long long)row * N2 + n];
                return make_double2(v.re, v.im);
            },
            [&](int k2, int f, double re, double im) {
                const int row = r0 + f;
                if (row >= N1) return;
                const long long iz = (long long)N1 * k2 + row;
                if (DST == kDstComplex) {
                    dst[iz] = C{re, im};
                } else {
                    emit(P.work, it, tr.c, tr.b, 2 * iz, re);
                    emit(P.work, it, tr.c, tr.b, 2 * iz + 1, -im);
                }
            });
    }
    tc_teardown(tmem);
}

// ------------------------------------------------------------------------------------------------------
// host side: FFT plans and tables (built in dd on the host, as the reference builds them)
// ------------------------------------------------------------------------------------------------------
struct HostCx {
    hd::dd re, im;
};

// Stockham plan of n points: radices 4,..,4,2,..,2,3,..,5,..,7,.. (fft.hpp:93-97), its stage twiddles to start
// at table entry tw0, m * (r - 1) entries per stage (one entry when there are none, keeping the table pointer
// valid for n = 1). Builds nothing but the plan.
int plan_sub(int n, int tw0, SubPlan& sp) {
    int rs[64], ns = 0, t = n;
    while (t % 4 == 0) { rs[ns++] = 4; t /= 4; }
    while (t % 2 == 0) { rs[ns++] = 2; t /= 2; }
    for (int p : {3, 5, 7})
        while (t % p == 0) { rs[ns++] = p; t /= p; }
    if (t != 1) return fail(KBSRC_GPU_E_UNSUPPORTED, "FFT length not 7-smooth");
    if (ns > kMaxStages) return fail(KBSRC_GPU_E_UNSUPPORTED, "FFT length has too many stages");
    std::memset(&sp, 0, sizeof sp);
    sp.n = n;
    sp.nst = ns;
    sp.tw0 = tw0;
    int rem = n, s = 1, at = tw0;
    for (int g = 0; g < ns; g++) {
        const int r = rs[g], m = rem / r;
        sp.st[g] = Stage{r, m, s, at};
        at += m * (r - 1);
        rem /= r;
        s *= r;
    }
    sp.twn = std::max(1, at - tw0);
    return KBSRC_GPU_OK;
}

// The plan of n points with its stage twiddles w_n^{s p u} appended to `tw` (fft.hpp:98-107).
int build_sub(int n, std::vector<HostCx>& tw, SubPlan& sp) {
    const int rc = plan_sub(n, (int)tw.size(), sp);
    if (rc) return rc;
    hd::RootTable rt(n);
    for (int g = 0; g < sp.nst; g++) {
        const Stage& st = sp.st[g];
        for (int p = 0; p < st.m; p++)
            for (int u = 1; u < st.r; u++) {
                HostCx w;
                rt.get(-(long long)st.s * p * u, w.re, w.im);
                tw.push_back(w);
            }
    }
    if ((int)tw.size() == sp.tw0) tw.push_back(HostCx{});
    return KBSRC_GPU_OK;
}

struct HostCfft {
    int n = 0, four = 0, N1 = 0, N2 = 0;
    SubPlan s1{}, s2{}, sd{};
    std::vector<HostCx> tw_stage, tw4;
};

// Complex FFT of n points (fft.hpp:226-265): direct up to 2048 points, else four-step with N1 the largest
// divisor <= sqrt(n) (falling back to direct when N1 < 8). The plan only: sub-plans with their stage twiddles laid
// out in one table (s1's, then s2's), no tables built.
int plan_cfft(int n, HostCfft& c) {
    c.n = n;
    if (!hd::smooth7(n)) return fail(KBSRC_GPU_E_UNSUPPORTED, "FFT length not 7-smooth (Bluestein)");
    c.four = n > 2048;
    if (c.four) {
        int best = 1;
        for (int d = 1; (long long)d * d <= n; d++)
            if (n % d == 0) best = d;
        c.N1 = best;
        c.N2 = n / best;
        if (c.N1 < 8) c.four = 0;
    }
    // the passes divide indices through fast_div, exact while index * divisor < 2^32: sub-FFTs up to 2^15 points
    if ((c.four ? std::max(c.N1, c.N2) : n) > 32768)
        return fail(KBSRC_GPU_E_UNSUPPORTED, "FFT length without a four-step split into sub-FFTs of at most 32768");
    if (!c.four) return plan_sub(n, 0, c.sd);
    const int rc = plan_sub(c.N1, 0, c.s1);
    return rc ? rc : plan_sub(c.N2, c.s1.twn, c.s2);
}

// The plan with its host tables: stage twiddles and the four-step twiddles w_n^{-k1 n2}.
int build_cfft(int n, HostCfft& c) {
    int rc = plan_cfft(n, c);
    if (rc) return rc;
    if (!c.four) return build_sub(n, c.tw_stage, c.sd);
    if ((rc = build_sub(c.N1, c.tw_stage, c.s1)) != KBSRC_GPU_OK) return rc;
    if ((rc = build_sub(c.N2, c.tw_stage, c.s2)) != KBSRC_GPU_OK) return rc;
    c.tw4.resize((size_t)n);
    hd::RootTable rt(n);
    for (int k1 = 0; k1 < c.N1; k1++)
        for (int n2 = 0; n2 < c.N2; n2++) {
            HostCx& w = c.tw4[(size_t)k1 * c.N2 + n2];
            rt.get(-(long long)k1 * n2, w.re, w.im);
        }
    return KBSRC_GPU_OK;
}

// w[k] = e^{-2 pi i k/N}, k <= N/2 (fft.hpp:356-357)
std::vector<HostCx> split_roots(int N) {
    std::vector<HostCx> w((size_t)N / 2 + 1);
    hd::RootTable rt(N);
    for (int k = 0; k <= N / 2; k++) rt.get(-k, w[k].re, w[k].im);
    return w;
}

// Device copy of a table: dd pairs for double-double, the high parts for f64 (fft.hpp:16)
// An owned device allocation. Move-only: a copy would free the same pointer twice (and leave the survivor
// pointing at freed memory).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) {
        o.p = nullptr;
        o.bytes = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    int alloc(size_t n) {
        release();
        if (n == 0) n = 16;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(e == cudaErrorMemoryAllocation ? KBSRC_GPU_E_NOMEM : KBSRC_GPU_E_CUDA,
                        std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        bytes = n;
        return KBSRC_GPU_OK;
    }
};

// Table formats on the device: the high parts (f64), (hi, lo) pairs (double-double), or the x87 extended value
// (long double)hi + (long double)lo (fft.hpp:16-17), 16 bytes each.
enum TabFmt { kTabF64 = 0, kTabDD = 1, kTabX80 = 2 };

size_t tab_esize(int tab) { return tab == kTabF64 ? 16 : 32; }
// Most threads per CTA the column (or row) pass kernels of a table format are compiled for
int tab_max_threads(int tab, bool column) {
    if (tab == kTabF64) return KB_MAXT_F64;
    if (tab == kTabX80) return KB_MAXT_X80;
    return column ? KB_MAXT_DD_COL : KB_MAXT_DD;
}

// Bytes of one input sample in a KBSRC_GPU_IN_* format
size_t in_bytes(int fmt) {
    static const size_t b[] = {8, 4, 4, 3, 2, 1};
    return fmt >= 0 && fmt <= 5 ? b[fmt] : 8;
}

// from_dd<long double> with the host's own x87 arithmetic, stored as the device's x80 (significand, sign and
// exponent)
x80 host_x80(const hd::dd& v) {
    const long double x = (long double)v.hi + (long double)v.lo;
    unsigned char b[sizeof(long double)] = {};
    std::memcpy(b, &x, 10);
    x80 r{};
    std::memcpy(&r.m, b, 8);
    r.se = b[8] | b[9] << 8;
    return r;
}

int upload_cx(const std::vector<HostCx>& v, int tab, DevBuf& out) {
    if (tab == kTabX80) {
        std::vector<x80> flat(v.size() * 2);
        for (size_t i = 0; i < v.size(); i++) {
            flat[2 * i] = host_x80(v[i].re);
            flat[2 * i + 1] = host_x80(v[i].im);
        }
        int rc = out.alloc(flat.size() * sizeof(x80));
        if (rc) return rc;
        KB_CUDA(cudaMemcpy(out.p, flat.data(), flat.size() * sizeof(x80), cudaMemcpyHostToDevice));
        return KBSRC_GPU_OK;
    }
    std::vector<double> flat;
    if (tab == kTabDD) {
        flat.resize(v.size() * 4);
        for (size_t i = 0; i < v.size(); i++) {
            flat[4 * i] = v[i].re.hi; flat[4 * i + 1] = v[i].re.lo;
            flat[4 * i + 2] = v[i].im.hi; flat[4 * i + 3] = v[i].im.lo;
        }
    } else {
        flat.resize(v.size() * 2);
        for (size_t i = 0; i < v.size(); i++) { flat[2 * i] = v[i].re.hi; flat[2 * i + 1] = v[i].im.hi; }
    }
    int rc = out.alloc(flat.size() * sizeof(double));
    if (rc) return rc;
    KB_CUDA(cudaMemcpy(out.p, flat.data(), flat.size() * sizeof(double), cudaMemcpyHostToDevice));
    return KBSRC_GPU_OK;
}

template <class W>
OddRoots<W> odd_roots() {
    OddRoots<W> o{};
    const int rr[3] = {3, 5, 7};
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < rr[i]; k++) {
            hd::dd c, s;
            hd::unit_root(k, rr[i], c, s);
            if constexpr (sizeof(W) == sizeof(double)) {
                o.c[i][k] = c.hi;
                o.s[i][k] = s.hi;
            } else if constexpr (std::is_same_v<W, x80>) {
                o.c[i][k] = host_x80(c);
                o.s[i][k] = host_x80(s);
            } else {
                o.c[i][k] = W{c.hi, c.lo};
                o.s[i][k] = W{s.hi, s.lo};
            }
        }
    return o;
}

// Threads per CTA of the float64 passes by default: with at most 5 sequences per CTA, more CTAs per SM overlap
// one CTA's loads with another's arithmetic (C2 fast: 1.65 against 1.73 ms per step with 16 x 256).
constexpr int kThreadsF64 = 128;

// Launch shape of a shared-memory pass over sequences of length n: F sequences per CTA, T threads.
struct Shape {
    int F, T;
    size_t smem;
    bool twg = false;  // double-double / extended: stage twiddles read from global memory, not staged in shared
};

int max_bfly(const SubPlan& sp) {
    int b = 1;
    for (int g = 0; g < sp.nst; g++) b = std::max(b, sp.st[g].m * sp.st[g].s);
    return b;
}

int env_int(const char* name, int dflt);

// F sequences per CTA (a divisor of `count` when one fits) and T threads, within a shared-memory budget; the
// block also holds the sub-FFT's twiddles in double-double, except where it holds a single sequence: those read
// the global table instead (a copy made for one sequence costs about a fifth of the CTA's shared memory for little
// reuse; the autotuner's choice on C5's 960- and 1008-point forward passes, 4.43 -> 3.96 and 4.04 -> 3.50 ms per
// wave). KBSRC_GPU_TW_GLOBAL=1 reads the table in every wide pass, =0 stages in every one.
Shape pick_shape(const SubPlan& sp, int count, size_t esize, int fmax, int maxT) {
    const size_t budget = (size_t)env_int("KBSRC_GPU_SMEM_KB", 100) * 1024;
    const int force = env_int("KBSRC_GPU_TW_GLOBAL", -1);
    bool twg = esize == 32 && force == 1;
    size_t tw = esize == 32 && !twg ? (size_t)sp.twn * esize : 0;
    int F = 1;
    for (int f = fmax; f >= 1; f--) {
        if (2 * (size_t)sp.n * f * esize + tw > budget) continue;
        if (F == 1) F = f;
        if (count % f == 0) { F = f; break; }
    }
    if (esize == 32 && F == 1 && force == -1) {
        twg = true;
        tw = 0;
    }
    int T = ((max_bfly(sp) * F + 31) / 32) * 32;
    T = std::max(64, std::min(std::min(env_int("KBSRC_GPU_THREADS", maxT), maxT), T));
    return Shape{F, T, 2 * (size_t)sp.n * F * esize + tw, twg};
}

Shape direct_shape(const SubPlan& sp, size_t esize) {
    int T = ((max_bfly(sp) + 31) / 32) * 32;
    T = std::max(64, std::min(env_int("KBSRC_GPU_THREADS", esize == 32 ? KB_MAXT_DD : kThreadsF64), T));
    return Shape{1, T, 2 * (size_t)sp.n * esize + (esize == 32 ? (size_t)sp.twn * esize : 0)};
}

long long next_smooth7(long long n) {
    while (!hd::smooth7(n)) n++;
    return n;
}

// A complex FFT resident on the device: a smooth plan (direct or four-step) with its twiddle tables and launch
// shapes, or Bluestein's chirp-z for a length that is not 7-smooth (fft.hpp:228-240): n points through the
// m-point smooth transform `inner`, with the chirp bc[t] = e^{+i pi t^2/n} and Vf = FFT(v)/m, v the chirp
// placed at t and m - t (computed once on the GPU with the scalar double-double FFT, as the reference does with
// CFFT<dd,dd,dd>).
struct DevCfft {
    HostCfft host;  // shapes and sub-plans (tables released after upload)
    DevBuf tw_stage, tw4;
    Shape col{}, row{}, dir{};
    int n = 0, m = 0;
    std::unique_ptr<DevCfft> inner;
    DevBuf bc, vf;
    long long slot() const { return m ? m : n; }  // complex values one task slot must hold
};

int bluestein_kernel(DevCfft& d, int tab, cudaStream_t st);  // Vf, defined with the launchers

int make_dev_cfft(int n, int tab, int fmax, DevCfft& d, cudaStream_t st) {
    d.n = n;
    int rc;
    const size_t esize = tab_esize(tab);
    if (!hd::smooth7(n)) {
        d.m = (int)next_smooth7(2LL * n - 1);
        d.inner = std::make_unique<DevCfft>();
        if ((rc = make_dev_cfft(d.m, tab, fmax, *d.inner, st)) != KBSRC_GPU_OK) return rc;
        std::vector<HostCx> bc((size_t)n);
        for (long long t = 0; t < n; t++) {
            const long long e = (long long)((__int128)t * t % (2LL * n));
            hd::unit_root(e, 2LL * n, bc[t].re, bc[t].im);
        }
        if ((rc = upload_cx(bc, tab, d.bc)) != KBSRC_GPU_OK) return rc;
        return bluestein_kernel(d, tab, st);
    }
    if ((rc = build_cfft(n, d.host)) != KBSRC_GPU_OK) return rc;
    if ((rc = upload_cx(d.host.tw_stage, tab, d.tw_stage)) != KBSRC_GPU_OK) return rc;
    if (d.host.four && (rc = upload_cx(d.host.tw4, tab, d.tw4)) != KBSRC_GPU_OK) return rc;
    std::vector<HostCx>().swap(d.host.tw_stage);
    std::vector<HostCx>().swap(d.host.tw4);
    if (d.host.four) {
        // default thread caps: float64 kThreadsF64 (the autotuner tries up to the compiled maximum)
        d.col = pick_shape(d.host.s1, d.host.N2, esize, fmax, tab == kTabF64 ? kThreadsF64 : tab_max_threads(tab, true));
        d.row = pick_shape(d.host.s2, d.host.N1, esize, fmax, tab == kTabF64 ? kThreadsF64 : tab_max_threads(tab, false));
    } else {
        d.dir = direct_shape(d.host.sd, esize);
    }
    return KBSRC_GPU_OK;
}

// ------------------------------------------------------------------------------------------------------
// split-precision plans: n = N1 * N2 (four-step, or N2 = 1 for one direct sub-FFT), each sub-FFT N = Ra * Rb
// (or, where no such pair exists, Ra * Rb * Rc) with radices <= 32, so that every stage is one tcgen05
// contraction with K, N <= 64.
// ------------------------------------------------------------------------------------------------------
// Ra * Rb = N with both in [2, 32], Ra the largest such divisor <= sqrt(N); a length of at most 32 without such a
// split (a prime) is one stage, Ra = N and Rb = 1. False when there is neither.
bool tc_factor(int N, int& Ra, int& Rb) {
    int best = 0;
    for (int a = 2; a <= 32 && a * a <= N; a++)
        if (N % a == 0 && N / a <= 32) best = a;
    if (best) {
        Ra = best;
        Rb = N / best;
        return true;
    }
    if (N < 2 || N > 32) return false;
    Ra = N;
    Rb = 1;
    return true;
}
// Ra * Rb * Rc = N, each <= 32 and >= N / 128 (so that every stage has at most 128 rows), the smallest radix as
// large as possible; false when there is none.
bool tc_factor3(int N, int& Ra, int& Rb, int& Rc) {
    const int lo = std::max(2, (N + kTcRows - 1) / kTcRows);
    int best = 0;
    for (int a = lo; a <= 32; a++) {
        if (N % a) continue;
        for (int b = a; b <= 32; b++) {
            if ((N / a) % b) continue;
            const int c = N / a / b;
            if (c < b || c > 32 || a <= best) continue;
            best = a;
            Ra = a;
            Rb = b;
            Rc = c;
        }
    }
    return best > 0;
}
int tc_kh(int R) { return R <= 16 ? 16 : 32; }
// Output columns per half of the matrix (real, imaginary): 16, 24 or 32; with two CTA halves a radix above 16 runs
// in two rounds of nh columns, and an MMA's N (blocks of nh) must stay a multiple of 16, so 24 becomes 32.
int tc_nh(int R, int halves) { return R <= 16 ? 16 : R <= 24 && halves == 1 ? 24 : 32; }
TcRadix tc_radix(int R, int halves) {
    if (R <= 1) return TcRadix{1, 0, 0, 1, nullptr};
    const int nh = tc_nh(R, halves);
    return TcRadix{R, tc_kh(R), nh, tc_rounds_for(nh, halves), nullptr};
}

// f16 bits of a small integer v (|v| <= 128): exact
uint16_t f16_bits(int v) {
    if (v == 0) return 0;
    const unsigned a = (unsigned)std::abs(v);
    int e = 0;
    while ((a >> (e + 1)) != 0) e++;                                      // 2^e <= a < 2^(e+1)
    const unsigned mant = (a << (10 - e)) & 0x3FFu;                       // a < 2^8: exact in 10 bits
    return (uint16_t)((v < 0 ? 0x8000u : 0u) | (unsigned)(e + 15) << 10 | mant);
}

// The real form of DFT_R (outputs n: real parts, then imaginary parts from nh; inputs k: real parts, then
// imaginary parts from kh), y_re[k1] = sum_j xr_j cos + xi_j sin, y_im[k1] = sum_j xi_j cos - xr_j sin with the
// angle 2 pi j k1 / R. Each entry w becomes W = rint(w 2^54) in seven balanced base-256 digits; slice t holds digit
// 6 - t of every entry as int8 (eb = 1) or f16 (eb = 2), slice kTcDigits stays zero. Layout
// [round][slice][2nh / rounds rows][2kh] (rad.rounds, rad.nh as planned).
void tc_matrix(const TcRadix& rad, int eb, std::vector<unsigned char>& out) {
    const int R = rad.R, kh = rad.kh, nh = rad.nh, kpad = 2 * kh * eb, npad = 2 * nh, nr = npad / rad.rounds;
    const size_t base = out.size();
    out.resize(base + (size_t)kTcMats * npad * kpad, 0);
    auto put = [&](int n, int k, double w) {
        const long long W = std::llrint(std::ldexp(w, 54));  // exact scaling, one rounding; |W| <= 2^54
        const unsigned long long b = (unsigned long long)(W + 0x80808080808080LL);
        const int rd = n / nr, nn = n - rd * nr;
        for (int i = 0; i < kTcDigits; i++) {
            const int digit = (int)((b >> (8 * i)) & 0xFF) - 128;
            unsigned char* at = &out[base + ((size_t)rd * kTcMats + (kTcDigits - 1 - i)) * nr * kpad +
                                     umma_off(nn, k * eb, kpad)];
            if (eb == 1) {
                *at = (unsigned char)(signed char)digit;
            } else {
                const uint16_t h = f16_bits(digit);
                at[0] = (unsigned char)(h & 0xFF);
                at[1] = (unsigned char)(h >> 8);
            }
        }
    };
    hd::RootTable rt(R);
    for (int k1 = 0; k1 < R; k1++)
        for (int j = 0; j < R; j++) {
            hd::dd c, sn;
            rt.get((long long)j * k1, c, sn);
            put(k1, j, c.hi);
            put(k1, kh + j, sn.hi);
            put(nh + k1, j, -sn.hi);
            put(nh + k1, kh + j, c.hi);
        }
}

// A transform of n points in the split form, resident on the device. eb: digit element bytes (1 int8, 2 f16).
struct TcFftDev {
    int n = 0, N1 = 0, N2 = 0, eb = 1;
    int ctas = 148;  // persistent CTAs per pass: one per SM
    TcSub col{}, row{};
    size_t smem_col = 0, smem_row = 0;
    DevBuf tw4, tw_in, mats;
    size_t bytes() const { return tw4.bytes + tw_in.bytes + mats.bytes; }
};

// Sub-FFT of N points over `count` sequences with digit elements of eb bytes: radices, items in flight per CTA
// (one; KBSRC_GPU_TC_HALVES=2 selects two halves of 256 threads, which measured slower on C2: 3.80 against 3.33 ms
// per step, the radices above 16 needing two rounds), sequences per item within the shared-memory limit
int tc_sub_plan(int N, int count, int eb, TcSub& sub, size_t& smem) {
    int Ra = 1, Rb = 1, Rc = 1;
    if (!tc_factor(N, Ra, Rb) && !tc_factor3(N, Ra, Rb, Rc))
        return fail(KBSRC_GPU_E_UNSUPPORTED, "split-precision form: no radix-32 factorisation");
    int rmin = std::min(Ra, Rb > 1 ? Rb : Ra);
    if (Rc > 1) rmin = std::min(rmin, Rc);
    const int rows1 = N / rmin;  // rows of the largest stage for one sequence
    const size_t limit = 227 * 1024;
    auto plan = [&](int halves, TcSub& t, size_t& bytes) {  // the most sequences per item that fit; 0: none
        t = TcSub{};
        t.N = N;
        t.ebytes = eb;
        t.halves = halves;
        t.a = tc_radix(Ra, halves);
        t.b = tc_radix(Rb, halves);
        t.c = tc_radix(Rc, halves);
        for (int F = std::max(1, std::min(kTcRows / rows1, count)); F >= 1; F--) {
            t.F = F;
            bytes = tc_smem_bytes(t);
            if (bytes <= limit) return F;
        }
        return 0;
    };
    TcSub one, two;
    size_t b1 = 0, b2 = 0;
    const int f1 = plan(1, one, b1), f2 = plan(2, two, b2);
    const int force = env_int("KBSRC_GPU_TC_HALVES", 0);
    const bool use2 = f2 > 0 && (force == 2 || (f1 == 0 && force != 1));
    if (!use2 && f1 == 0) return fail(KBSRC_GPU_E_UNSUPPORTED, "split-precision form: sub-FFT too large");
    sub = use2 ? two : one;
    smem = use2 ? b2 : b1;
    return KBSRC_GPU_OK;
}

int make_tc_fft(int n, int eb, TcFftDev& t) {
    int rc, a, b, dev = 0;
    t.eb = eb;
    KB_CUDA(cudaGetDevice(&dev));
    KB_CUDA(cudaDeviceGetAttribute(&t.ctas, cudaDevAttrMultiProcessorCount, dev));
    t.n = n;
    t.N1 = t.N2 = 0;
    int c;
    // two radices per sub-FFT where possible, three where the length needs them
    for (int three = 0; three < 2 && !t.N1; three++) {
        auto ok = [&](int N) { return tc_factor(N, a, b) || (three && tc_factor3(N, a, b, c)); };
        if (n <= 1024 && ok(n)) {
            t.N1 = n;
            t.N2 = 1;
            break;
        }
        for (int N1 = (int)std::sqrt((double)n) + 1; N1 >= 2; N1--) {
            if ((long long)N1 * N1 > n || n % N1) continue;
            const int N2 = n / N1;
            if (N2 <= 1024 && ok(N1) && ok(N2)) {
                t.N1 = N1;
                t.N2 = N2;
                break;
            }
        }
    }
    if (!t.N1)
        return fail(KBSRC_GPU_E_UNSUPPORTED, "split-precision form: transform length " + std::to_string(n) +
                                                 " has no factorisation into radices <= 32");
    if ((rc = tc_sub_plan(t.N1, t.N2, eb, t.col, t.smem_col)) != KBSRC_GPU_OK) return rc;
    if (t.N2 > 1 && (rc = tc_sub_plan(t.N2, t.N1, eb, t.row, t.smem_row)) != KBSRC_GPU_OK) return rc;
    // sliced matrices of the (up to six) radices, the inner twiddles of each sub-FFT, and the four-step twiddles
    std::vector<unsigned char> mats;
    size_t off[6];
    TcRadix* rads[6] = {&t.col.a, &t.col.b, &t.col.c, &t.row.a, &t.row.b, &t.row.c};
    const int nr = t.N2 > 1 ? 6 : 3;
    for (int i = 0; i < nr; i++) {
        off[i] = mats.size();
        if (rads[i]->R > 1) tc_matrix(*rads[i], eb, mats);
    }
    if ((rc = t.mats.alloc(mats.size())) != KBSRC_GPU_OK) return rc;
    KB_CUDA(cudaMemcpy(t.mats.p, mats.data(), mats.size(), cudaMemcpyHostToDevice));
    for (int i = 0; i < nr; i++)
        if (rads[i]->R > 1)
            rads[i]->slices = reinterpret_cast<const uint4*>(static_cast<unsigned char*>(t.mats.p) + off[i]);
    std::vector<double> tw;
    auto roots = [&](int N, int A, int B) {  // [k1 * B + m] = e^{-2 pi i m k1 / N}, k1 < A, m < B
        hd::RootTable rt(N);
        for (int k1 = 0; k1 < A; k1++)
            for (int m = 0; m < B; m++) {
                hd::dd c, sn;
                rt.get(-(long long)m * k1, c, sn);
                tw.push_back(c.hi);
                tw.push_back(sn.hi);
            }
    };
    auto inner = [&](const TcSub& sub) {
        if (sub.c.R > 1) {
            roots(sub.N, sub.a.R, sub.b.R * sub.c.R);
            roots(sub.b.R * sub.c.R, sub.b.R, sub.c.R);
        } else {
            roots(sub.N, sub.a.R, sub.b.R);
        }
    };
    inner(t.col);
    const size_t row_off = tw.size();
    if (t.N2 > 1) inner(t.row);
    if ((rc = t.tw_in.alloc(tw.size() * sizeof(double))) != KBSRC_GPU_OK) return rc;
    KB_CUDA(cudaMemcpy(t.tw_in.p, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice));
    t.col.tw = static_cast<const double2*>(t.tw_in.p);
    if (t.N2 > 1) {
        t.row.tw = reinterpret_cast<const double2*>(static_cast<double*>(t.tw_in.p) + row_off);
        std::vector<double> w4(2 * (size_t)n);
        hd::RootTable rt(n);
        for (int k1 = 0; k1 < t.N1; k1++)
            for (int n2 = 0; n2 < t.N2; n2++) {
                hd::dd c, sn;
                rt.get(-(long long)k1 * n2, c, sn);
                w4[2 * ((size_t)k1 * t.N2 + n2)] = c.hi;
                w4[2 * ((size_t)k1 * t.N2 + n2) + 1] = sn.hi;
            }
        if ((rc = t.tw4.alloc(w4.size() * sizeof(double))) != KBSRC_GPU_OK) return rc;
        KB_CUDA(cudaMemcpy(t.tw4.p, w4.data(), w4.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    return KBSRC_GPU_OK;
}

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}

}  // namespace

// ------------------------------------------------------------------------------------------------------
// the engine
// ------------------------------------------------------------------------------------------------------
// The transform plan of one conversion shape: its FFTs, split/merge roots and kernel spectrum. Conversions that
// share it (a batch group) run in the same launches.
struct PlanCore {
    kbsrc_gpu_desc d{};  // the shape (H is not kept)
    bool exact = false;
    bool split = false;        // split-precision form: tfw / tiv instead of fw / iv
    TcFftDev tfw, tiv;
    DevBuf tc_err;             // int: a tensor-core stage timed out
    int tab = 0;  // TabFmt of the tables and of the values in the work buffers
    int Nb = 0, Mb = 0, hf = 0, hi = 0, hop = 0;
    DevCfft fw, iv;
    DevBuf w_fw, w_iv, H;
    // complex values one task slot must hold: h+1, h'+1 and the Bluestein lengths
    long long slot() const {
        const long long n = std::max({(long long)hf + 1, (long long)hi + 1, fw.slot(), iv.slot()});
        return (n + 7) / 8 * 8;
    }
    size_t esize() const { return tab_esize(tab); }
};

// A batch group: conversions with one plan, their tasks listed block-major per conversion.
struct BatchGroup : PlanCore {
    std::vector<int> members;
    long long tasks = 0, stride = 0, wave = 0;
    DevBuf refs;  // TaskRef[tasks]
    bool queued = false;  // runs through the batch queue (else its own launches)
};

// A wave of the batch queue: tasks of any groups, largest transform first, and the units of each pass.
struct QueueWave {
    long long ntasks = 0;
    DevBuf tasks;                 // QueueTask[ntasks]
    DevBuf units[6];              // QueueUnit lists: forward column, forward row, split, merge, inverse column, row
    int nunits[6] = {};
};

struct kbsrc_gpu_batch {
    std::vector<kbsrc_gpu_desc> descs;  // per conversion (H not kept)
    std::vector<std::unique_ptr<BatchGroup>> groups;
    bool queued = false;                // some groups run through the queue kernels
    bool q_exact = false;               // their arithmetic: double-double (else float64)
    DevBuf q_groups;                    // QueueGroup[queued groups]
    std::vector<QueueWave> q_waves;
    DevBuf q_counters;                  // int[waves * 6], zeroed at the start of every run
    int q_threads[6] = {}, q_ctas[6] = {};
    size_t q_smem[6] = {};
    std::vector<int> group_of;          // conversion -> group, -1 when it has no tasks
    int device = 0;
    cudaStream_t stream = nullptr;
    DevBuf items;                       // Item[count], rewritten from items_host by every run
    Item* items_host = nullptr;         // pinned
    DevBuf bufA, bufB;
    cudaGraphExec_t graph = nullptr;    // the whole run, recorded on first use
    cudaEvent_t done = nullptr;         // end of the last run (guards items_host)
    long long launches = 0;
    std::vector<DevBuf> d_in, d_head, d_tail, d_out;  // run_host buffers, allocated on first use
    ~kbsrc_gpu_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (done) cudaEventDestroy(done);
        if (items_host) cudaFreeHost(items_host);
        if (stream) cudaStreamDestroy(stream);
    }
};

// Copies between pageable host memory and the device through two pinned bounce buffers: the host-side copy of
// one chunk (split over threads) overlaps the DMA of the other. Pinned host memory is copied directly.
struct Stager {
    static constexpr size_t kChunk = (size_t)32 << 20;
    void* pin[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~Stager() {
        for (int i = 0; i < 2; i++) {
            if (pin[i]) cudaFreeHost(pin[i]);
            if (ev[i]) cudaEventDestroy(ev[i]);
        }
    }
};

struct kbsrc_gpu_engine : PlanCore {
    int device = 0;
    long long tasks = 0, wave = 0, stride = 0, launches = 0;
    long long t_begin = 0, t_end = 0;  // the share's tasks: blocks [blk0, blk1) x channels, task = b*ch + c
    cudaStream_t stream = nullptr;
    cudaStream_t copy_in = nullptr, copy_out = nullptr;  // run_host's copy pipeline
    cudaEvent_t ev_in[2] = {}, ev_done[2] = {};
    DevBuf bufA, bufB;
    DevBuf d_in, d_head, d_tail, d_out;
    Stager stager;                    // pageable host buffers of run_host / run_host_packed
    cudaStream_t side = nullptr;      // run_host_packed's dither generator
    std::vector<cudaEvent_t> events;  // per-pass timing trail, created on first use
    ~kbsrc_gpu_engine() {
        if (side) cudaStreamDestroy(side);
        for (cudaEvent_t x : events) cudaEventDestroy(x);
        for (cudaEvent_t x : {ev_in[0], ev_in[1], ev_done[0], ev_done[1]})
            if (x) cudaEventDestroy(x);
        if (copy_in) cudaStreamDestroy(copy_in);
        if (copy_out) cudaStreamDestroy(copy_out);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// Radix 3/5/7 constants, computed once per process
template <class W>
const OddRoots<W>& odd_table() {
    static const OddRoots<W> t = odd_roots<W>();
    return t;
}

// Lets every pass kernel use up to the device's shared memory per block. The attribute belongs to the current
// context, so whether it is set is read back from the context (the last kernel set below) rather than remembered.
int allow_large_smem() {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    int dev = 0;
    KB_CUDA(cudaGetDevice(&dev));
    int mx = 0;
    KB_CUDA(cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    KB_CUDA(cudaFuncGetAttributes(&fa, (const void*)k_tc_row<TcF16, kDstOutput, 1>));
    if (fa.maxDynamicSharedSizeBytes >= mx) return KBSRC_GPU_OK;
    // the dynamic limit is what the static shared memory of the kernel leaves of the opt-in maximum
#define KB_SMEM(k)                                                                                          \
    do {                                                                                                    \
        cudaFuncAttributes ka{};                                                                            \
        KB_CUDA(cudaFuncGetAttributes(&ka, (const void*)(k)));                                              \
        KB_CUDA(cudaFuncSetAttribute((const void*)(k), cudaFuncAttributeMaxDynamicSharedMemorySize,          \
                                     mx - (int)ka.sharedSizeBytes));                                        \
    } while (0)
    KB_SMEM((k_column<ArF64, kSrcSignal, false>));
    KB_SMEM((k_column<ArF64, kSrcComplex, false>));
    KB_SMEM((k_column<ArDDShort, kSrcSignal, false>));
    KB_SMEM((k_column<ArDDShort, kSrcSignal, true>));
    KB_SMEM((k_column<ArDDShort, kSrcComplex, false>));
    KB_SMEM((k_column<ArDDShort, kSrcComplex, true>));
    KB_SMEM((k_column<ArDDAccurate, kSrcDDReal, false>));
    KB_SMEM((k_column<ArDDAccurate, kSrcDDReal, true>));
    KB_SMEM((k_column<ArDDAccurate, kSrcComplex, false>));
    KB_SMEM((k_column<ArDDAccurate, kSrcComplex, true>));
    KB_SMEM((k_row<ArF64, kDstComplex, false>));
    KB_SMEM((k_row<ArF64, kDstOutput, false>));
    KB_SMEM((k_row<ArDDShort, kDstComplex, false>));
    KB_SMEM((k_row<ArDDShort, kDstComplex, true>));
    KB_SMEM((k_row<ArDDShort, kDstOutput, false>));
    KB_SMEM((k_row<ArDDShort, kDstOutput, true>));
    KB_SMEM((k_row<ArDDAccurate, kDstComplex, false>));
    KB_SMEM((k_row<ArDDAccurate, kDstComplex, true>));
    KB_SMEM((k_direct<ArF64, kSrcSignal, kDstComplex>));
    KB_SMEM((k_direct<ArF64, kSrcComplex, kDstComplex>));
    KB_SMEM((k_direct<ArF64, kSrcComplex, kDstOutput>));
    KB_SMEM((k_direct<ArDDAccurate, kSrcSignal, kDstComplex>));
    KB_SMEM((k_direct<ArDDAccurate, kSrcComplex, kDstComplex>));
    KB_SMEM((k_direct<ArDDAccurate, kSrcComplex, kDstOutput>));
    KB_SMEM((k_direct<ArDDAccurate, kSrcDDReal, kDstComplex>));
    KB_SMEM((k_column<ArX80, kSrcSignal, false>));
    KB_SMEM((k_column<ArX80, kSrcSignal, true>));
    KB_SMEM((k_column<ArX80, kSrcComplex, false>));
    KB_SMEM((k_column<ArX80, kSrcComplex, true>));
    KB_SMEM((k_row<ArX80, kDstComplex, false>));
    KB_SMEM((k_row<ArX80, kDstComplex, true>));
    KB_SMEM((k_row<ArX80, kDstOutput, false>));
    KB_SMEM((k_row<ArX80, kDstOutput, true>));
    KB_SMEM((k_direct<ArX80, kSrcSignal, kDstComplex>));
    KB_SMEM((k_direct<ArX80, kSrcComplex, kDstComplex>));
    KB_SMEM((k_direct<ArX80, kSrcComplex, kDstOutput>));
    KB_SMEM((k_column_q<ArDDShort, kSrcSignal, true>));
    KB_SMEM((k_column_q<ArDDShort, kSrcComplex, false>));
    KB_SMEM((k_row_q<ArDDShort, kDstComplex, true>));
    KB_SMEM((k_row_q<ArDDShort, kDstOutput, false>));
    KB_SMEM((k_column_q<ArF64, kSrcSignal, true>));
    KB_SMEM((k_column_q<ArF64, kSrcComplex, false>));
    KB_SMEM((k_row_q<ArF64, kDstComplex, true>));
    KB_SMEM((k_row_q<ArF64, kDstOutput, false>));
#define KB_SMEM_TC(S, H)                                 \
    KB_SMEM((k_tc_column<S, kSrcSignal, kDstComplex, H>));  \
    KB_SMEM((k_tc_column<S, kSrcComplex, kDstComplex, H>)); \
    KB_SMEM((k_tc_column<S, kSrcComplex, kDstOutput, H>));  \
    KB_SMEM((k_tc_row<S, kDstComplex, H>));                 \
    KB_SMEM((k_tc_row<S, kDstOutput, H>))
    KB_SMEM_TC(TcI8, 1);
    KB_SMEM_TC(TcI8, 2);
    KB_SMEM_TC(TcF16, 2);
    KB_SMEM_TC(TcF16, 1);  // last: k_tc_row<TcF16, kDstOutput, 1> is the marker read above
#undef KB_SMEM_TC
#undef KB_SMEM
    return KBSRC_GPU_OK;
}

// A usable CUDA device, or KBSRC_GPU_E_NODEVICE with the runtime's reason.
int require_device() {
    int ndev = 0;
    const cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return fail(KBSRC_GPU_E_NODEVICE, std::string("no usable CUDA device: ") +
                                              (e != cudaSuccess ? cudaGetErrorString(e) : "none found"));
    }
    return KBSRC_GPU_OK;
}

unsigned grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    return (unsigned)std::max(1LL, std::min(b, 65535LL));
}

// Pass kinds for per-pass timing (kbsrc_gpu_engine_run_device_timed)
enum PassKind { kFwdA = 0, kFwdB, kSplit, kMerge, kInvA, kInvB, kPassKinds };

// Optional per-launch event trail: an event before the first launch, then one after each launch.
struct Trail {
    std::vector<cudaEvent_t>* ev = nullptr;
    std::vector<int>* kind = nullptr;
    size_t n = 0;
    long long launches = 0;
    int mark(cudaStream_t st, int k) {
        if (k >= 0) launches++;
        if (!ev) return KBSRC_GPU_OK;
        if (n >= ev->size()) {
            cudaEvent_t x;
            KB_CUDA(cudaEventCreate(&x));
            ev->push_back(x);
        }
        KB_CUDA(cudaEventRecord((*ev)[n], st));
        if (kind) kind->push_back(k);
        n++;
        return KBSRC_GPU_OK;
    }
};

// What every pass of one launch group shares: task slots, the signal view, the output.
struct Slots {
    long long stride, task0;
    unsigned nt;
    Work work;
    const double* ddreal;
};

template <class Ar>
PassParams<Ar> pass_params(const Slots& sl, const DevCfft& c, void* src, void* dst) {
    PassParams<Ar> p{};
    p.tw_stage = static_cast<const CxW<Ar>*>(c.tw_stage.p);
    p.tw4 = static_cast<const CxW<Ar>*>(c.tw4.p);
    p.odd = odd_table<typename Ar::W>();
    p.src = static_cast<CxR<Ar>*>(src);
    p.dst = static_cast<CxR<Ar>*>(dst);
    p.stride = sl.stride;
    p.task0 = sl.task0;
    p.work = sl.work;
    p.ddreal = sl.ddreal;
    return p;
}

// The smooth complex FFT `c` of every slot: input from SRC (x when complex; the four-step column pass works in
// place on x), result to y in natural order, or to the output epilogue (DST). ArL: four-step sub-FFT
// arithmetic; ArS: the direct transform's.
template <class ArL, class ArS, int SRC, int DST>
int launch_smooth(const DevCfft& c, const Slots& sl, void* x, void* y, cudaStream_t st, Trail& tr, int kA, int kB) {
    const HostCfft& h = c.host;
    int rc;
    if (h.four) {
        PassParams<ArL> p = pass_params<ArL>(sl, c, x, x);
        p.sp = h.s1; p.N1 = h.N1; p.N2 = h.N2; p.F = c.col.F;
        const unsigned groups = (unsigned)((h.N2 + p.F - 1) / p.F);
        const dim3 gc = SRC == kSrcSignal ? dim3((unsigned)sl.nt, groups) : dim3(groups, (unsigned)sl.nt);
        if constexpr (ArL::kWide) {
            if (c.col.twg) k_column<ArL, SRC, true><<<gc, c.col.T, c.col.smem, st>>>(p);
            else k_column<ArL, SRC, false><<<gc, c.col.T, c.col.smem, st>>>(p);
        } else {
            k_column<ArL, SRC, false><<<gc, c.col.T, c.col.smem, st>>>(p);
        }
        if ((rc = tr.mark(st, kA)) != KBSRC_GPU_OK) return rc;
        p.sp = h.s2; p.F = c.row.F; p.src = static_cast<CxR<ArL>*>(x); p.dst = static_cast<CxR<ArL>*>(y);
        const dim3 gr((h.N1 + p.F - 1) / p.F, sl.nt);
        if constexpr (ArL::kWide) {
            if (c.row.twg) k_row<ArL, DST, true><<<gr, c.row.T, c.row.smem, st>>>(p);
            else k_row<ArL, DST, false><<<gr, c.row.T, c.row.smem, st>>>(p);
        } else {
            k_row<ArL, DST, false><<<gr, c.row.T, c.row.smem, st>>>(p);
        }
        return tr.mark(st, kB);
    }
    PassParams<ArS> p = pass_params<ArS>(sl, c, x, y);
    p.sp = h.sd; p.F = 1;
    k_direct<ArS, SRC, DST><<<dim3(1, sl.nt), c.dir.T, c.dir.smem, st>>>(p);
    return tr.mark(st, kA);
}

// Any complex FFT: smooth, or Bluestein (pre -> inner -> kernel -> inner -> post) through the work buffers
// a and b (m values per slot each). x: complex input when SRC says so (read before a and b are written, so it
// may alias b); y: the result (may alias a), unless DST writes the output.
template <class ArL, class ArS, int SRC, int DST>
int launch_cfft(const DevCfft& c, const Slots& sl, void* x, void* a, void* b, void* y, cudaStream_t st, Trail& tr,
                int kA, int kB) {
    if (!c.m) return launch_smooth<ArL, ArS, SRC, DST>(c, sl, x, y, st, tr, kA, kB);
    int rc;
    PassParams<ArS> p = pass_params<ArS>(sl, c, x, a);
    p.bc = static_cast<const CxW<ArS>*>(c.bc.p);
    p.vf = static_cast<const CxW<ArS>*>(c.vf.p);
    p.bn = c.n;
    p.bm = c.m;
    const dim3 gm(grid_for(c.m, 256), sl.nt), gn(grid_for(c.n, 256), sl.nt);
    k_blue_pre<ArS, SRC><<<gm, 256, 0, st>>>(p);
    if ((rc = tr.mark(st, kA)) != KBSRC_GPU_OK) return rc;
    if ((rc = launch_smooth<ArL, ArS, kSrcComplex, kDstComplex>(*c.inner, sl, a, b, st, tr, kA, kB)) != KBSRC_GPU_OK)
        return rc;
    p.src = static_cast<CxR<ArS>*>(b);
    p.dst = static_cast<CxR<ArS>*>(a);
    k_blue_mid<ArS><<<gm, 256, 0, st>>>(p);
    if ((rc = tr.mark(st, kA)) != KBSRC_GPU_OK) return rc;
    if ((rc = launch_smooth<ArL, ArS, kSrcComplex, kDstComplex>(*c.inner, sl, a, b, st, tr, kA, kB)) != KBSRC_GPU_OK)
        return rc;
    p.src = static_cast<CxR<ArS>*>(b);
    p.dst = static_cast<CxR<ArS>*>(y);
    k_blue_post<ArS, DST><<<gn, 256, 0, st>>>(p);
    return tr.mark(st, kA);
}

// Vf = FFT(v)/m for Bluestein, v[t] = v[m-t] = e^{+i pi t^2/n} (fft.hpp:230-238): the m-point transform in
// scalar double-double (the reference's CFFT<dd,dd,dd>), divided by m in dd, stored in the engine's precision.
__global__ void k_vf_scale(const cx<dd>* __restrict__ V, int m, double* __restrict__ out, int tab) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const dd re = div_dd_f64(V[k].re, (double)m), im = div_dd_f64(V[k].im, (double)m);
        if (tab == kTabX80) {  // from_dd<long double>: (long double)hi + (long double)lo
            x80* o = reinterpret_cast<x80*>(out);
            o[2 * k] = x80_add(x80_from_f64(re.hi), x80_from_f64(re.lo));
            o[2 * k + 1] = x80_add(x80_from_f64(im.hi), x80_from_f64(im.lo));
        } else if (tab == kTabDD) {
            out[4 * k] = re.hi; out[4 * k + 1] = re.lo; out[4 * k + 2] = im.hi; out[4 * k + 3] = im.lo;
        } else {
            out[2 * k] = re.hi; out[2 * k + 1] = im.hi;
        }
    }
}

int bluestein_kernel(DevCfft& d, int tab, cudaStream_t st) {
    const int n = d.n, m = d.m;
    std::vector<HostCx> v((size_t)m);
    for (long long t = 0; t < n; t++) {
        const long long e = (long long)((__int128)t * t % (2LL * n));
        hd::unit_root(e, 2LL * n, v[t].re, v[t].im);
        if (t) v[m - t] = v[t];
    }
    DevCfft des;  // the same m-point plan with double-double tables, run in scalar dd
    int rc;
    if ((rc = make_dev_cfft(m, kTabDD, 4, des, st)) != KBSRC_GPU_OK) return rc;
    DevBuf vin, vout;
    if ((rc = upload_cx(v, kTabDD, vin)) != KBSRC_GPU_OK) return rc;
    if ((rc = vout.alloc((size_t)m * 32)) != KBSRC_GPU_OK) return rc;
    if ((rc = d.vf.alloc((size_t)m * tab_esize(tab))) != KBSRC_GPU_OK) return rc;
    Slots sl{};
    sl.nt = 1;
    Trail tr;
    if ((rc = launch_smooth<ArDDAccurate, ArDDAccurate, kSrcComplex, kDstComplex>(des, sl, vin.p, vout.p, st, tr, -1,
                                                                                  -1)) != KBSRC_GPU_OK)
        return rc;
    k_vf_scale<<<grid_for(m, 256), 256, 0, st>>>(static_cast<const cx<dd>*>(vout.p), m, static_cast<double*>(d.vf.p),
                                                  tab);
    KB_CUDA(cudaGetLastError());
    KB_CUDA(cudaStreamSynchronize(st));  // the temporaries are freed on return
    return KBSRC_GPU_OK;
}

// Enqueues the block loop of tasks [t_begin, t_end) of one plan, wave by wave through the slot buffers a, b.
// ArL: four-step sub-FFT arithmetic, ArS: everything else.
template <class ArL, class ArS>
int enqueue_plan(const PlanCore& pc, const Work& work, long long t_begin, long long t_end, void* a, void* b,
                 long long stride, long long wave, cudaStream_t st, Trail& tr) {
    static_assert(sizeof(CxR<ArL>) == sizeof(CxR<ArS>), "one element size per mode");
    using CS = CxR<ArS>;
    using WS = typename ArS::W;
    const kbsrc_gpu_desc& d = pc.d;
    Slots sl{};
    sl.stride = stride;
    sl.work = work;
    void* buf[2] = {a, b};
    int rc;
    for (long long t0 = t_begin; t0 < t_end; t0 += wave) {
        sl.task0 = t0;
        sl.nt = (unsigned)std::min(wave, t_end - t0);
        // forward real FFT: gather + complex FFT; the spectrum Z lands in buf[z]
        int z;
        if (pc.fw.m) {
            z = 0;
            rc = launch_cfft<ArL, ArS, kSrcSignal, kDstComplex>(pc.fw, sl, nullptr, buf[0], buf[1], buf[0], st, tr,
                                                                 kFwdA, kFwdB);
        } else {
            z = 1;
            rc = launch_cfft<ArL, ArS, kSrcSignal, kDstComplex>(pc.fw, sl, buf[0], nullptr, nullptr, buf[1], st, tr,
                                                                 kFwdA, kFwdB);
        }
        if (rc) return rc;
        // split into the real spectrum (buf[z] -> buf[1-z]), multiply/fold and merge (buf[1-z] -> buf[z])
        SpecParams<ArS> s{};
        s.Z = static_cast<CS*>(buf[z]);
        s.X = static_cast<CS*>(buf[1 - z]);
        s.Zi = static_cast<CS*>(buf[z]);
        s.stride = stride;
        s.w_fw = static_cast<const CxW<ArS>*>(pc.w_fw.p);
        s.w_iv = static_cast<const CxW<ArS>*>(pc.w_iv.p);
        s.H = static_cast<const WS*>(pc.H.p);
        s.h = pc.hf; s.hi = pc.hi; s.Nb = pc.Nb; s.Mb = pc.Mb; s.up = d.up; s.Jg = d.Jg;
        const dim3 gmerge(grid_for(pc.hi / 2 + 1 + (ArS::kWide ? 0 : pc.hi / 2), 256), sl.nt);
        int zi = z;  // the buffer that holds the inverse FFT's input
        if constexpr (ArS::kWide) {
            k_split<ArS><<<dim3(grid_for(pc.hf / 2 + 1, 256), sl.nt), 256, 0, st>>>(s);
            if ((rc = tr.mark(st, kSplit)) != KBSRC_GPU_OK) return rc;
            k_merge<ArS><<<gmerge, 256, 0, st>>>(s);
        } else {  // float64: one pass from Z (buf[z]) to the inverse input in buf[1-z]
            zi = 1 - z;
            s.Zi = static_cast<CS*>(buf[zi]);
            k_spectrum_z<ArS><<<gmerge, 256, 0, st>>>(s);
        }
        if ((rc = tr.mark(st, kMerge)) != KBSRC_GPU_OK) return rc;
        // inverse complex FFT of buf[zi] and the output epilogue
        rc = launch_cfft<ArL, ArS, kSrcComplex, kDstOutput>(pc.iv, sl, buf[zi], buf[1 - zi], buf[zi], nullptr, st, tr,
                                                             kInvA, kInvB);
        if (rc) return rc;
    }
    return KBSRC_GPU_OK;
}

// One split-form transform of every slot: column pass (x in place, or straight to y / the output when N2 == 1),
// then the row pass x -> y or to the output epilogue (DST).
template <class S, int SRC, int DST>
int launch_tc(const TcFftDev& t, const Slots& sl, void* x, void* y, int* err, cudaStream_t st, Trail& tr, int kA,
              int kB) {
    PassParams<ArF64> p{};
    p.src = static_cast<CxR<ArF64>*>(x);
    p.dst = static_cast<CxR<ArF64>*>(t.N2 == 1 ? y : x);
    p.stride = sl.stride;
    p.task0 = sl.task0;
    p.work = sl.work;
    TcParams T{};
    T.sub = t.col;
    T.tw4 = t.N2 > 1 ? static_cast<const double2*>(t.tw4.p) : nullptr;
    T.N1 = t.N1;
    T.N2 = t.N2;
    T.slots = (int)sl.nt;
    T.err = err;
    // persistent CTAs, one per SM at most, each working on `halves` items at once
    auto grid = [&](long long items, int halves) {
        return (unsigned)std::max(1LL, std::min((items + halves - 1) / halves, (long long)t.ctas));
    };
    auto column = [&](auto kernel, long long items) {
        kernel<<<grid(items, T.sub.halves), kTcThreads, t.smem_col, st>>>(p, T);
    };
    const long long col_items = t.N2 == 1 ? (long long)sl.nt : (long long)((t.N2 + t.col.F - 1) / t.col.F) * sl.nt;
    if (t.N2 == 1) {
        if (T.sub.halves == 2) column(k_tc_column<S, SRC, DST, 2>, col_items);
        else column(k_tc_column<S, SRC, DST, 1>, col_items);
        return tr.mark(st, kA);
    }
    if (T.sub.halves == 2) column(k_tc_column<S, SRC, kDstComplex, 2>, col_items);
    else column(k_tc_column<S, SRC, kDstComplex, 1>, col_items);
    int rc = tr.mark(st, kA);
    if (rc) return rc;
    p.src = static_cast<CxR<ArF64>*>(x);
    p.dst = static_cast<CxR<ArF64>*>(y);
    T.sub = t.row;
    T.tw4 = nullptr;
    const long long row_items = (long long)((t.N1 + t.row.F - 1) / t.row.F) * sl.nt;
    if (T.sub.halves == 2)
        k_tc_row<S, DST, 2><<<grid(row_items, 2), kTcThreads, t.smem_row, st>>>(p, T);
    else
        k_tc_row<S, DST, 1><<<grid(row_items, 1), kTcThreads, t.smem_row, st>>>(p, T);
    return tr.mark(st, kB);
}

// The block loop in the split-precision form: tensor-core transforms, float64 split, spectrum and merge. S: the
// digit slices' element kind.
template <class S>
int enqueue_split(const PlanCore& pc, const Work& work, long long t_begin, long long t_end, void* a, void* b,
                  long long stride, long long wave, cudaStream_t st, Trail& tr) {
    const kbsrc_gpu_desc& d = pc.d;
    int* err = static_cast<int*>(pc.tc_err.p);
    Slots sl{};
    sl.stride = stride;
    sl.work = work;
    int rc;
    for (long long t0 = t_begin; t0 < t_end; t0 += wave) {
        sl.task0 = t0;
        sl.nt = (unsigned)std::min(wave, t_end - t0);
        if ((rc = launch_tc<S, kSrcSignal, kDstComplex>(pc.tfw, sl, a, b, err, st, tr, kFwdA, kFwdB)) != KBSRC_GPU_OK)
            return rc;
        // float64 split, spectrum and merge in one pass: Z in b, the inverse input to a
        SpecParams<ArF64> s{};
        s.Z = static_cast<CxR<ArF64>*>(b);
        s.Zi = static_cast<CxR<ArF64>*>(a);
        s.stride = stride;
        s.w_fw = static_cast<const CxW<ArF64>*>(pc.w_fw.p);
        s.w_iv = static_cast<const CxW<ArF64>*>(pc.w_iv.p);
        s.H = static_cast<const double*>(pc.H.p);
        s.h = pc.hf; s.hi = pc.hi; s.Nb = pc.Nb; s.Mb = pc.Mb; s.up = d.up; s.Jg = d.Jg;
        k_spectrum_z<ArF64><<<dim3(grid_for(pc.hi, 256), sl.nt), 256, 0, st>>>(s);
        if ((rc = tr.mark(st, kMerge)) != KBSRC_GPU_OK) return rc;
        if ((rc = launch_tc<S, kSrcComplex, kDstOutput>(pc.tiv, sl, a, nullptr, err, st, tr, kInvA, kInvB)) !=
            KBSRC_GPU_OK)
            return rc;
    }
    return KBSRC_GPU_OK;
}

int enqueue_any(const PlanCore& pc, const Work& work, long long t_begin, long long t_end, void* a, void* b,
                long long stride, long long wave, cudaStream_t st, Trail& tr) {
    if (pc.split && pc.tfw.eb == 2) return enqueue_split<TcF16>(pc, work, t_begin, t_end, a, b, stride, wave, st, tr);
    if (pc.split) return enqueue_split<TcI8>(pc, work, t_begin, t_end, a, b, stride, wave, st, tr);
    if (pc.tab == kTabX80) return enqueue_plan<ArX80, ArX80>(pc, work, t_begin, t_end, a, b, stride, wave, st, tr);
    if (pc.exact) return enqueue_plan<ArDDShort, ArDDAccurate>(pc, work, t_begin, t_end, a, b, stride, wave, st, tr);
    return enqueue_plan<ArF64, ArF64>(pc, work, t_begin, t_end, a, b, stride, wave, st, tr);
}

// The share of a descriptor that an engine runs: its own shard, or the whole conversion when the shard is zero.
kbsrc_gpu_shard effective_shard(const kbsrc_gpu_desc& d) {
    if (d.shard.blk1 > 0) return d.shard;
    return kbsrc_gpu_shard{0, d.nblk, 0, d.frames, 0, d.nout};
}

Work single_work(const PlanCore& pc, const double* in, const double* head, const double* tail, double* out) {
    const kbsrc_gpu_desc& d = pc.d;
    const kbsrc_gpu_shard sh = effective_shard(d);
    Work w{};
    w.item0 = Item{in, head, tail, out, d.frames, d.edge_len, d.lead, d.nout, d.o, d.channels, d.in_format,
                   sh.frame0, sh.out0, sh.nout};
    w.hopQ = (long long)pc.hop * d.Q;
    w.hopP = (long long)pc.hop * d.P;
    w.margP = (long long)d.marg * d.P;
    return w;
}

long long cfft_launches(const DevCfft& c) {
    if (c.m) return 3 + 2 * cfft_launches(*c.inner);
    return c.host.four ? 2 : 1;
}

size_t cfft_bytes(const DevCfft& c) {
    size_t b = c.tw_stage.bytes + c.tw4.bytes + c.bc.bytes + c.vf.bytes;
    return c.m ? b + cfft_bytes(*c.inner) : b;
}

// Kernel launches of one wave, and the device bytes of the plan's tables
long long plan_launches(const PlanCore& pc) {
    if (pc.split) return (pc.tfw.N2 > 1 ? 2 : 1) + 1 + (pc.tiv.N2 > 1 ? 2 : 1);
    const int spectrum = pc.exact || pc.tab == kTabX80 ? 2 : 1;  // float64 fuses split, spectrum and merge
    return cfft_launches(pc.fw) + spectrum + cfft_launches(pc.iv);
}
size_t plan_table_bytes(const PlanCore& pc) {
    return cfft_bytes(pc.fw) + cfft_bytes(pc.iv) + pc.tfw.bytes() + pc.tiv.bytes() + pc.w_fw.bytes + pc.w_iv.bytes +
           pc.H.bytes;
}

// After a synchronous run of the split form: a tensor-core stage that timed out is an error (the flag is reset)
int check_tc(const PlanCore& pc) {
    if (!pc.split || !pc.tc_err.p) return KBSRC_GPU_OK;
    int flag = 0;
    KB_CUDA(cudaMemcpy(&flag, pc.tc_err.p, sizeof flag, cudaMemcpyDeviceToHost));
    if (!flag) return KBSRC_GPU_OK;
    KB_CUDA(cudaMemset(pc.tc_err.p, 0, sizeof flag));
    return fail(KBSRC_GPU_E_CUDA, "split-precision form: a tensor-core stage did not complete");
}

// The input frames blocks [b0, b1) read (staged samples [b*hop*Q, b*hop*Q + nb*Q) of each block, frame = staged
// sample - lead, clipped to the signal) and the output samples they write ([b*hop*P - o, (b+1)*hop*P - o) clipped
// to [0, nout)).
int shard_span(const kbsrc_gpu_desc& d, long long b0, long long b1, kbsrc_gpu_shard& s) {
    const long long hop = d.nb - 2LL * d.marg, hopQ = hop * d.Q, hopP = hop * d.P, Nb = (long long)d.nb * d.Q;
    s.blk0 = b0;
    s.blk1 = b1;
    const long long f0 = std::max(0LL, b0 * hopQ - d.lead), f1 = std::min(d.frames, (b1 - 1) * hopQ + Nb - d.lead);
    s.frame0 = std::min(f0, d.frames);
    s.frames = std::max(0LL, f1 - s.frame0);
    const long long o0 = std::min(d.nout, std::max(0LL, b0 * hopP - d.o)),
                    o1 = std::min(d.nout, std::max(0LL, b1 * hopP - d.o));
    s.out0 = o0;
    s.nout = std::max(0LL, o1 - o0);
    return KBSRC_GPU_OK;
}

int check_desc(const kbsrc_gpu_desc* d) {
    if (!d) return fail(KBSRC_GPU_E_ARG, "null descriptor");
    if (d->precision != KBSRC_GPU_FAST && d->precision != KBSRC_GPU_EXACT && d->precision != KBSRC_GPU_LD &&
        d->precision != KBSRC_GPU_SPLIT && d->precision != KBSRC_GPU_SPLIT_F16)
        return fail(KBSRC_GPU_E_ARG, "precision");
    if (d->channels < 1 || d->P < 1 || d->Q < 1 || d->nb < 2 || d->nb % 2 || d->marg < 0 || d->nb <= 2 * d->marg)
        return fail(KBSRC_GPU_E_ARG, "bad plan shape");
    if (d->frames < 0 || d->nout < 0 || d->nblk < 0 || d->edge_len < 0 || d->lead < 0 || d->Jg < 0)
        return fail(KBSRC_GPU_E_ARG, "bad plan sizes");
    if (d->in_format < KBSRC_GPU_IN_F64 || d->in_format > KBSRC_GPU_IN_U8) return fail(KBSRC_GPU_E_ARG, "input format");
    if ((long long)d->nb * std::max(d->P, d->Q) > (1LL << 30)) return fail(KBSRC_GPU_E_ARG, "transform too large");
    const long long need = d->Jg ? (long long)d->Jg + 1 : (d->up ? d->nb * d->P / 2 + 1 : d->nb * d->Q / 2 + 1);
    if (!d->H || d->H_len < need) return fail(KBSRC_GPU_E_ARG, "kernel spectrum too short");
    const kbsrc_gpu_shard& s = d->shard;
    if (s.blk0 || s.blk1 || s.frame0 || s.frames || s.out0 || s.nout) {
        // a share must hold every input frame its blocks read and every output sample they write: the kernels
        // index its buffers relative to frame0 and out0 without further checks on the input side
        kbsrc_gpu_shard want;
        if (s.blk0 < 0 || s.blk1 <= s.blk0 || s.blk1 > d->nblk || s.frame0 < 0 || s.frames < 0 ||
            s.frame0 + s.frames > d->frames || s.out0 < 0 || s.nout < 0 || s.out0 + s.nout > d->nout ||
            shard_span(*d, s.blk0, s.blk1, want) != KBSRC_GPU_OK ||
            (want.frames > 0 && (want.frame0 < s.frame0 || want.frame0 + want.frames > s.frame0 + s.frames)) ||
            (want.nout > 0 && (want.out0 < s.out0 || want.out0 + want.nout > s.out0 + s.nout)))
            return fail(KBSRC_GPU_E_ARG, "shard does not hold the input span or output range of its blocks");
    }
    return KBSRC_GPU_OK;
}

int upload_real(const double* hilo, long long n, int tab, DevBuf& out) {
    if (tab == kTabX80) {
        std::vector<x80> v((size_t)n);
        for (long long i = 0; i < n; i++) v[i] = host_x80(hd::dd{hilo[2 * i], hilo[2 * i + 1]});
        int rc = out.alloc(v.size() * sizeof(x80));
        if (rc) return rc;
        KB_CUDA(cudaMemcpy(out.p, v.data(), v.size() * sizeof(x80), cudaMemcpyHostToDevice));
        return KBSRC_GPU_OK;
    }
    std::vector<double> v;
    if (tab == kTabDD) v.assign(hilo, hilo + 2 * n);
    else {
        v.resize((size_t)n);
        for (long long i = 0; i < n; i++) v[i] = hilo[2 * i];
    }
    int rc = out.alloc(v.size() * sizeof(double));
    if (rc) return rc;
    KB_CUDA(cudaMemcpy(out.p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
    return KBSRC_GPU_OK;
}

// Builds the plan of a descriptor (check_desc first): FFT tables, split/merge roots, kernel spectrum.
int make_core(const kbsrc_gpu_desc* desc, PlanCore& pc, cudaStream_t st) {
    int rc;
    pc.d = *desc;
    pc.d.H = nullptr;
    pc.exact = desc->precision == KBSRC_GPU_EXACT;
    pc.split = desc->precision == KBSRC_GPU_SPLIT || desc->precision == KBSRC_GPU_SPLIT_F16;
    pc.tab = desc->precision == KBSRC_GPU_FAST || pc.split ? kTabF64
             : desc->precision == KBSRC_GPU_EXACT          ? kTabDD
                                                           : kTabX80;
    pc.Nb = (int)(desc->nb * desc->Q);
    pc.Mb = (int)(desc->nb * desc->P);
    pc.hf = pc.Nb / 2;
    pc.hi = pc.Mb / 2;
    pc.hop = desc->nb - 2 * desc->marg;
    const int fmax = env_int("KBSRC_GPU_FMAX", pc.tab == kTabF64 ? 5 : 8);
    if (pc.split) {
        const int eb = desc->precision == KBSRC_GPU_SPLIT_F16 ? 2 : 1;
        if ((rc = make_tc_fft(pc.hf, eb, pc.tfw)) != KBSRC_GPU_OK) return rc;
        if ((rc = make_tc_fft(pc.hi, eb, pc.tiv)) != KBSRC_GPU_OK) return rc;
        if ((rc = pc.tc_err.alloc(16)) != KBSRC_GPU_OK) return rc;
        KB_CUDA(cudaMemset(pc.tc_err.p, 0, 16));
    } else {
        if ((rc = make_dev_cfft(pc.hf, pc.tab, fmax, pc.fw, st)) != KBSRC_GPU_OK) return rc;
        if ((rc = make_dev_cfft(pc.hi, pc.tab, fmax, pc.iv, st)) != KBSRC_GPU_OK) return rc;
    }
    if ((rc = upload_cx(split_roots(pc.Nb), pc.tab, pc.w_fw)) != KBSRC_GPU_OK) return rc;
    if ((rc = upload_cx(split_roots(pc.Mb), pc.tab, pc.w_iv)) != KBSRC_GPU_OK) return rc;
    return upload_real(desc->H, desc->H_len, pc.tab, pc.H);
}

int create_impl(const kbsrc_gpu_desc* desc, kbsrc_gpu_engine** out) {
    int rc = check_desc(desc);
    if (rc) return rc;
    if ((rc = require_device()) != KBSRC_GPU_OK) return rc;
    if ((rc = allow_large_smem()) != KBSRC_GPU_OK) return rc;
    auto* e = new kbsrc_gpu_engine();
    struct Guard {
        kbsrc_gpu_engine* p;
        ~Guard() { delete p; }
    } guard{e};
    KB_CUDA(cudaGetDevice(&e->device));
    KB_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    if ((rc = make_core(desc, *e, e->stream)) != KBSRC_GPU_OK) return rc;
    const kbsrc_gpu_shard sh = effective_shard(*desc);
    e->t_begin = sh.blk0 * desc->channels;
    e->t_end = sh.blk1 * desc->channels;
    e->tasks = e->t_end - e->t_begin;
    e->stride = e->slot();
    const long long budget = (long long)env_int("KBSRC_GPU_WAVE_MB", 4096) << 20;
    const long long per_task = 2 * e->stride * (long long)e->esize();
    e->wave = std::max(1LL, std::min({e->tasks, budget / per_task, 65535LL}));
    if (e->tasks > 0) {
        if ((rc = e->bufA.alloc((size_t)(e->wave * e->stride * e->esize()))) != KBSRC_GPU_OK) return rc;
        if ((rc = e->bufB.alloc((size_t)(e->wave * e->stride * e->esize()))) != KBSRC_GPU_OK) return rc;
    }
    guard.p = nullptr;
    *out = e;
    return KBSRC_GPU_OK;
}

int run_device_impl(kbsrc_gpu_engine* e, const double* in, const double* head, const double* tail, double* out,
                    cudaStream_t st, Trail* trail = nullptr) {
    const kbsrc_gpu_desc& d = e->d;
    const kbsrc_gpu_shard sh = effective_shard(d);
    if (sh.nout > 0) KB_CUDA(cudaMemsetAsync(out, 0, (size_t)sh.nout * d.channels * sizeof(double), st));
    if (e->tasks == 0 || sh.nout == 0) return KBSRC_GPU_OK;
    if (d.frames > 0 && !in) return fail(KBSRC_GPU_E_ARG, "null input");
    if (d.edge_len > 0 && (!head || !tail)) return fail(KBSRC_GPU_E_ARG, "null edge buffers");
    Trail none;
    Trail& tr = trail ? *trail : none;
    int rc;
    if ((rc = tr.mark(st, -1)) != KBSRC_GPU_OK) return rc;
    rc = enqueue_any(*e, single_work(*e, in, head, tail, out), e->t_begin, e->t_end, e->bufA.p, e->bufB.p, e->stride,
                     e->wave, st, tr);
    if (rc) return rc;
    e->launches = tr.launches;
    KB_CUDA(cudaGetLastError());
    return KBSRC_GPU_OK;
}

}  // namespace

// ------------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------------
// ---- output conversion: WAV sample packing and TPDF dither on the GPU -------------------------------------------
//
// The reference's writer (src/io/wav.cpp:242-255,371-418) interleaves the planar output and, for integer
// formats, scales by 2^(8B-1), adds two draws of uniform_real_distribution<double>(-0.5, 0.5) from
// std::mt19937_64 seeded 12345 per sample (frame-major, channel-minor), rounds to nearest, clips and counts the
// clipped samples. The packer reproduces it sample for sample; the dither stream is the same generator run on the
// GPU (MT19937-64, Matsumoto and Nishimura 2000). The stream is cut into chunks of 2^20 draws; a jump-ahead tree
// finds each chunk's start state and one CTA per chunk then runs the generator: it updates the 312-word state in
// parallel in the order the sequential twist would and tempers 312 outputs, two per sample.
namespace {

constexpr int kMtN = 312, kMtM = 156;
constexpr unsigned long long kMtA = 0xB5026F5AA96619E9ULL, kMtUpper = 0xFFFFFFFF80000000ULL,
                             kMtLower = 0x7FFFFFFFULL;

__device__ __forceinline__ unsigned long long mt_temper(unsigned long long y) {
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= y >> 43;
    return y;
}

// uniform_real_distribution<double>(-0.5, 0.5) of one 64-bit draw: u / 2^64 (kept below 1), times (b - a), plus a
__device__ __forceinline__ double mt_uniform(unsigned long long u) {
    double r = __ddiv_rn(__ull2double_rn(u), 18446744073709551616.0);
    if (r >= 1.0) r = 0x1.fffffffffffffp-1;
    return __dadd_rn(__dmul_rn(r, 1.0), -0.5);
}

__device__ __forceinline__ unsigned long long mt_twist(unsigned long long a, unsigned long long b) {
    const unsigned long long x = (a & kMtUpper) | (b & kMtLower);
    return (x >> 1) ^ ((x & 1) ? kMtA : 0ULL);
}

// Jump-ahead (Haramoto, Matsumoto, Nishimura, Panneton and L'Ecuyer 2008, "Efficient jump ahead for F2-linear
// random number generators"). The generator is linear over GF(2). Write x_k for its untempered words (x_0..x_311
// the seeded state, draw d = temper(x_{312+d})) and W_k = (x_k .. x_{k+311}) for the window at k. For k >= 1 the
// windows lie in the 19937-dimensional subspace on which the transition A has the primitive characteristic
// polynomial phi, so A^J W = g(A) W for g = x^J mod phi, and word i of g(A) W_s is the XOR of x_{s+k+i} over the
// set coefficients k of g. kMtChunk draws make one chunk; W[c] holds the window x_{312+c*kMtChunk} .. .
constexpr int kMtDeg = 19937;                            // degree of phi; polynomials below it fit kMtN words
constexpr int kMtSeq = kMtDeg + kMtN;                    // words x_s .. x_{s+20248} the jump reads
constexpr long long kMtChunk = 1LL << 20;                // draws per chunk (even: a chunk holds whole samples)
constexpr int kMtJumpParts = 3, kMtJumpThreads = 320 * kMtJumpParts;
constexpr size_t kMtJumpSmem = (size_t)(kMtSeq + kMtN + kMtJumpParts * kMtN) * 8;

// W[b + half] = g(A) W[b] for b < min(half, G - half): one level of the doubling tree of chunk starts
__global__ void __launch_bounds__(kMtJumpThreads) k_mt_jump(const unsigned long long* __restrict__ g,
                                                           unsigned long long* __restrict__ W, int half, int G) {
    extern __shared__ __align__(16) unsigned long long mt_sh[];
    unsigned long long* X = mt_sh;             // kMtSeq words of the sequence from W[b]
    unsigned long long* gs = X + kMtSeq;       // kMtN words of g
    unsigned long long* part = gs + kMtN;      // kMtJumpParts x kMtN partial sums
    const int b = blockIdx.x, t = threadIdx.x;
    if (b + half >= G) return;
    for (int i = t; i < kMtN; i += blockDim.x) {
        X[i] = W[(size_t)b * kMtN + i];
        gs[i] = g[i];
    }
    __syncthreads();
    // X[j + 312] = X[j + 156] ^ twist(X[j], X[j + 1]); 156 consecutive j only read words written before them
    for (int base = kMtN; base < kMtSeq; base += kMtN - kMtM) {
        const int o = base + t;
        if (t < kMtN - kMtM && o < kMtSeq) X[o] = X[o - kMtM] ^ mt_twist(X[o - kMtN], X[o - kMtN + 1]);
        __syncthreads();
    }
    const int p = t / 320, i = t % 320;
    if (i < kMtN) {
        unsigned long long acc = 0;
        constexpr int per = kMtN / kMtJumpParts;
        for (int w = p * per; w < (p + 1) * per; w++) {  // g's bits are warp-uniform: no divergence
            unsigned long long gw = gs[w];
            while (gw) {
                const int k = 64 * w + __ffsll((long long)gw) - 1;  // k < kMtDeg, so k + i < kMtSeq
                gw &= gw - 1;
                acc ^= X[k + i];
            }
        }
        part[p * kMtN + i] = acc;
    }
    __syncthreads();
    if (t < kMtN) {
        unsigned long long v = 0;
#pragma unroll
        for (int q = 0; q < kMtJumpParts; q++) v ^= part[q * kMtN + t];
        W[(size_t)(b + half) * kMtN + t] = v;
    }
}

// D[k] = U(draw 2k) + U(draw 2k+1) for k < n: the dither added to sample k (frame-major, channel-minor). Block c
// makes the kMtChunk draws of chunk c from its start window W[c]: 312 draws from the window, then a twist.
__global__ void __launch_bounds__(320) k_mt_chunks(const unsigned long long* __restrict__ W, long long n,
                                                   double* __restrict__ D) {
    __shared__ unsigned long long st[kMtN];
    const int t = threadIdx.x;
    const long long k0 = blockIdx.x * (kMtChunk / 2), k1 = min(n, k0 + kMtChunk / 2);
    if (t < kMtN) st[t] = W[(size_t)blockIdx.x * kMtN + t];
    __syncthreads();
    for (long long base = k0; base < k1; base += kMtN / 2) {
        if (t < kMtN / 2 && base + t < k1)
            D[base + t] = __dadd_rn(mt_uniform(mt_temper(st[2 * t])), mt_uniform(mt_temper(st[2 * t + 1])));
        unsigned long long a = 0, b = 0;
        if (t < kMtN) {
            a = st[t];
            if (t + 1 < kMtN) b = st[t + 1];
        }
        __syncthreads();
        if (t < kMtN - kMtM) st[t] = st[t + kMtM] ^ mt_twist(a, b);  // words 0..155 read only old words
        __syncthreads();
        if (t >= kMtN - kMtM && t < kMtN) {  // words 156..311 read the new words t-156 (and 0 for the last)
            if (t == kMtN - 1) b = st[0];
            st[t] = st[t - (kMtN - kMtM)] ^ mt_twist(a, b);
        }
        __syncthreads();
    }
}

// ---- host side of the jump: phi by Berlekamp-Massey, the jump polynomials by squaring mod phi -------------------
using Words = std::vector<unsigned long long>;

unsigned long long mt_twist_h(unsigned long long a, unsigned long long b) {
    const unsigned long long x = (a & kMtUpper) | (b & kMtLower);
    return (x >> 1) ^ ((x & 1) ? kMtA : 0ULL);
}

// untempered words x_0 .. x_{n-1} of mt19937_64(seed), n >= 312
Words mt_words(unsigned long long seed, size_t n) {
    Words x(n);
    x[0] = seed;
    for (int i = 1; i < kMtN; i++) x[i] = 6364136223846793005ULL * (x[i - 1] ^ (x[i - 1] >> 62)) + (unsigned long long)i;
    for (size_t k = kMtN; k < n; k++) x[k] = x[k - kMtM] ^ mt_twist_h(x[k - kMtN], x[k - kMtN + 1]);
    return x;
}

inline unsigned long long bits64(const Words& v, long long pos) {  // bits pos .. pos+63 of v (zero beyond)
    const size_t w = (size_t)(pos >> 6);
    const int s = (int)(pos & 63);
    const unsigned long long lo = w < v.size() ? v[w] : 0, hi = w + 1 < v.size() ? v[w + 1] : 0;
    return s ? (lo >> s) | (hi << (64 - s)) : lo;
}

void xor_shifted(Words& c, const Words& b, long long m, size_t bwords) {  // c ^= b * x^m
    const size_t w = (size_t)(m >> 6);
    const int s = (int)(m & 63);
    for (size_t i = 0; i < bwords && i + w < c.size(); i++) {
        c[i + w] ^= b[i] << s;
        if (s && i + w + 1 < c.size()) c[i + w + 1] ^= b[i] >> (64 - s);
    }
}

// Characteristic polynomial (bit j = coefficient of x^j) of bit 0 of x_312, x_313, ...; degree kMtDeg
Words mt_phi() {
    const int N = 2 * kMtDeg + 128;
    const Words x = mt_words(12345, (size_t)N + kMtN);
    const size_t nw = (size_t)(2 * N) / 64 + 4;
    Words rs(nw, 0), C(nw, 0), B(nw, 0), T;
    for (int n = 0; n < N; n++)  // s_n at bit N-1-n, so s_{n-i}, i = 0.. are consecutive bits from N-1-n
        if (x[kMtN + n] & 1) rs[(size_t)(N - 1 - n) >> 6] |= 1ULL << ((N - 1 - n) & 63);
    C[0] = B[0] = 1;
    int L = 0;
    long long m = 1;
    for (int n = 0; n < N; n++) {
        unsigned long long acc = 0;  // discrepancy: sum_{i<=L} c_i s_{n-i}
        for (int w = 0; w <= L / 64; w++) acc ^= C[(size_t)w] & bits64(rs, (long long)(N - 1 - n) + 64LL * w);
        if (!(__builtin_popcountll(acc) & 1)) {
            m++;
            continue;
        }
        const size_t bw = (size_t)n / 64 + 2;
        if (2 * L <= n) {
            T = C;
            xor_shifted(C, B, m, bw);
            L = n + 1 - L;
            B.swap(T);
            m = 1;
        } else {
            xor_shifted(C, B, m, bw);
            m++;
        }
    }
    if (L != kMtDeg) throw std::runtime_error("dither jump: unexpected linear complexity");
    Words phi((size_t)kMtN + 1, 0);  // phi = x^L + c_1 x^(L-1) + ... + c_L
    for (int i = 0; i <= L; i++)
        if ((C[(size_t)i >> 6] >> (i & 63)) & 1) phi[(size_t)(L - i) >> 6] |= 1ULL << ((L - i) & 63);
    return phi;
}

inline unsigned long long spread32(unsigned long long v) {  // bit j -> bit 2j
    v &= 0xFFFFFFFFULL;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFULL;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFULL;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0FULL;
    v = (v | (v << 2)) & 0x3333333333333333ULL;
    v = (v | (v << 1)) & 0x5555555555555555ULL;
    return v;
}

struct MtJumpTables {
    std::vector<Words> phis;  // phi * x^s, s = 0..63
    std::vector<Words> g;     // g[l] = x^(2^l kMtChunk) mod phi, kMtN words each
    Words w312;               // x_312 .. x_623 of mt19937_64(12345)
};

Words sqr_mod(const Words& a, const std::vector<Words>& phis) {  // a^2 mod phi, deg a < kMtDeg
    Words pr(2 * (size_t)kMtN + 2, 0);
    for (int w = 0; w < kMtN; w++) {
        pr[2 * (size_t)w] = spread32(a[(size_t)w]);
        pr[2 * (size_t)w + 1] = spread32(a[(size_t)w] >> 32);
    }
    for (long long p = 2LL * (kMtDeg - 1); p >= kMtDeg; p--) {
        if (!((pr[(size_t)p >> 6] >> (p & 63)) & 1)) continue;
        const long long q = p - kMtDeg;  // pr ^= phi * x^q clears bit p
        const Words& ph = phis[(size_t)(q & 63)];
        const size_t w0 = (size_t)(q >> 6);
        for (size_t i = 0; i < ph.size() && w0 + i < pr.size(); i++) pr[w0 + i] ^= ph[i];
    }
    pr.resize(kMtN);
    return pr;
}

// word i of g(A) W_s from the sequence X = x_s .. x_{s + kMtSeq - 1}
Words mt_apply_h(const Words& g, const Words& X) {
    Words out(kMtN, 0);
    for (int k = 0; k < kMtDeg; k++)
        if ((g[(size_t)k >> 6] >> (k & 63)) & 1)
            for (int i = 0; i < kMtN; i++) out[(size_t)i] ^= X[(size_t)(k + i)];
    return out;
}

// The tables with at least `levels` jump polynomials, built once per process (and extended on demand). The first
// polynomial is checked against the directly generated window 2^20 draws ahead.
const MtJumpTables& mt_tables(int levels) {
    static MtJumpTables t;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (t.phis.empty()) {
        const Words phi = mt_phi();
        for (int s = 0; s < 64; s++) {
            Words v((size_t)kMtN + 2, 0);
            xor_shifted(v, phi, s, phi.size());
            t.phis.push_back(std::move(v));
        }
        Words g(kMtN, 0);
        g[0] = 2;  // x
        for (long long e = 1; e < kMtChunk; e *= 2) g = sqr_mod(g, t.phis);
        const Words x = mt_words(12345, (size_t)(kMtN + kMtChunk + kMtSeq));
        t.w312.assign(x.begin() + kMtN, x.begin() + 2 * kMtN);
        const Words want(x.begin() + kMtN + kMtChunk, x.begin() + 2 * kMtN + kMtChunk);
        if (mt_apply_h(g, Words(x.begin() + kMtN, x.begin() + kMtN + kMtSeq)) != want)
            throw std::runtime_error("dither jump: self-check failed");
        t.g.push_back(std::move(g));
    }
    while ((int)t.g.size() < levels) t.g.push_back(sqr_mod(t.g.back(), t.phis));
    return t;
}

// Enqueues D[0..n) (the dither of n samples) on `st`; tmp receives chunk windows and jump polynomials.
int enqueue_dither(long long n, double* D, DevBuf& tmp, cudaStream_t st) {
    if (n <= 0) return KBSRC_GPU_OK;
    const long long G = (2 * n + kMtChunk - 1) / kMtChunk;
    if (G > (1LL << 30)) return fail(KBSRC_GPU_E_ARG, "dither stream too long");
    int levels = 0;
    while ((1LL << levels) < G) levels++;
    static bool smem_done[64] = {};
    static std::mutex mu;
    int dev = 0;
    KB_CUDA(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lock(mu);
        if (dev >= 64 || !smem_done[dev]) {
            KB_CUDA(cudaFuncSetAttribute((const void*)k_mt_jump, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kMtJumpSmem));
            if (dev < 64) smem_done[dev] = true;
        }
    }
    const MtJumpTables& tb = mt_tables(std::max(levels, 1));
    Words host((size_t)(G + levels) * kMtN, 0);  // W[0], then the level polynomials
    std::copy(tb.w312.begin(), tb.w312.end(), host.begin());
    for (int l = 0; l < levels; l++) std::copy(tb.g[(size_t)l].begin(), tb.g[(size_t)l].end(), host.begin() + (size_t)(G + l) * kMtN);
    int rc;
    if ((rc = tmp.alloc(host.size() * 8)) != KBSRC_GPU_OK) return rc;
    unsigned long long* W = static_cast<unsigned long long*>(tmp.p);
    KB_CUDA(cudaMemcpyAsync(W, host.data(), (size_t)kMtN * 8, cudaMemcpyHostToDevice, st));
    if (levels)
        KB_CUDA(cudaMemcpyAsync(W + (size_t)G * kMtN, host.data() + (size_t)G * kMtN, (size_t)levels * kMtN * 8,
                                cudaMemcpyHostToDevice, st));
    for (int l = 0; l < levels; l++) {
        const long long half = 1LL << l;
        k_mt_jump<<<(unsigned)std::min(half, G - half), kMtJumpThreads, kMtJumpSmem, st>>>(
            W + (size_t)(G + l) * kMtN, W, (int)half, (int)G);
    }
    k_mt_chunks<<<(unsigned)G, 320, 0, st>>>(W, n, D);
    KB_CUDA(cudaGetLastError());
    return KBSRC_GPU_OK;  // copies from pageable memory have left `host` when cudaMemcpyAsync returns
}

// Jump polynomials that enqueue_dither(n, ...) needs, built on a host thread beside other work (0 if none)
int dither_levels(long long n) {
    const long long G = (2 * n + kMtChunk - 1) / kMtChunk;
    int levels = 0;
    while ((1LL << levels) < G && levels < 40) levels++;
    return levels;
}

// Interleaved little-endian WAV data of planar samples y (ch x frames, row stride `stride`)
template <int FMT>  // 0 f64, 1 f32, 2 s32, 3 s24, 4 s16
__global__ void k_pack(const double* __restrict__ y, int ch, long long frames, long long stride,
                       const double* __restrict__ D, unsigned char* __restrict__ out,
                       unsigned long long* __restrict__ clipped) {
    constexpr int B = FMT == 0 ? 8 : FMT == 1 ? 4 : FMT == 2 ? 4 : FMT == 3 ? 3 : 2;
    constexpr double sc = FMT == 4 ? 32768.0 : FMT == 3 ? 8388608.0 : 2147483648.0;
    const long long n = frames * ch;
    unsigned long long clip = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const long long i = s / ch;
        const int c = (int)(s - i * ch);
        const double x = y[c * stride + i];
        unsigned char* p = out + s * B;
        if constexpr (FMT == 0) {
            const unsigned long long bits = __double_as_longlong(x);
#pragma unroll
            for (int k = 0; k < 8; k++) p[k] = (unsigned char)(bits >> (8 * k));
        } else if constexpr (FMT == 1) {
            const unsigned int bits = __float_as_uint(__double2float_rn(x));
#pragma unroll
            for (int k = 0; k < 4; k++) p[k] = (unsigned char)(bits >> (8 * k));
        } else {
            double v = __dmul_rn(x, sc);
            if (D) v = __dadd_rn(v, D[s]);
            v = rint(v);
            if (v > sc - 1) {
                v = sc - 1;
                clip++;
            } else if (v < -sc) {
                v = -sc;
                clip++;
            }
            const long long iv = isnan(v) ? 0 : (long long)v;  // NaN is written as zero
#pragma unroll
            for (int k = 0; k < B; k++) p[k] = (unsigned char)((iv >> (8 * k)) & 255);
        }
    }
    if (FMT >= 2) {
        for (int o = 16; o > 0; o >>= 1) clip += __shfl_down_sync(0xffffffffu, clip, o);
        if ((threadIdx.x & 31) == 0 && clip) atomicAdd(clipped, clip);
    }
}

int format_bytes(int format) { return format == 0 ? 8 : format == 1 ? 4 : format == 2 ? 4 : format == 3 ? 3 : 2; }

// Packs planar device samples into device WAV data; D: device dither values (nullptr: none).
int enqueue_pack(const double* y, int ch, long long frames, long long stride, int format, const double* D,
                 unsigned char* out, unsigned long long* clipped, cudaStream_t st) {
    const long long n = frames * ch;
    if (n == 0) return KBSRC_GPU_OK;
    const unsigned g = grid_for(n, 256);
    switch (format) {
        case 0: k_pack<0><<<g, 256, 0, st>>>(y, ch, frames, stride, nullptr, out, clipped); break;
        case 1: k_pack<1><<<g, 256, 0, st>>>(y, ch, frames, stride, nullptr, out, clipped); break;
        case 2: k_pack<2><<<g, 256, 0, st>>>(y, ch, frames, stride, D, out, clipped); break;
        case 3: k_pack<3><<<g, 256, 0, st>>>(y, ch, frames, stride, D, out, clipped); break;
        case 4: k_pack<4><<<g, 256, 0, st>>>(y, ch, frames, stride, D, out, clipped); break;
        default: return fail(KBSRC_GPU_E_ARG, "unknown sample format");
    }
    KB_CUDA(cudaGetLastError());
    return KBSRC_GPU_OK;
}

}  // namespace

// Chunks of blocks for run_host's copy pipeline: 32 (measured on C2: 88% of the copy floor against 82% with 16
// and 76% with 48), at most one per block (KBSRC_GPU_CHUNKS overrides).
long long nout_chunks(const kbsrc_gpu_engine* e, long long nblk) {
    const long long want = env_int("KBSRC_GPU_CHUNKS", 32);
    return std::max(1LL, std::min(want, nblk));
}

// ---- batches: many conversions, grouped by plan -------------------------------------------------------------
namespace {

// Zeroes every conversion's output (the reference's value-initialised output), reading the pointers from the
// item table so that the recorded run stays valid for new buffers.
__global__ void k_zero_items(const Item* __restrict__ items, int count) {
    const Item it = items[blockIdx.y];
    const long long n = it.nout * it.ch;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        it.out[i] = 0.0;
}

bool same_plan(const kbsrc_gpu_desc& a, const kbsrc_gpu_desc& b) {
    if (a.precision != b.precision || a.P != b.P || a.Q != b.Q || a.nb != b.nb || a.marg != b.marg || a.up != b.up ||
        a.Jg != b.Jg || a.H_len != b.H_len)
        return false;
    return a.H == b.H || std::memcmp(a.H, b.H, (size_t)a.H_len * 16) == 0;
}

// Whether a group can run through the queue kernels: double-double or float64, both transforms four-step and
// 7-smooth (no direct or Bluestein transform).
bool queue_eligible(const BatchGroup& g) {
    if (g.split || g.tab == kTabX80) return false;
    return g.fw.host.four && !g.fw.m && g.iv.host.four && !g.iv.m;
}

template <class K>
int queue_ctas(K kernel, int threads, size_t smem, int sms, int& ctas) {
    int per = 0;
    KB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
    ctas = std::max(1, per) * sms;
    return KBSRC_GPU_OK;
}

// Builds the batch queue of the eligible groups of the first eligible group's arithmetic (KBSRC_GPU_QUEUE=0 keeps
// every group on its own launches): the group table, waves of their tasks (largest transform first) within the slot
// buffers, each pass's units. The other groups run their own launches after the queue.
int build_queue(kbsrc_gpu_batch& b) {
    if (b.groups.empty() || !env_int("KBSRC_GPU_QUEUE", 1)) return KBSRC_GPU_OK;
    int first = -1;
    for (size_t i = 0; i < b.groups.size() && first < 0; i++)
        if (queue_eligible(*b.groups[i])) first = (int)i;
    if (first < 0) return KBSRC_GPU_OK;
    const bool exact = b.groups[first]->exact;
    const size_t es = b.groups[first]->esize();
    // Every group shares each pass's launch shape, so a group's sequences per unit are cut (launch shapes only: the
    // bytes do not change) until its shared memory leaves room for as many CTAs per SM as the kernel is compiled
    // for; the largest of those then sizes the launch. A group that fits no such shape runs on its own launches.
    int per_sm = 0;
    KB_CUDA(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, b.device));
    const int colT = exact ? KB_MAXT_DD_COL : KB_MAXT_F64, rowT = exact ? KB_MAXT_DD : KB_MAXT_F64;
    const int colB = exact ? KB_MINB_DD_COL : KB_MINB_F64, rowB = exact ? KB_MINB_DD : KB_MINB_F64;
    const int pass[4] = {0, 1, 4, 5}, maxT[4] = {colT, rowT, colT, rowT};
    size_t limit[4];
    for (int k = 0; k < 4; k++) limit[k] = (size_t)per_sm / (k & 1 ? rowB : colB) - 2048;
    auto fit = [&](const SubPlan& sp, int F, int kk, Shape& out) {  // the largest F' <= F within limit[kk]
        const size_t tw = es == 32 ? (size_t)sp.twn * es : 0;
        for (int f = F; f >= 1; f--) {
            const size_t sm = 2 * (size_t)sp.n * f * es + tw;
            if (sm > limit[kk]) continue;
            int t = ((max_bfly(sp) * f + 31) / 32) * 32;
            out = Shape{f, std::max(64, std::min(maxT[kk], t)), sm};
            return true;
        }
        return false;
    };
    // A group with enough units to fill the GPU on every pass runs on its own launches, whose shapes are its own
    // (a queue launch shares one thread count and one shared-memory size among its groups: C4's 54 groups, all
    // large, took 500 ms per step through the queue against 384 ms on their own launches); the queue gathers the
    // groups whose own launches would leave SMs idle. KBSRC_GPU_QUEUE_FILL sets the threshold in units per pass.
    int sms_q = 0;
    KB_CUDA(cudaDeviceGetAttribute(&sms_q, cudaDevAttrMultiProcessorCount, b.device));
    const long long fill = env_int("KBSRC_GPU_QUEUE_FILL", 8 * sms_q);
    auto fills = [&](const BatchGroup& g) {
        const long long col = std::min((g.fw.host.N2 + g.fw.col.F - 1) / g.fw.col.F,
                                       (g.iv.host.N2 + g.iv.col.F - 1) / g.iv.col.F);
        const long long row = std::min((g.fw.host.N1 + g.fw.row.F - 1) / g.fw.row.F,
                                       (g.iv.host.N1 + g.iv.row.F - 1) / g.iv.row.F);
        return g.tasks * std::min(col, row) >= fill;
    };
    std::vector<int> qi;  // queued groups in the batch's group order
    std::vector<std::array<Shape, 4>> qs;
    for (size_t i = 0; i < b.groups.size(); i++) {
        const BatchGroup& g = *b.groups[i];
        if (!queue_eligible(g) || g.exact != exact || fills(g)) continue;
        const SubPlan* sp[4] = {&g.fw.host.s1, &g.fw.host.s2, &g.iv.host.s1, &g.iv.host.s2};
        const Shape sh[4] = {g.fw.col, g.fw.row, g.iv.col, g.iv.row};
        std::array<Shape, 4> q;
        bool ok = true;
        for (int k = 0; k < 4 && ok; k++) ok = fit(*sp[k], sh[k].F, k, q[k]);
        if (!ok) continue;
        qi.push_back((int)i);
        qs.push_back(q);
    }
    if (qi.empty()) return KBSRC_GPU_OK;
    std::vector<QueueGroup> qg(qi.size());
    int T[6] = {}, sms = 0;
    size_t S[6] = {};
    for (size_t i = 0; i < qi.size(); i++) {
        const BatchGroup& g = *b.groups[qi[i]];
        QueueGroup& q = qg[i];
        q.fs1 = g.fw.host.s1; q.fs2 = g.fw.host.s2; q.is1 = g.iv.host.s1; q.is2 = g.iv.host.s2;
        q.fN1 = g.fw.host.N1; q.fN2 = g.fw.host.N2; q.iN1 = g.iv.host.N1; q.iN2 = g.iv.host.N2;
        q.fcF = qs[i][0].F; q.frF = qs[i][1].F; q.icF = qs[i][2].F; q.irF = qs[i][3].F;
        q.ftw_stage = g.fw.tw_stage.p; q.ftw4 = g.fw.tw4.p; q.itw_stage = g.iv.tw_stage.p; q.itw4 = g.iv.tw4.p;
        q.w_fw = g.w_fw.p; q.w_iv = g.w_iv.p; q.H = g.H.p;
        q.h = g.hf; q.hi = g.hi; q.Nb = g.Nb; q.Mb = g.Mb; q.up = g.d.up; q.Jg = g.d.Jg;
        q.hopQ = (long long)g.hop * g.d.Q; q.hopP = (long long)g.hop * g.d.P; q.margP = (long long)g.d.marg * g.d.P;
        for (int k = 0; k < 4; k++) {
            T[pass[k]] = std::max(T[pass[k]], qs[i][k].T);
            S[pass[k]] = std::max(S[pass[k]], qs[i][k].smem);
        }
    }
    T[2] = T[3] = kQueueBinThreads;
    int rc;
    if ((rc = b.q_groups.alloc(qg.size() * sizeof(QueueGroup))) != KBSRC_GPU_OK) return rc;
    KB_CUDA(cudaMemcpy(b.q_groups.p, qg.data(), qg.size() * sizeof(QueueGroup), cudaMemcpyHostToDevice));
    // every task, largest forward transform first (ties: group, then the group's own block-major order)
    struct Pending {
        int group;
        TaskRef ref;
    };
    std::vector<Pending> all;
    for (size_t k = 0; k < qi.size(); k++)
        for (int i : b.groups[qi[k]]->members)
            for (long long blk = 0; blk < b.descs[i].nblk; blk++)
                for (int c = 0; c < b.descs[i].channels; c++) all.push_back(Pending{(int)k, TaskRef{i, c, blk}});
    std::stable_sort(all.begin(), all.end(), [&](const Pending& x, const Pending& y) {
        return b.groups[qi[x.group]]->hf > b.groups[qi[y.group]]->hf;
    });
    const long long budget = (long long)b.bufA.bytes;
    size_t at = 0;
    while (at < all.size()) {
        std::vector<QueueTask> tasks;
        long long used = 0;
        while (at < all.size()) {
            const BatchGroup& g = *b.groups[qi[all[at].group]];
            const long long bytes = g.stride * (long long)es;
            if (!tasks.empty() && used + bytes > budget) break;
            tasks.push_back(QueueTask{all[at].ref, all[at].group, used / (long long)es});
            used += bytes;
            at++;
        }
        QueueWave w;
        w.ntasks = (long long)tasks.size();
        std::vector<QueueUnit> units[6];
        for (int ti = 0; ti < (int)tasks.size(); ti++) {
            const QueueGroup& q = qg[tasks[ti].group];
            const int split_last_bin = exact ? q.h / 2 : q.h - 1, merge_last_bin = exact ? q.hi / 2 : q.hi - 1;
            const int n[6] = {(q.fN2 + q.fcF - 1) / q.fcF, (q.fN1 + q.frF - 1) / q.frF,
                              split_last_bin / kQueueBins + 1, merge_last_bin / kQueueBins + 1,
                              (q.iN2 + q.icF - 1) / q.icF, (q.iN1 + q.irF - 1) / q.irF};
            for (int p = 0; p < 6; p++)
                for (int u = 0; u < n[p]; u++) units[p].push_back(QueueUnit{ti, u});
        }
        if ((rc = w.tasks.alloc(tasks.size() * sizeof(QueueTask))) != KBSRC_GPU_OK) return rc;
        KB_CUDA(cudaMemcpy(w.tasks.p, tasks.data(), tasks.size() * sizeof(QueueTask), cudaMemcpyHostToDevice));
        for (int p = 0; p < 6; p++) {
            w.nunits[p] = (int)units[p].size();
            if ((rc = w.units[p].alloc(units[p].size() * sizeof(QueueUnit))) != KBSRC_GPU_OK) return rc;
            KB_CUDA(cudaMemcpy(w.units[p].p, units[p].data(), units[p].size() * sizeof(QueueUnit),
                               cudaMemcpyHostToDevice));
        }
        b.q_waves.push_back(std::move(w));
    }
    if ((rc = b.q_counters.alloc(b.q_waves.size() * 6 * sizeof(int))) != KBSRC_GPU_OK) return rc;
    KB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b.device));
    for (int p = 0; p < 6; p++) {
        b.q_threads[p] = T[p];
        b.q_smem[p] = S[p];
    }
    if (exact) {
        if ((rc = queue_ctas(k_column_q<ArDDShort, kSrcSignal, true>, T[0], S[0], sms, b.q_ctas[0])) ||
            (rc = queue_ctas(k_row_q<ArDDShort, kDstComplex, true>, T[1], S[1], sms, b.q_ctas[1])) ||
            (rc = queue_ctas(k_bins_q<ArDDAccurate, true>, T[2], 0, sms, b.q_ctas[2])) ||
            (rc = queue_ctas(k_bins_q<ArDDAccurate, false>, T[3], 0, sms, b.q_ctas[3])) ||
            (rc = queue_ctas(k_column_q<ArDDShort, kSrcComplex, false>, T[4], S[4], sms, b.q_ctas[4])) ||
            (rc = queue_ctas(k_row_q<ArDDShort, kDstOutput, false>, T[5], S[5], sms, b.q_ctas[5])))
            return rc;
    } else {
        if ((rc = queue_ctas(k_column_q<ArF64, kSrcSignal, true>, T[0], S[0], sms, b.q_ctas[0])) ||
            (rc = queue_ctas(k_row_q<ArF64, kDstComplex, true>, T[1], S[1], sms, b.q_ctas[1])) ||
            (rc = queue_ctas(k_bins_q<ArF64, true>, T[2], 0, sms, b.q_ctas[2])) ||
            (rc = queue_ctas(k_bins_q<ArF64, false>, T[3], 0, sms, b.q_ctas[3])) ||
            (rc = queue_ctas(k_column_q<ArF64, kSrcComplex, false>, T[4], S[4], sms, b.q_ctas[4])) ||
            (rc = queue_ctas(k_row_q<ArF64, kDstOutput, false>, T[5], S[5], sms, b.q_ctas[5])))
            return rc;
    }
    for (int i : qi) b.groups[i]->queued = true;
    b.q_exact = exact;
    b.queued = true;
    return KBSRC_GPU_OK;
}

// One wave's six queue launches; every unit counter of the run was zeroed before the first.
template <class ArL, class ArS>
int enqueue_queue_wave(const kbsrc_gpu_batch& b, size_t wi, cudaStream_t st, Trail& tr) {
    const QueueWave& w = b.q_waves[wi];
    int* counters = static_cast<int*>(b.q_counters.p) + 6 * wi;
    QueueParams<typename ArL::W> q{};
    q.groups = static_cast<const QueueGroup*>(b.q_groups.p);
    q.tasks = static_cast<const QueueTask*>(w.tasks.p);
    q.items = static_cast<const Item*>(b.items.p);
    q.A = b.bufA.p;
    q.B = b.bufB.p;
    q.odd = odd_table<typename ArL::W>();
    auto set = [&](int p) {
        q.units = static_cast<const QueueUnit*>(w.units[p].p);
        q.nunits = w.nunits[p];
        q.counter = counters + p;
    };
    auto launch = [&](auto kernel, int p) -> int {
        set(p);
        const cudaError_t before = cudaPeekAtLastError();
        if (before != cudaSuccess)
            return fail(KBSRC_GPU_E_CUDA, std::string("before the batch queue: ") + cudaGetErrorString(before));
        kernel<<<b.q_ctas[p], b.q_threads[p], b.q_smem[p], st>>>(q);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            return fail(KBSRC_GPU_E_CUDA, "batch queue pass " + std::to_string(p) + " (" + std::to_string(b.q_ctas[p]) +
                                              " CTAs of " + std::to_string(b.q_threads[p]) + " threads, " +
                                              std::to_string(b.q_smem[p]) + " bytes): " + cudaGetErrorString(e));
        return tr.mark(st, p);
    };
    int rc;
    if ((rc = launch(k_column_q<ArL, kSrcSignal, true>, 0)) || (rc = launch(k_row_q<ArL, kDstComplex, true>, 1)) ||
        (rc = launch(k_bins_q<ArS, true>, 2)) || (rc = launch(k_bins_q<ArS, false>, 3)) ||
        (rc = launch(k_column_q<ArL, kSrcComplex, false>, 4)) || (rc = launch(k_row_q<ArL, kDstOutput, false>, 5)))
        return rc;
    return KBSRC_GPU_OK;
}

int batch_create_impl(const kbsrc_gpu_desc* descs, int count, kbsrc_gpu_batch** out) {
    if (!descs || count < 1) return fail(KBSRC_GPU_E_ARG, "empty batch");
    int rc;
    for (int i = 0; i < count; i++) {
        if ((rc = check_desc(descs + i)) != KBSRC_GPU_OK) return fail(rc, "conversion " + std::to_string(i) + ": " + g_error);
        if (descs[i].shard.blk1 > 0) return fail(KBSRC_GPU_E_ARG, "batches run whole conversions (no shards)");
    }
    if ((rc = require_device()) != KBSRC_GPU_OK) return rc;
    if ((rc = allow_large_smem()) != KBSRC_GPU_OK) return rc;
    auto bp = std::make_unique<kbsrc_gpu_batch>();
    kbsrc_gpu_batch& b = *bp;
    KB_CUDA(cudaGetDevice(&b.device));
    KB_CUDA(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
    KB_CUDA(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
    b.descs.assign(descs, descs + count);
    b.group_of.assign(count, -1);
    std::vector<int> rep;  // representative conversion of each group
    for (int i = 0; i < count; i++) {
        if (descs[i].nblk == 0 || descs[i].nout == 0) continue;
        int g = -1;
        for (size_t k = 0; k < rep.size() && g < 0; k++)
            if (same_plan(descs[rep[k]], descs[i])) g = (int)k;
        if (g < 0) {
            g = (int)rep.size();
            rep.push_back(i);
            b.groups.push_back(std::make_unique<BatchGroup>());
            if ((rc = make_core(descs + i, *b.groups.back(), b.stream)) != KBSRC_GPU_OK) return rc;
        }
        b.group_of[i] = g;
        b.groups[g]->members.push_back(i);
    }
    // task tables (block-major per conversion) and slot buffers shared by the groups
    long long bytes = 0, need = 0;
    const long long budget = (long long)env_int("KBSRC_GPU_WAVE_MB", 4096) << 20;
    for (auto& gp : b.groups) {
        BatchGroup& g = *gp;
        std::vector<TaskRef> refs;
        for (int i : g.members)
            for (long long blk = 0; blk < descs[i].nblk; blk++)
                for (int c = 0; c < descs[i].channels; c++) refs.push_back(TaskRef{i, c, blk});
        g.tasks = (long long)refs.size();
        if ((rc = g.refs.alloc(refs.size() * sizeof(TaskRef))) != KBSRC_GPU_OK) return rc;
        KB_CUDA(cudaMemcpy(g.refs.p, refs.data(), refs.size() * sizeof(TaskRef), cudaMemcpyHostToDevice));
        g.stride = g.slot();
        const long long per = g.stride * (long long)g.esize();
        need = std::max(need, per);
        bytes = std::max(bytes, std::min(g.tasks * per, budget));
    }
    bytes = std::max(bytes, need);
    for (auto& gp : b.groups)
        gp->wave = std::max(1LL, std::min({gp->tasks, bytes / (gp->stride * (long long)gp->esize()), 65535LL}));
    if (!b.groups.empty()) {
        if ((rc = b.bufA.alloc((size_t)bytes)) != KBSRC_GPU_OK) return rc;
        if ((rc = b.bufB.alloc((size_t)bytes)) != KBSRC_GPU_OK) return rc;
    }
    if ((rc = b.items.alloc((size_t)count * sizeof(Item))) != KBSRC_GPU_OK) return rc;
    KB_CUDA(cudaMallocHost(&b.items_host, (size_t)count * sizeof(Item)));
    if ((rc = build_queue(b)) != KBSRC_GPU_OK) return rc;
    *out = bp.release();
    return KBSRC_GPU_OK;
}

// The whole batch on one stream: item table upload, output zeroing, every group's block loop.
int batch_enqueue(kbsrc_gpu_batch& b, cudaStream_t st, Trail& tr) {
    const int count = (int)b.descs.size();
    KB_CUDA(cudaMemcpyAsync(b.items.p, b.items_host, (size_t)count * sizeof(Item), cudaMemcpyHostToDevice, st));
    long long most = 1;
    for (const auto& d : b.descs) most = std::max(most, d.nout * d.channels);
    k_zero_items<<<dim3(grid_for(most, 256), count), 256, 0, st>>>(static_cast<const Item*>(b.items.p), count);
    int rc;
    if ((rc = tr.mark(st, -2)) != KBSRC_GPU_OK) return rc;
    if (b.queued) {
        KB_CUDA(cudaMemsetAsync(b.q_counters.p, 0, b.q_counters.bytes, st));
        for (size_t wi = 0; wi < b.q_waves.size(); wi++) {
            rc = b.q_exact ? enqueue_queue_wave<ArDDShort, ArDDAccurate>(b, wi, st, tr)
                           : enqueue_queue_wave<ArF64, ArF64>(b, wi, st, tr);
            if (rc) return rc;
        }
    }
    for (auto& gp : b.groups) {
        const BatchGroup& g = *gp;
        if (g.queued) continue;
        Work w{};
        w.items = static_cast<const Item*>(b.items.p);
        w.refs = static_cast<const TaskRef*>(g.refs.p);
        w.hopQ = (long long)g.hop * g.d.Q;
        w.hopP = (long long)g.hop * g.d.P;
        w.margP = (long long)g.d.marg * g.d.P;
        if ((rc = enqueue_any(g, w, 0, g.tasks, b.bufA.p, b.bufB.p, g.stride, g.wave, st, tr)) != KBSRC_GPU_OK)
            return rc;
    }
    KB_CUDA(cudaGetLastError());
    return KBSRC_GPU_OK;
}

int batch_run_device_impl(kbsrc_gpu_batch& b, const double* const* in, const double* const* head,
                          const double* const* tail, double* const* out, cudaStream_t st) {
    const int count = (int)b.descs.size();
    for (int i = 0; i < count; i++) {
        const kbsrc_gpu_desc& d = b.descs[i];
        if ((d.frames > 0 && !in[i]) || (d.nout > 0 && !out[i]) || (d.edge_len > 0 && (!head[i] || !tail[i])))
            return fail(KBSRC_GPU_E_ARG, "null buffer for conversion " + std::to_string(i));
    }
    KB_CUDA(cudaEventSynchronize(b.done));  // the previous run has read the item table
    for (int i = 0; i < count; i++) {
        const kbsrc_gpu_desc& d = b.descs[i];
        b.items_host[i] = Item{in[i], head ? head[i] : nullptr, tail ? tail[i] : nullptr, out[i], d.frames,
                               d.edge_len, d.lead, d.nout, d.o, d.channels, d.in_format, 0, 0, d.nout};
    }
    if (!b.graph) {
        // record the run once; it reads every pointer from the item table, so it replays for new buffers
        cudaGraph_t g = nullptr;
        KB_CUDA(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal));
        Trail tr;
        int rc = batch_enqueue(b, b.stream, tr);
        const cudaError_t ce = cudaStreamEndCapture(b.stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return fail(KBSRC_GPU_E_CUDA, std::string("stream capture: ") + cudaGetErrorString(ce));
        const cudaError_t ie = cudaGraphInstantiate(&b.graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            b.graph = nullptr;
            return fail(KBSRC_GPU_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        }
        b.launches = tr.launches;
    }
    KB_CUDA(cudaGraphLaunch(b.graph, st));
    KB_CUDA(cudaEventRecord(b.done, st));
    return KBSRC_GPU_OK;
}

}  // namespace

// ---- kernel spectrum for callers that cannot allocate device memory ----------------------------------------
//
// Some callers may not let a library allocate GPU memory. An application that reserves the device's memory up
// front for its own pool (a framework's caching allocator, an audio host that budgets the GPU at start-up) can
// have nothing left for cudaMalloc, and cudaFree waits for the whole device, stalling the caller's other streams.
// For them kbsrc_gpu_kernel_spectrum_static takes its taps and its output in device memory and keeps all of its
// scratch (the placed taps, two FFT work buffers, the twiddle tables and the root tables they are built from) in
// one file-scope device array below. The array is part of the library image: every GPU that loads the library
// holds it until the process exits. The tables are computed on the GPU as well, so the call builds nothing on
// the host and copies nothing from host memory: it only launches kernels on the caller's stream.

// Capacity of the shared scratch: transforms up to about 300,000 points (80 bytes per point), which covers the
// automatic plans of the common rates (for example 201,600 points for 96 kHz -> 44.1 kHz at --len 0.2).
constexpr size_t kSpectrumScratchBytes = (size_t)24 << 20;
static __device__ __align__(256) unsigned char g_spectrum_scratch[kSpectrumScratchBytes];

namespace {

// Roots of unity on the device, bit-identical to the host's tables: kbsrc::host::unit_root and RootTable
// (host/ddh.hpp), which build the reference's CisTable (src/dsp/fft.hpp:29-43) from dd Taylor series after an
// exact octant reduction. Each function below runs the host function's IEEE operations in the same order: the
// accurate dd add, the dd product with one fma, the dd-by-double product and the three-digit division.
constexpr double kPiHi = 3.141592653589793116e+00, kPiLo = 1.224646799147353207e-16;

__device__ __forceinline__ dd dvr_mul_f(dd a, double b) {  // dd * double
    const double p = __dmul_rn(a.hi, b);
    double e = __fma_rn(a.hi, b, -p);
    e = __dadd_rn(e, __dmul_rn(a.lo, b));
    return qts(p, e);
}

// cos and sin of x in [0, pi/4] by their Taylor series in dd
__device__ void dvr_sincos(dd x, dd& c, dd& s) {
    const dd x2 = mul_dd(x, x);
    dd ts = x, ss = x, tc{1.0, 0.0}, cc{1.0, 0.0};
    for (int k = 1; k < 40; k++) {
        tc = div_dd_f64(dd_neg(mul_dd(tc, x2)), (double)((2 * k - 1) * (2 * k)));
        cc = add_accurate(cc, tc);
        ts = div_dd_f64(dd_neg(mul_dd(ts, x2)), (double)((2 * k) * (2 * k + 1)));
        ss = add_accurate(ss, ts);
        if (fabs(ts.hi) < 1e-40 && fabs(tc.hi) < 1e-40) break;
    }
    c = cc;
    s = ss;
}

// e^{+2 pi i k / n} = c + i s
__device__ void dvr_unit_root(long long k, long long n, dd& c, dd& s) {
    k %= n;
    if (k < 0) k += n;
    const long long eighths = 8 * k, oct = eighths / n, rem = eighths - oct * n;
    const bool mirrored = oct & 1;
    long long quadrant = oct / 2;
    const dd phi = div_dd_f64(dvr_mul_f(dd{kPiHi / 4, kPiLo / 4}, (double)(mirrored ? n - rem : rem)), (double)n);
    dd cr, sr;
    dvr_sincos(phi, cr, sr);
    if (mirrored) {
        sr = dd_neg(sr);
        quadrant += 1;
    }
    switch (quadrant & 3) {
        case 0: c = cr; s = sr; break;
        case 1: c = dd_neg(sr); s = cr; break;
        case 2: c = dd_neg(cr); s = dd_neg(sr); break;
        default: c = sr; s = dd_neg(cr); break;
    }
}

// A root table of n on the device: `coarse` entries w^(j step) followed by `step` entries w^l, as cx<dd> (c, s).
struct DevRoots {
    const cx<dd>* t;
    long long n, step, coarse;
};
DevRoots dev_roots_shape(long long n) {
    DevRoots r{};
    r.n = n;
    r.step = (long long)std::ceil(std::sqrt((double)n));  // as RootTable's constructor
    r.coarse = n / r.step + 1;
    return r;
}

__global__ void k_roots_build(DevRoots r, cx<dd>* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < r.coarse + r.step;
         i += (long long)gridDim.x * blockDim.x) {
        dd c, s;
        dvr_unit_root(i < r.coarse ? i * r.step : i - r.coarse, r.n, c, s);
        out[i] = cx<dd>{c, s};
    }
}

// e^{2 pi i k/n} from the table: the dd product of a coarse and a fine entry (RootTable::get)
__device__ cx<dd> dvr_get(const DevRoots& r, long long k) {
    k %= r.n;
    if (k < 0) k += r.n;
    const long long j = k / r.step, l = k % r.step;
    const cx<dd> a = r.t[j], b = r.t[r.coarse + l];
    if (l == 0) return a;
    if (j == 0) return b;
    return cx<dd>{add_accurate(mul_dd(a.re, b.re), dd_neg(mul_dd(a.im, b.im))),
                  add_accurate(mul_dd(a.re, b.im), mul_dd(a.im, b.re))};
}

// out[k] = w^(-k) for k < count (the real-FFT split roots), or out[k1 * N2 + n2] = w^(-k1 n2) (four-step twiddles;
// N2 > 0)
__global__ void k_roots_table(DevRoots r, long long count, int N2, cx<dd>* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = dvr_get(r, N2 ? -(i / N2) * (i % N2) : -i);
}

// The stage twiddles of a sub-plan, w^(-s p u) at sp.st[g].tw + p (r - 1) + u - 1 (build_sub's layout); `out` is
// entry sp.tw0
__global__ void k_roots_stages(DevRoots r, SubPlan sp, cx<dd>* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < sp.twn; i += gridDim.x * blockDim.x) {
        const int e = sp.tw0 + i;
        int g = 0;
        while (g + 1 < sp.nst && e >= sp.st[g + 1].tw) g++;
        const Stage& st = sp.st[g];
        if (sp.nst == 0 || e - st.tw >= st.m * (st.r - 1)) {  // the placeholder entry of a plan without twiddles
            out[i] = cx<dd>{dd{0.0, 0.0}, dd{0.0, 0.0}};
            continue;
        }
        const int p = (e - st.tw) / (st.r - 1), u = (e - st.tw) % (st.r - 1) + 1;
        out[i] = dvr_get(r, -(long long)st.s * p * u);
    }
}

// r[i] = h[i] for i <= L, h[n - i] for i >= n - L, else 0 (the circular placement of design.cpp:42-43);
// every entry is written, so nothing left by an earlier call survives.
__global__ void k_place_taps(const double* __restrict__ taps, int L, int n, double* __restrict__ r) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int m = i <= L ? i : (i >= n - L ? n - i : -1);
        r[2 * i] = m >= 0 ? taps[2 * m] : 0.0;
        r[2 * i + 1] = m >= 0 ? taps[2 * m + 1] : 0.0;
    }
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

bool host_pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// memcpy split over up to 8 threads (pieces of at least 4 MB)
void par_memcpy(void* dst, const void* src, size_t n) {
    const int nt = (int)std::max<size_t>(1, std::min<size_t>(8, n >> 22));
    if (nt == 1) {
        std::memcpy(dst, src, n);
        return;
    }
    std::vector<std::thread> th;
    const size_t piece = (n + nt - 1) / nt;
    for (int t = 0; t < nt; t++) {
        const size_t off = (size_t)t * piece;
        if (off >= n) break;
        th.emplace_back([=] {
            std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, std::min(piece, n - off));
        });
    }
    for (auto& x : th) x.join();
}

int stager_ready(Stager& sg) {
    for (int i = 0; i < 2; i++) {
        if (!sg.pin[i]) KB_CUDA(cudaMallocHost(&sg.pin[i], Stager::kChunk));
        if (!sg.ev[i]) KB_CUDA(cudaEventCreateWithFlags(&sg.ev[i], cudaEventDisableTiming));
    }
    return KBSRC_GPU_OK;
}

// Host -> device on `st`; returns once the last chunk is in flight (its bounce buffer is not reused before
// its DMA completes).
int copy_h2d(Stager& sg, void* dst, const void* src, size_t n, cudaStream_t st) {
    if (!n) return KBSRC_GPU_OK;
    if (host_pinned(src)) {
        KB_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st));
        return KBSRC_GPU_OK;
    }
    int rc;
    if ((rc = stager_ready(sg)) != KBSRC_GPU_OK) return rc;
    for (size_t off = 0, k = 0; off < n; off += Stager::kChunk, k++) {
        const int b = (int)(k & 1);
        const size_t m = std::min(Stager::kChunk, n - off);
        KB_CUDA(cudaEventSynchronize(sg.ev[b]));
        par_memcpy(sg.pin[b], static_cast<const char*>(src) + off, m);
        KB_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + off, sg.pin[b], m, cudaMemcpyHostToDevice, st));
        KB_CUDA(cudaEventRecord(sg.ev[b], st));
    }
    return KBSRC_GPU_OK;
}

// Device -> host after the work already on `st`; synchronous (returns with the data in dst).
int copy_d2h(Stager& sg, void* dst, const void* src, size_t n, cudaStream_t st) {
    if (!n) return KBSRC_GPU_OK;
    if (host_pinned(dst)) {
        KB_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaStreamSynchronize(st));
        return KBSRC_GPU_OK;
    }
    int rc;
    if ((rc = stager_ready(sg)) != KBSRC_GPU_OK) return rc;
    const size_t chunks = (n + Stager::kChunk - 1) / Stager::kChunk;
    auto issue = [&](size_t k) -> int {
        const int b = (int)(k & 1);
        const size_t off = k * Stager::kChunk, m = std::min(Stager::kChunk, n - off);
        KB_CUDA(cudaEventSynchronize(sg.ev[b]));
        KB_CUDA(cudaMemcpyAsync(sg.pin[b], static_cast<const char*>(src) + off, m, cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaEventRecord(sg.ev[b], st));
        return KBSRC_GPU_OK;
    };
    if ((rc = issue(0)) != KBSRC_GPU_OK) return rc;
    for (size_t k = 0; k < chunks; k++) {
        if (k + 1 < chunks && (rc = issue(k + 1)) != KBSRC_GPU_OK) return rc;
        const int b = (int)(k & 1);
        const size_t off = k * Stager::kChunk, m = std::min(Stager::kChunk, n - off);
        KB_CUDA(cudaEventSynchronize(sg.ev[b]));
        par_memcpy(static_cast<char*>(dst) + off, sg.pin[b], m);
    }
    return KBSRC_GPU_OK;
}

}  // namespace

extern "C" {

int kbsrc_gpu_init(void) {
    try {
        int rc;
        const char* tr = std::getenv("KBSRC_TRACE");
        const bool trace = tr && *tr && *tr != '0';
        const auto t0 = std::chrono::steady_clock::now();
        auto since = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
        if ((rc = require_device()) != KBSRC_GPU_OK) return rc;
        const double t_dev = since();
        KB_CUDA(cudaFree(nullptr));  // creates the context
        const double t_ctx = since();
        rc = allow_large_smem();
        if (trace)
            std::fprintf(stderr, "kbsrc trace: GPU start: device %.3fs  context %.3fs  kernel attributes %.3fs\n", t_dev,
                         t_ctx - t_dev, since() - t_ctx);
        return rc;
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_use_device(int device) {
    int rc = require_device();
    if (rc) return rc;
    int n = 0;
    KB_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n)
        return fail(KBSRC_GPU_E_ARG, "no CUDA device " + std::to_string(device) + " (" + std::to_string(n) + " present)");
    KB_CUDA(cudaSetDevice(device));
    return KBSRC_GPU_OK;
}

int kbsrc_gpu_shard_plan(const kbsrc_gpu_desc* d, int count, kbsrc_gpu_shard* shards) {
    if (!d || !shards || count < 1) return fail(KBSRC_GPU_E_ARG, "bad shard plan arguments");
    kbsrc_gpu_desc whole = *d;
    whole.shard = kbsrc_gpu_shard{};
    int rc = check_desc(&whole);
    if (rc) return rc;
    if (count > whole.nblk) return fail(KBSRC_GPU_E_ARG, "more shares than blocks");
    long long next_out = 0;
    for (int k = 0; k < count; k++) {
        const long long b0 = whole.nblk * k / count, b1 = whole.nblk * (k + 1) / count;
        kbsrc_gpu_shard& s = shards[k];
        shard_span(whole, b0, b1, s);
        // output ranges partition [0, nout): each share starts where the previous one ended, the last runs to nout
        const long long end = k == count - 1 ? whole.nout : s.out0 + s.nout;
        s.out0 = next_out;
        s.nout = std::max(0LL, end - next_out);
        next_out = s.out0 + s.nout;
    }
    return KBSRC_GPU_OK;
}

int kbsrc_gpu_engine_create(const kbsrc_gpu_desc* desc, kbsrc_gpu_engine** out) {
    if (!out) return fail(KBSRC_GPU_E_ARG, "null output pointer");
    *out = nullptr;
    try {
        return create_impl(desc, out);
    } catch (const std::bad_alloc&) {
        return fail(KBSRC_GPU_E_NOMEM, "host allocation failed");
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_ARG, x.what());
    }
}

int kbsrc_gpu_engine_run_device(kbsrc_gpu_engine* e, const double* d_in, const double* d_head, const double* d_tail,
                                double* d_out, void* stream) {
    if (!e) return fail(KBSRC_GPU_E_ARG, "null engine");
    if (!d_out && e->d.nout > 0) return fail(KBSRC_GPU_E_ARG, "null output");
    try {
        return run_device_impl(e, d_in, d_head, d_tail, d_out, stream ? (cudaStream_t)stream : e->stream);
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_engine_run_device_timed(kbsrc_gpu_engine* e, const double* d_in, const double* d_head,
                                      const double* d_tail, double* d_out, void* stream, float* pass_ms,
                                      int* pass_launches) {
    if (!e || !pass_ms) return fail(KBSRC_GPU_E_ARG, "null engine or timing array");
    if (!d_out && e->d.nout > 0) return fail(KBSRC_GPU_E_ARG, "null output");
    try {
        cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;
        std::vector<int> kinds;
        Trail tr{&e->events, &kinds, 0};
        int rc = run_device_impl(e, d_in, d_head, d_tail, d_out, st, &tr);
        if (rc) return rc;
        for (int k = 0; k < kPassKinds; k++) {
            pass_ms[k] = 0;
            if (pass_launches) pass_launches[k] = 0;
        }
        if (tr.n > 0) KB_CUDA(cudaEventSynchronize(e->events[tr.n - 1]));
        if ((rc = check_tc(*e)) != KBSRC_GPU_OK) return rc;
        for (size_t i = 1; i < tr.n; i++) {
            float ms = 0;
            KB_CUDA(cudaEventElapsedTime(&ms, e->events[i - 1], e->events[i]));
            const int k = kinds[i];
            if (k >= 0 && k < kPassKinds) {
                pass_ms[k] += ms;
                if (pass_launches) pass_launches[k] += 1;
            }
        }
        return KBSRC_GPU_OK;
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_engine_tune(kbsrc_gpu_engine* e, const double* d_in, const double* d_head, const double* d_tail,
                          double* d_out, void* stream, int* shapes) {
    if (!e || !shapes) return fail(KBSRC_GPU_E_ARG, "null engine or shape array");
    if (!d_out && e->d.nout > 0) return fail(KBSRC_GPU_E_ARG, "null output");
    try {
        for (int i = 0; i < 8; i++) shapes[i] = 0;
        cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;
        // the four shared-memory passes of the four-step transforms (kinds kFwdA, kFwdB, kInvA, kInvB)
        Shape* pass[4] = {nullptr, nullptr, nullptr, nullptr};
        const SubPlan* sub[4] = {};
        int count[4] = {};
        if (!e->split && !e->fw.m && e->fw.host.four) {
            pass[0] = &e->fw.col; sub[0] = &e->fw.host.s1; count[0] = e->fw.host.N2;
            pass[1] = &e->fw.row; sub[1] = &e->fw.host.s2; count[1] = e->fw.host.N1;
        }
        if (!e->split && !e->iv.m && e->iv.host.four) {
            pass[2] = &e->iv.col; sub[2] = &e->iv.host.s1; count[2] = e->iv.host.N2;
            pass[3] = &e->iv.row; sub[3] = &e->iv.host.s2; count[3] = e->iv.host.N1;
        }
        const size_t esize = e->esize();
        const int maxT[4] = {tab_max_threads(e->tab, true), tab_max_threads(e->tab, false),
                             tab_max_threads(e->tab, true), tab_max_threads(e->tab, false)};  // col, row, col, row
        int dev = 0, smem_max = 0;
        KB_CUDA(cudaGetDevice(&dev));
        KB_CUDA(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        std::vector<Shape> cand[4];
        for (int p = 0; p < 4; p++) {
            if (!pass[p]) continue;
            const size_t tw = esize == 32 ? (size_t)sub[p]->twn * esize : 0;
            for (int F : {1, 2, 3, 4, 5, 6, 8, 10, 12, 16})
                for (bool twg : {false, true}) {  // wide types: stage twiddles in shared memory, or read them
                    if (twg && esize != 32) continue;
                    const size_t sm = 2 * (size_t)sub[p]->n * F * esize + (twg ? 0 : tw);
                    if (F > count[p] || sm > (size_t)smem_max) continue;
                    for (int T = 64; T <= maxT[p]; T += 32) cand[p].push_back(Shape{F, T, sm, twg});
                }
            cand[p].push_back(*pass[p]);  // the default stays a candidate
        }
        size_t rounds = 0;
        for (int p = 0; p < 4; p++) rounds = std::max(rounds, cand[p].size());
        std::vector<float> best(4, 1e30f);
        Shape chosen[4];
        for (int p = 0; p < 4; p++)
            if (pass[p]) chosen[p] = *pass[p];
        std::vector<int> kinds;
        for (size_t r = 0; r <= rounds; r++) {  // round 0 warms up with the defaults
            for (int p = 0; p < 4; p++)
                if (pass[p] && r > 0) *pass[p] = cand[p][(r - 1) % cand[p].size()];
            float ms[kPassKinds] = {};
            for (int rep = 0; rep < 2; rep++) {  // the faster of two runs
                kinds.clear();
                Trail tr{&e->events, &kinds, 0};
                int rc = run_device_impl(e, d_in, d_head, d_tail, d_out, st, &tr);
                if (rc) return rc;
                if (tr.n > 0) KB_CUDA(cudaEventSynchronize(e->events[tr.n - 1]));
                float t[kPassKinds] = {};
                for (size_t i = 1; i < tr.n; i++) {
                    float x = 0;
                    KB_CUDA(cudaEventElapsedTime(&x, e->events[i - 1], e->events[i]));
                    if (kinds[i] >= 0 && kinds[i] < kPassKinds) t[kinds[i]] += x;
                }
                for (int k = 0; k < kPassKinds; k++) ms[k] = rep ? std::min(ms[k], t[k]) : t[k];
            }
            if (r == 0) continue;
            const int kind[4] = {kFwdA, kFwdB, kInvA, kInvB};
            for (int p = 0; p < 4; p++)
                if (pass[p] && ms[kind[p]] < best[p]) {
                    best[p] = ms[kind[p]];
                    chosen[p] = *pass[p];
                }
        }
        for (int p = 0; p < 4; p++)
            if (pass[p]) {
                *pass[p] = chosen[p];
                shapes[2 * p] = chosen[p].F;
                shapes[2 * p + 1] = chosen[p].T;
            }
        return KBSRC_GPU_OK;
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_engine_staging(const kbsrc_gpu_engine* e, int* staged) {
    if (!e || !staged) return fail(KBSRC_GPU_E_ARG, "null engine or output");
    const DevCfft* c[2] = {&e->fw, &e->iv};
    for (int i = 0; i < 2; i++) {
        const bool four = !e->split && !c[i]->m && c[i]->host.four, wide = e->esize() == 32;
        staged[2 * i] = four ? (wide && !c[i]->col.twg ? 1 : 0) : -1;
        staged[2 * i + 1] = four ? (wide && !c[i]->row.twg ? 1 : 0) : -1;
    }
    return KBSRC_GPU_OK;
}

int kbsrc_gpu_engine_run_host(kbsrc_gpu_engine* e, const double* in, const double* head, const double* tail,
                              double* out) {
    if (!e) return fail(KBSRC_GPU_E_ARG, "null engine");
    const kbsrc_gpu_desc& d = e->d;
    const kbsrc_gpu_shard sh = effective_shard(d);
    if ((sh.frames > 0 && !in) || (sh.nout > 0 && !out) || (d.edge_len > 0 && (!head || !tail)))
        return fail(KBSRC_GPU_E_ARG, "null buffer");
    try {
        int rc;
        const size_t nin = (size_t)sh.frames * d.channels, ne = (size_t)d.edge_len * d.channels,
                     no = (size_t)sh.nout * d.channels;
        if (!e->d_in.p && (rc = e->d_in.alloc(nin * in_bytes(d.in_format))) != KBSRC_GPU_OK) return rc;
        if (!e->d_head.p && (rc = e->d_head.alloc(ne * 8)) != KBSRC_GPU_OK) return rc;
        if (!e->d_tail.p && (rc = e->d_tail.alloc(ne * 8)) != KBSRC_GPU_OK) return rc;
        if (!e->d_out.p && (rc = e->d_out.alloc(no * 8)) != KBSRC_GPU_OK) return rc;
        if (!e->copy_in) {
            KB_CUDA(cudaStreamCreateWithFlags(&e->copy_in, cudaStreamNonBlocking));
            KB_CUDA(cudaStreamCreateWithFlags(&e->copy_out, cudaStreamNonBlocking));
            for (int k = 0; k < 2; k++) {
                KB_CUDA(cudaEventCreateWithFlags(&e->ev_in[k], cudaEventDisableTiming));
                KB_CUDA(cudaEventCreateWithFlags(&e->ev_done[k], cudaEventDisableTiming));
            }
        }
        // Pipeline by chunks of blocks: the input frames a chunk reads go up while the previous chunk computes,
        // and its output goes down while the next one computes. Tasks are block-major, so a chunk of blocks is a
        // contiguous task range; every frame is copied once, in order. A share's buffers start at its first held
        // frame (frame0) and output sample (out0).
        if (e->tasks == 0 || sh.nout == 0) return KBSRC_GPU_OK;
        cudaStream_t cs = e->stream, hs = e->copy_in, ds = e->copy_out;
        const double* dinp = (const double*)e->d_in.p;
        double* dout = (double*)e->d_out.p;
        KB_CUDA(cudaMemsetAsync(dout, 0, no * 8, cs));
        if (ne) {
            KB_CUDA(cudaMemcpyAsync(e->d_head.p, head, ne * 8, cudaMemcpyHostToDevice, hs));
            KB_CUDA(cudaMemcpyAsync(e->d_tail.p, tail, ne * 8, cudaMemcpyHostToDevice, hs));
        }
        const long long ch = d.channels, hopQ = (long long)e->hop * d.Q, hopP = (long long)e->hop * d.P;
        const long long nblk = sh.blk1 - sh.blk0, F0 = sh.frame0, F1 = sh.frame0 + sh.frames;
        const long long O0 = sh.out0, O1 = sh.out0 + sh.nout;
        const long long bps = in_bytes(d.in_format);
        const long long chunks = nout_chunks(e, nblk);
        const bool out_pinned = host_pinned(out);  // pageable output: one staged copy at the end
        const Work w = single_work(*e, dinp, (const double*)e->d_head.p, (const double*)e->d_tail.p, dout);
        long long copied = F0;  // frames already sent
        auto send = [&](long long upto) -> int {
            return copy_h2d(e->stager, static_cast<char*>(e->d_in.p) + (copied - F0) * ch * bps,
                            reinterpret_cast<const char*>(in) + (copied - F0) * ch * bps,
                            (size_t)((upto - copied) * ch * bps), hs);
        };
        Trail tr;
        for (long long k = 0; k < chunks; k++) {
            const long long b0 = sh.blk0 + nblk * k / chunks, b1 = sh.blk0 + nblk * (k + 1) / chunks;
            if (b0 == b1) continue;
            const long long f_hi = std::min(F1, std::max(F0, (b1 - 1) * hopQ + e->Nb - d.lead));
            if (f_hi > copied) {
                if ((rc = send(f_hi)) != KBSRC_GPU_OK) return rc;
                copied = f_hi;
            }
            KB_CUDA(cudaEventRecord(e->ev_in[k % 2], hs));
            KB_CUDA(cudaStreamWaitEvent(cs, e->ev_in[k % 2], 0));
            if ((rc = enqueue_any(*e, w, b0 * ch, b1 * ch, e->bufA.p, e->bufB.p, e->stride, e->wave, cs, tr)) !=
                KBSRC_GPU_OK)
                return rc;
            KB_CUDA(cudaEventRecord(e->ev_done[k % 2], cs));
            KB_CUDA(cudaStreamWaitEvent(ds, e->ev_done[k % 2], 0));
            const long long o0 = std::max(O0, b0 * hopP - d.o), o1 = k == chunks - 1 ? O1 : std::min(O1, b1 * hopP - d.o);
            if (o1 > o0 && out_pinned)
                KB_CUDA(cudaMemcpy2DAsync(out + (o0 - O0), (size_t)sh.nout * 8, dout + (o0 - O0), (size_t)sh.nout * 8,
                                          (size_t)(o1 - o0) * 8, (size_t)ch, cudaMemcpyDeviceToHost, ds));
        }
        if (copied < F1 && nin && (rc = send(F1)) != KBSRC_GPU_OK)  // frames no block reads (none in a valid plan)
            return rc;
        e->launches = tr.launches;
        KB_CUDA(cudaGetLastError());
        KB_CUDA(cudaStreamSynchronize(hs));
        KB_CUDA(cudaStreamSynchronize(cs));
        KB_CUDA(cudaStreamSynchronize(ds));
        if (!out_pinned && (rc = copy_d2h(e->stager, out, dout, no * 8, cs)) != KBSRC_GPU_OK) return rc;
        return check_tc(*e);
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_engine_run_host_packed(kbsrc_gpu_engine* e, const double* in, const double* head,
                                     const double* tail, int format, int dither, unsigned char* out_bytes,
                                     long long* clipped) {
    if (!e) return fail(KBSRC_GPU_E_ARG, "null engine");
    const kbsrc_gpu_desc& d = e->d;
    if (format < 0 || format > 4) return fail(KBSRC_GPU_E_ARG, "unknown sample format");
    if (d.shard.blk1 > 0)  // the dither stream runs from the file's first sample
        return fail(KBSRC_GPU_E_UNSUPPORTED, "packed output of a multi-GPU share");
    if ((d.frames > 0 && !in) || (d.nout > 0 && !out_bytes) || (d.edge_len > 0 && (!head || !tail)))
        return fail(KBSRC_GPU_E_ARG, "null buffer");
    try {
        int rc;
        const size_t nin = (size_t)d.frames * d.channels, ne = (size_t)d.edge_len * d.channels,
                     no = (size_t)d.nout * d.channels, nb = no * format_bytes(format);
        if (!e->d_in.p && (rc = e->d_in.alloc(nin * in_bytes(d.in_format))) != KBSRC_GPU_OK) return rc;
        if (!e->d_head.p && (rc = e->d_head.alloc(ne * 8)) != KBSRC_GPU_OK) return rc;
        if (!e->d_tail.p && (rc = e->d_tail.alloc(ne * 8)) != KBSRC_GPU_OK) return rc;
        if (!e->d_out.p && (rc = e->d_out.alloc(no * 8)) != KBSRC_GPU_OK) return rc;
        DevBuf bytes, dith, cnt, mtbuf;
        if ((rc = bytes.alloc(nb)) != KBSRC_GPU_OK || (rc = cnt.alloc(8)) != KBSRC_GPU_OK) return rc;
        const bool use_dither = dither && format >= 2 && no > 0;
        if (use_dither && (rc = dith.alloc(no * 8)) != KBSRC_GPU_OK) return rc;
        // the dither's jump tables (first use in the process) are built while the input is copied
        const int levels = use_dither ? dither_levels((long long)no) : 0;
        auto tables = std::async(std::launch::async, [levels] {
            if (levels) mt_tables(levels);
        });
        cudaStream_t st = e->stream;
        KB_CUDA(cudaMemsetAsync(cnt.p, 0, 8, st));
        if ((rc = copy_h2d(e->stager, e->d_in.p, in, nin * in_bytes(d.in_format), st)) != KBSRC_GPU_OK) return rc;
        if (ne) {
            KB_CUDA(cudaMemcpyAsync(e->d_head.p, head, ne * 8, cudaMemcpyHostToDevice, st));
            KB_CUDA(cudaMemcpyAsync(e->d_tail.p, tail, ne * 8, cudaMemcpyHostToDevice, st));
        }
        rc = run_device_impl(e, (const double*)e->d_in.p, (const double*)e->d_head.p, (const double*)e->d_tail.p,
                             (double*)e->d_out.p, st);
        if (rc) return rc;
        tables.get();
        cudaEvent_t dith_done = nullptr;
        struct EventGuard {
            cudaEvent_t& e;
            ~EventGuard() {
                if (e) cudaEventDestroy(e);
            }
        } guard_ev{dith_done};
        if (use_dither) {  // the generator on its own stream, beside the conversion
            if (!e->side) KB_CUDA(cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking));
            KB_CUDA(cudaEventCreateWithFlags(&dith_done, cudaEventDisableTiming));
            if ((rc = enqueue_dither((long long)no, static_cast<double*>(dith.p), mtbuf, e->side)) != KBSRC_GPU_OK)
                return rc;
            KB_CUDA(cudaEventRecord(dith_done, e->side));
            KB_CUDA(cudaStreamWaitEvent(st, dith_done, 0));
        }
        if ((rc = enqueue_pack((const double*)e->d_out.p, d.channels, d.nout, d.nout, format,
                               use_dither ? (const double*)dith.p : nullptr, (unsigned char*)bytes.p,
                               (unsigned long long*)cnt.p, st)) != KBSRC_GPU_OK)
            return rc;
        unsigned long long c = 0;
        if ((rc = copy_d2h(e->stager, out_bytes, bytes.p, nb, st)) != KBSRC_GPU_OK) return rc;
        KB_CUDA(cudaMemcpyAsync(&c, cnt.p, 8, cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaStreamSynchronize(st));
        if (clipped) *clipped = (long long)c;
        return KBSRC_GPU_OK;
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_pack(const double* d_planar, int channels, long long frames, long long stride, int format, int dither,
                   unsigned char* d_out, long long* clipped, void* stream) {
    if ((!d_planar || !d_out) && frames > 0) return fail(KBSRC_GPU_E_ARG, "null buffer");
    if (channels < 1 || frames < 0 || stride < frames || format < 0 || format > 4)
        return fail(KBSRC_GPU_E_ARG, "bad pack arguments");
    try {
        const long long n = frames * channels;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        int rc;
        DevBuf dith, cnt, mtbuf;
        if ((rc = cnt.alloc(8)) != KBSRC_GPU_OK) return rc;
        const bool use_dither = dither && format >= 2 && n > 0;
        if (use_dither && (rc = dith.alloc((size_t)n * 8)) != KBSRC_GPU_OK) return rc;
        KB_CUDA(cudaMemsetAsync(cnt.p, 0, 8, st));
        if (use_dither && (rc = enqueue_dither(n, static_cast<double*>(dith.p), mtbuf, st)) != KBSRC_GPU_OK) return rc;
        if ((rc = enqueue_pack(d_planar, channels, frames, stride, format,
                               use_dither ? (const double*)dith.p : nullptr, d_out, (unsigned long long*)cnt.p, st)) !=
            KBSRC_GPU_OK)
            return rc;
        unsigned long long c = 0;
        KB_CUDA(cudaMemcpyAsync(&c, cnt.p, 8, cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaStreamSynchronize(st));  // the temporaries are freed on return
        if (clipped) *clipped = (long long)c;
        return KBSRC_GPU_OK;
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_engine_info(const kbsrc_gpu_engine* e, long long* tasks, long long* launches, long long* device_bytes) {
    if (!e) return fail(KBSRC_GPU_E_ARG, "null engine");
    if (tasks) *tasks = e->tasks;
    if (launches) {
        const long long per_wave = plan_launches(*e);
        *launches = e->tasks ? per_wave * ((e->tasks + e->wave - 1) / e->wave) : 0;
    }
    if (device_bytes) {
        *device_bytes = (long long)(plan_table_bytes(*e) + e->bufA.bytes + e->bufB.bytes + e->d_in.bytes + e->d_head.bytes +
                                    e->d_tail.bytes + e->d_out.bytes);
    }
    return KBSRC_GPU_OK;
}

void kbsrc_gpu_engine_destroy(kbsrc_gpu_engine* e) { delete e; }

int kbsrc_gpu_kernel_spectrum(const double* taps, int L, int n, double scale, double* H) {
    if (!taps || !H || L < 0 || n < 2 || n % 2 || 2LL * L >= n)
        return fail(KBSRC_GPU_E_ARG, "bad kernel spectrum arguments");
    try {
        int rc = require_device();
        if (rc) return rc;
        if ((rc = allow_large_smem()) != KBSRC_GPU_OK) return rc;
        cudaStream_t st = nullptr;
        KB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamDestroy(s); }
        } sg{st};
        // the symmetric kernel placed circularly (design.cpp:42-43)
        std::vector<double> r((size_t)2 * n, 0.0);
        r[0] = taps[0];
        r[1] = taps[1];
        for (int m = 1; m <= L; m++) {
            r[2 * (size_t)m] = taps[2 * m]; r[2 * (size_t)m + 1] = taps[2 * m + 1];
            r[2 * (size_t)(n - m)] = taps[2 * m]; r[2 * (size_t)(n - m) + 1] = taps[2 * m + 1];
        }
        const int h = n / 2;
        DevCfft c;  // scalar double-double transform (RFFT<dd,dd,dd>), Bluestein when h is not 7-smooth
        if ((rc = make_dev_cfft(h, kTabDD, 4, c, st)) != KBSRC_GPU_OK) return rc;
        DevBuf w, rin, A, B, Hd;
        if ((rc = upload_cx(split_roots(n), kTabDD, w)) != KBSRC_GPU_OK) return rc;
        if ((rc = rin.alloc(r.size() * 8)) != KBSRC_GPU_OK) return rc;
        const size_t slot = (size_t)std::max<long long>(h + 1, c.slot()) * 32;
        if ((rc = A.alloc(slot)) != KBSRC_GPU_OK) return rc;
        if ((rc = B.alloc(slot)) != KBSRC_GPU_OK) return rc;
        if ((rc = Hd.alloc((size_t)(h + 1) * 16)) != KBSRC_GPU_OK) return rc;
        KB_CUDA(cudaMemcpyAsync(rin.p, r.data(), r.size() * 8, cudaMemcpyHostToDevice, st));
        using C = CxR<ArDDAccurate>;
        Slots sl{};
        sl.nt = 1;
        sl.ddreal = static_cast<const double*>(rin.p);
        Trail tr;
        void *zbuf, *xbuf;
        if (c.m) {
            zbuf = A.p;
            xbuf = B.p;
            rc = launch_cfft<ArDDAccurate, ArDDAccurate, kSrcDDReal, kDstComplex>(c, sl, nullptr, A.p, B.p, A.p, st, tr,
                                                                               -1, -1);
        } else {
            zbuf = B.p;
            xbuf = A.p;
            rc = launch_cfft<ArDDAccurate, ArDDAccurate, kSrcDDReal, kDstComplex>(c, sl, A.p, nullptr, nullptr, B.p,
                                                                               st, tr, -1, -1);
        }
        if (rc) return rc;
        SpecParams<ArDDAccurate> s{};
        s.Z = static_cast<C*>(zbuf);
        s.X = static_cast<C*>(xbuf);
        s.w_fw = static_cast<const CxW<ArDDAccurate>*>(w.p);
        s.h = h; s.scale = scale; s.Hout = static_cast<dd*>(Hd.p);
        k_split<ArDDAccurate><<<grid_for(h / 2 + 1, 256), 256, 0, st>>>(s);
        k_design_out<<<grid_for(h + 1, 256), 256, 0, st>>>(s);
        KB_CUDA(cudaGetLastError());
        KB_CUDA(cudaMemcpyAsync(H, Hd.p, (size_t)(h + 1) * 16, cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaStreamSynchronize(st));
        return KBSRC_GPU_OK;
    } catch (const std::bad_alloc&) {
        return fail(KBSRC_GPU_E_NOMEM, "host allocation failed");
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_kernel_spectrum_static(const double* d_taps, int L, int n, double scale, double* d_H, void* stream) {
    if (!d_taps || !d_H || L < 0 || n < 2 || n % 2 || 2LL * L >= n)
        return fail(KBSRC_GPU_E_ARG, "bad kernel spectrum arguments");
    try {
        int rc = require_device();
        if (rc) return rc;
        rc = allow_large_smem();
        if (rc) return rc;
        // the device address of the scratch array in the current device's context, looked up on every call (it
        // allocates nothing and stays right if the context is ever recreated)
        void* sym = nullptr;
        const cudaError_t se = cudaGetSymbolAddress(&sym, g_spectrum_scratch);
        if (se != cudaSuccess || !sym)
            return fail(KBSRC_GPU_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(se));
        unsigned char* base = static_cast<unsigned char*>(sym);
        // the plan only (fixed-size structures); every table is computed on the device below
        const int h = n / 2;
        HostCfft c;
        if ((rc = plan_cfft(h, c)) != KBSRC_GPU_OK) return rc;
        const size_t esize = 32;
        const long long n_stage = c.four ? (long long)c.s1.twn + c.s2.twn : c.sd.twn;
        DevRoots rt_w = dev_roots_shape(n), rt_h = dev_roots_shape(h), rt_1 = dev_roots_shape(c.four ? c.N1 : h),
                 rt_2 = dev_roots_shape(c.four ? c.N2 : 1);
        size_t at = 0;
        auto take = [&](size_t bytes) {
            const size_t o = at;
            at = align256(at + bytes);
            return o;
        };
        const size_t off_r = take((size_t)n * 16), off_A = take((size_t)(h + 1) * esize),
                     off_B = take((size_t)(h + 1) * esize), off_w = take((size_t)(h + 1) * esize),
                     off_ts = take((size_t)n_stage * esize), off_t4 = take(c.four ? (size_t)h * esize : 0),
                     off_rw = take((size_t)(rt_w.coarse + rt_w.step) * esize),
                     off_rh = take(c.four ? (size_t)(rt_h.coarse + rt_h.step) * esize : 0),
                     off_r1 = take((size_t)(rt_1.coarse + rt_1.step) * esize),
                     off_r2 = take(c.four ? (size_t)(rt_2.coarse + rt_2.step) * esize : 0);
        if (at > kSpectrumScratchBytes)
            return fail(KBSRC_GPU_E_ARG, "kernel spectrum of " + std::to_string(n) + " points needs " +
                                             std::to_string(at) + " bytes of scratch; the static scratch holds " +
                                             std::to_string(kSpectrumScratchBytes) + " (about 300,000 points)");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        using C = CxR<ArDDAccurate>;
        auto tab = [&](size_t off) { return reinterpret_cast<cx<dd>*>(base + off); };
        // root tables, then the real-FFT split roots w_n^-k (k <= n/2), the stage and the four-step twiddles
        auto roots = [&](DevRoots& r, size_t off) {
            r.t = tab(off);
            k_roots_build<<<grid_for(r.coarse + r.step, 128), 128, 0, st>>>(r, tab(off));
        };
        roots(rt_w, off_rw);
        roots(rt_1, off_r1);
        if (c.four) {
            roots(rt_h, off_rh);
            roots(rt_2, off_r2);
        }
        k_roots_table<<<grid_for(h + 1, 128), 128, 0, st>>>(rt_w, h + 1, 0, tab(off_w));
        if (c.four) {
            k_roots_stages<<<grid_for(c.s1.twn, 128), 128, 0, st>>>(rt_1, c.s1, tab(off_ts));
            k_roots_stages<<<grid_for(c.s2.twn, 128), 128, 0, st>>>(rt_2, c.s2, tab(off_ts) + c.s1.twn);
            k_roots_table<<<grid_for(h, 128), 128, 0, st>>>(rt_h, h, c.N2, tab(off_t4));
        } else {
            k_roots_stages<<<grid_for(c.sd.twn, 128), 128, 0, st>>>(rt_1, c.sd, tab(off_ts));
        }
        double* r = reinterpret_cast<double*>(base + off_r);
        C* A = reinterpret_cast<C*>(base + off_A);
        C* B = reinterpret_cast<C*>(base + off_B);
        k_place_taps<<<grid_for(n, 256), 256, 0, st>>>(d_taps, L, n, r);
        PassParams<ArDDAccurate> p{};
        p.tw_stage = reinterpret_cast<const CxW<ArDDAccurate>*>(base + off_ts);
        p.odd = odd_table<dd>();
        p.ddreal = r;
        p.stride = 0;
        if (c.four) {
            const Shape sc = pick_shape(c.s1, c.N2, esize, 4, KB_MAXT_DD_COL), sr = pick_shape(c.s2, c.N1, esize, 4, KB_MAXT_DD);
            p.sp = c.s1; p.N1 = c.N1; p.N2 = c.N2; p.F = sc.F;
            p.tw4 = reinterpret_cast<const CxW<ArDDAccurate>*>(base + off_t4);
            p.src = A; p.dst = A;
            const dim3 gc((c.N2 + sc.F - 1) / sc.F, 1), gr((c.N1 + sr.F - 1) / sr.F, 1);
            if (sc.twg) k_column<ArDDAccurate, kSrcDDReal, true><<<gc, sc.T, sc.smem, st>>>(p);
            else k_column<ArDDAccurate, kSrcDDReal, false><<<gc, sc.T, sc.smem, st>>>(p);
            p.sp = c.s2; p.F = sr.F; p.src = A; p.dst = B;
            if (sr.twg) k_row<ArDDAccurate, kDstComplex, true><<<gr, sr.T, sr.smem, st>>>(p);
            else k_row<ArDDAccurate, kDstComplex, false><<<gr, sr.T, sr.smem, st>>>(p);
        } else {
            const Shape sd = direct_shape(c.sd, esize);
            p.sp = c.sd; p.F = 1; p.dst = B;
            k_direct<ArDDAccurate, kSrcDDReal, kDstComplex><<<dim3(1, 1), sd.T, sd.smem, st>>>(p);
        }
        SpecParams<ArDDAccurate> s{};
        s.Z = B; s.X = A;
        s.w_fw = reinterpret_cast<const CxW<ArDDAccurate>*>(base + off_w);
        s.h = h; s.scale = scale; s.Hout = reinterpret_cast<dd*>(d_H);
        k_split<ArDDAccurate><<<grid_for(h / 2 + 1, 256), 256, 0, st>>>(s);
        k_design_out<<<grid_for(h + 1, 256), 256, 0, st>>>(s);
        KB_CUDA(cudaGetLastError());
        return KBSRC_GPU_OK;
    } catch (const std::bad_alloc&) {
        return fail(KBSRC_GPU_E_NOMEM, "host allocation failed");
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_batch_create(const kbsrc_gpu_desc* descs, int count, kbsrc_gpu_batch** out) {
    if (!out) return fail(KBSRC_GPU_E_ARG, "null output pointer");
    *out = nullptr;
    try {
        return batch_create_impl(descs, count, out);
    } catch (const std::bad_alloc&) {
        return fail(KBSRC_GPU_E_NOMEM, "host allocation failed");
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_ARG, x.what());
    }
}

int kbsrc_gpu_batch_run_device(kbsrc_gpu_batch* b, const double* const* d_in, const double* const* d_head,
                               const double* const* d_tail, double* const* d_out, void* stream) {
    if (!b || !d_in || !d_out) return fail(KBSRC_GPU_E_ARG, "null batch or buffer array");
    try {
        return batch_run_device_impl(*b, d_in, d_head, d_tail, d_out, stream ? (cudaStream_t)stream : b->stream);
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_batch_run_host(kbsrc_gpu_batch* b, const double* const* in, const double* const* head,
                             const double* const* tail, double* const* out) {
    if (!b || !in || !out) return fail(KBSRC_GPU_E_ARG, "null batch or buffer array");
    try {
        const int count = (int)b->descs.size();
        int rc;
        if (b->d_in.empty()) {
            b->d_in.resize(count); b->d_head.resize(count); b->d_tail.resize(count); b->d_out.resize(count);
            for (int i = 0; i < count; i++) {
                const kbsrc_gpu_desc& d = b->descs[i];
                if ((rc = b->d_in[i].alloc((size_t)(d.frames * d.channels * in_bytes(d.in_format)))) != KBSRC_GPU_OK)
                    return rc;
                if ((rc = b->d_head[i].alloc((size_t)(d.edge_len * d.channels * 8))) != KBSRC_GPU_OK) return rc;
                if ((rc = b->d_tail[i].alloc((size_t)(d.edge_len * d.channels * 8))) != KBSRC_GPU_OK) return rc;
                if ((rc = b->d_out[i].alloc((size_t)(d.nout * d.channels * 8))) != KBSRC_GPU_OK) return rc;
            }
        }
        std::vector<const double*> pi(count), ph(count), pt(count);
        std::vector<double*> po(count);
        cudaStream_t st = b->stream;
        for (int i = 0; i < count; i++) {
            const kbsrc_gpu_desc& d = b->descs[i];
            const size_t ni = (size_t)(d.frames * d.channels * in_bytes(d.in_format)),
                         ne = (size_t)(d.edge_len * d.channels * 8);
            if (ni) KB_CUDA(cudaMemcpyAsync(b->d_in[i].p, in[i], ni, cudaMemcpyHostToDevice, st));
            if (ne && head && tail) {
                KB_CUDA(cudaMemcpyAsync(b->d_head[i].p, head[i], ne, cudaMemcpyHostToDevice, st));
                KB_CUDA(cudaMemcpyAsync(b->d_tail[i].p, tail[i], ne, cudaMemcpyHostToDevice, st));
            }
            pi[i] = (const double*)b->d_in[i].p; ph[i] = (const double*)b->d_head[i].p;
            pt[i] = (const double*)b->d_tail[i].p; po[i] = (double*)b->d_out[i].p;
        }
        if ((rc = batch_run_device_impl(*b, pi.data(), ph.data(), pt.data(), po.data(), st)) != KBSRC_GPU_OK) return rc;
        for (int i = 0; i < count; i++) {
            const kbsrc_gpu_desc& d = b->descs[i];
            if (d.nout) KB_CUDA(cudaMemcpyAsync(out[i], po[i], (size_t)(d.nout * d.channels * 8), cudaMemcpyDeviceToHost, st));
        }
        KB_CUDA(cudaStreamSynchronize(st));
        return KBSRC_GPU_OK;
    } catch (const std::exception& x) {
        return fail(KBSRC_GPU_E_CUDA, x.what());
    }
}

int kbsrc_gpu_batch_info(const kbsrc_gpu_batch* b, long long* groups, long long* tasks, long long* launches) {
    if (!b) return fail(KBSRC_GPU_E_ARG, "null batch");
    long long t = 0, l = 0;
    for (const auto& g : b->groups) {
        t += g->tasks;
        l += plan_launches(*g) * ((g->tasks + g->wave - 1) / g->wave);
    }
    if (b->queued) {
        l = 6 * (long long)b->q_waves.size();
        for (const auto& g : b->groups)
            if (!g->queued) l += plan_launches(*g) * ((g->tasks + g->wave - 1) / g->wave);
    }
    if (groups) *groups = (long long)b->groups.size();
    if (tasks) *tasks = t;
    if (launches) *launches = l + 1;  // + the output zeroing
    return KBSRC_GPU_OK;
}

void kbsrc_gpu_batch_destroy(kbsrc_gpu_batch* b) {
    if (b && b->done) cudaEventSynchronize(b->done);
    delete b;
}

const char* kbsrc_gpu_last_error(void) { return g_error.c_str(); }

const char* kbsrc_gpu_engine_name(void) { return "sm_100a"; }

}  // extern "C"
