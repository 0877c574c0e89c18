// Split-precision DFT on the tensor cores: each stage of a sub-FFT is one dense DFT-matrix contraction of 8-bit
// digit slices on tcgen05, accumulated exactly in TMEM and recombined in float64.
//
// A stage transforms up to 128 row vectors of R complex float64 values. Each row is scaled by its own power of
// two and rounded to an integer of at most 55 bits, x = 2^(E-55) * X with |X| <= 2^55 - 2^48 (E the exponent bound
// of the row's largest magnitude, one higher when its top six mantissa bits are all set), and X is written in
// seven balanced base-256 digits, X = sum_i s_i 256^i with s_i in [-128, 127]: the bytes of X + 0x80808080808080,
// each minus 128. The real form of the DFT_R matrix (entries cos and +-sin, |w| <= 1) is cut the same way from
// W = rint(w 2^54). Digit slices are numbered from the top (slice t holds digit 6 - t); the products of data slice
// ta and matrix slice tb with ta + tb = d accumulate in accumulator d for d <= 7 (34 of the 49 products; the
// dropped ones sum to below 2^-54 of the row's scale per output), and
//     y = 2^(E-109) * 2^40 * sum_d C_d 256^(7-d) = hi 2^(E-37) + lo 2^(E-69)
// with hi, lo two exact integer Horner sums of four accumulators each: two exact conversions and one rounded
// float64 addition. The result is within float64 rounding of the exact stage output: the accuracy of a float64
// engine, not the bit pattern of any reference engine.
//
// The digits reach the tensor cores as int8 (kind::i8, int32 accumulators) or as f16 (kind::f16, f32
// accumulators): every digit product is below 2^14 and every accumulator below 2^23 in magnitude, so both sums are
// exact and the two element kinds give the same bits.
//
// Shared-memory operands use the canonical K-major layout of tc.cuh: K = [real half | imaginary half] of 2*kh
// elements, N = [real outputs | imaginary outputs] of 2*nh columns.
#pragma once
#include <cuda_fp16.h>

#include "fft.cuh"
#include "tc.cuh"

namespace kbsrc::dev {

constexpr int kTcDigits = 7;           // 8-bit digits per value (56 bits, 55 used)
constexpr int kTcAcc = 8;              // accumulators d = ta + tb = 0..7
constexpr int kTcMats = kTcDigits + 1; // matrix slices, the last one zero (it initialises accumulator 7)
constexpr int kTcRows = 128;           // MMA M: row vectors per stage
constexpr int kTcThreads = 512;        // four threads per row while slicing; four warpgroups while recombining
constexpr int kTcWaitLimit = 1 << 22;  // mbarrier polls before a stage reports a timeout

// Element kinds of the digit slices. kBytes: bytes per element; the MMA consumes 32 bytes of K per instruction.
struct TcI8 {
    static constexpr int kBytes = 1;
    static __device__ __forceinline__ uint32_t idesc(int M, int N) { return umma_idesc_s8(M, N); }
    static __device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
        umma_s8(d, a, b, id, acc);
    }
    static __device__ __forceinline__ int acc_value(int32_t v) { return v; }
};
struct TcF16 {
    static constexpr int kBytes = 2;
    static __device__ __forceinline__ uint32_t idesc(int M, int N) { return umma_idesc_f16(M, N); }
    static __device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
        umma_f16(d, a, b, id, acc);
    }
    // the f32 accumulator holds an integer below 2^23 exactly
    static __device__ __forceinline__ int acc_value(int32_t v) { return __float2int_rn(__int_as_float(v)); }
};

// One radix of the split form: the sliced real DFT_R matrix (global memory, kTcMats * 2nh * 2kh elements). Its
// output columns come in `rounds` (1, or 2 when the accumulators of all 2nh columns do not fit the TMEM columns a
// CTA half owns: real outputs, then imaginary outputs), laid out [round][slice][2nh / rounds rows][2kh], so that
// consecutive slices of a round form one operand of kTcMats times its columns.
struct TcRadix {
    int R, kh, nh, rounds;
    const uint4* slices;
};

// A sub-FFT of N = a.R * b.R * c.R points (b.R == 1: one stage; c.R == 1: two stages) on F sequences per item,
// every stage at most 128 rows (F * N / R <= 128 for each radix R); ebytes: element kind (1 int8, 2 f16). halves:
// items a CTA works on at once (1, or 2: each half of the CTA, 256 threads, with its own planes, slices, TMEM
// columns and mbarrier, so that one item's MMAs and waits overlap the other's slicing and recombination). Inner
// twiddles, M = b.R * c.R: tw[k1 * M + m] = e^{-2 pi i m k1 / N}, then (three radices)
// tw[N + c1 * c.R + v] = e^{-2 pi i v c1 / M}.
struct TcSub {
    int N, F, ebytes, halves;
    TcRadix a, b, c;
    const double2* tw;
};
__host__ __device__ inline int tc_tw_count(const TcSub& s) { return s.c.R > 1 ? s.N + s.b.R * s.c.R : s.N; }
// TMEM columns a CTA half owns, and the rounds of a radix with 2nh output columns
__host__ __device__ inline int tc_half_cols(int halves) { return halves == 2 ? 256 : 512; }
__host__ __device__ inline int tc_rounds_for(int nh, int halves) {
    return kTcAcc * 2 * nh <= tc_half_cols(halves) ? 1 : 2;
}

__host__ __device__ inline int tc_bm_bytes(const TcRadix& r, int eb) {
    return r.R > 1 ? kTcMats * (2 * r.nh) * (2 * r.kh) * eb : 0;
}
// K row bytes of the data slices: the widest radix of the sub-FFT
__host__ __device__ inline int tc_kpad(const TcSub& s) {
    int k = s.a.kh > s.b.kh ? s.a.kh : s.b.kh;
    if (s.c.R > 1 && s.c.kh > k) k = s.c.kh;
    return 2 * k * s.ebytes;
}
__host__ __device__ inline size_t tc_align(size_t v) { return (v + 127) & ~(size_t)127; }
// plane pairs an item needs: Y between the stages, and X too with three radices
__host__ __device__ inline int tc_plane_pairs(const TcSub& s) { return s.c.R > 1 ? 2 : 1; }
__host__ __device__ inline size_t tc_half_bytes(const TcSub& s) {
    return tc_align((size_t)tc_plane_pairs(s) * s.N * s.F * 16) + tc_align((size_t)kTcDigits * kTcRows * tc_kpad(s)) +
           tc_align(kTcRows * 4);
}

// Shared bytes of a split-form CTA: per half its planes, slices and row exponents; then the sliced matrices, the
// inner twiddles, the mbarriers and the TMEM address.
__host__ __device__ inline size_t tc_smem_bytes(const TcSub& s) {
    return s.halves * tc_half_bytes(s) + tc_align(tc_bm_bytes(s.a, s.ebytes)) + tc_align(tc_bm_bytes(s.b, s.ebytes)) +
           tc_align(tc_bm_bytes(s.c, s.ebytes)) + tc_align((size_t)tc_tw_count(s) * 16) + 128;
}

// What one half of a CTA works with: its threads (t = index within the half, kT of them), planes, slices, row
// exponents, TMEM columns and mbarrier; the shared matrices and twiddles.
struct TcHalf {
    int id, t;
    Planes<ArF64> X, Y;
    unsigned char* slices;
    int* expo;
    uint64_t* mbar;
    uint32_t tmem;
    const unsigned char* bm_a;
    const unsigned char* bm_b;
    const unsigned char* bm_c;
    const double2* tw;
};

struct TcSmem {
    unsigned char* half[2];
    unsigned char* bm_a;
    unsigned char* bm_b;
    unsigned char* bm_c;
    double2* tw;
    uint64_t* mbar;  // one per half
    uint32_t* tmem_slot;
};

__device__ inline TcSmem tc_carve(unsigned char* p, const TcSub& s) {
    TcSmem m;
    for (int h = 0; h < 2; h++) {
        m.half[h] = p;
        if (h < s.halves) p += tc_half_bytes(s);
    }
    m.bm_a = p;
    p += tc_align(tc_bm_bytes(s.a, s.ebytes));
    m.bm_b = p;
    p += tc_align(tc_bm_bytes(s.b, s.ebytes));
    m.bm_c = p;
    p += tc_align(tc_bm_bytes(s.c, s.ebytes));
    m.tw = reinterpret_cast<double2*>(p);
    p += tc_align((size_t)tc_tw_count(s) * 16);
    m.mbar = reinterpret_cast<uint64_t*>(p);
    m.tmem_slot = reinterpret_cast<uint32_t*>(p + 16);
    return m;
}

// The view of half `id` (threads 256 id .. when there are two halves, all threads otherwise).
__device__ inline TcHalf tc_half(const TcSmem& m, const TcSub& s, int id, uint32_t tmem) {
    TcHalf h;
    h.id = id;
    h.t = s.halves == 2 ? (int)threadIdx.x - 256 * id : (int)threadIdx.x;
    unsigned char* p = m.half[id];
    const int nf = s.N * s.F;
    double* pl = reinterpret_cast<double*>(p);
    h.Y = Planes<ArF64>{pl, pl + nf};
    h.X = tc_plane_pairs(s) > 1 ? Planes<ArF64>{pl + 2 * nf, pl + 3 * nf} : h.Y;
    p += tc_align((size_t)tc_plane_pairs(s) * nf * 16);
    h.slices = p;
    p += tc_align((size_t)kTcDigits * kTcRows * tc_kpad(s));
    h.expo = reinterpret_cast<int*>(p);
    h.mbar = m.mbar + id;
    h.tmem = tmem + (uint32_t)(id * tc_half_cols(s.halves));
    h.bm_a = m.bm_a;
    h.bm_b = m.bm_b;
    h.bm_c = m.bm_c;
    h.tw = m.tw;
    return h;
}

// TMEM allocation (all 512 columns), the mbarriers, and the CTA's copies of the sliced matrices and inner
// twiddles. Ends with the CTA synchronised; returns the TMEM base address.
__device__ inline uint32_t tc_setup(const TcSmem& m, const TcSub& s) {
    if (threadIdx.x < 32) tmem_alloc(m.tmem_slot, 512u);
    if (threadIdx.x == 0) {
        mbar_init(m.mbar, 1);
        mbar_init(m.mbar + 1, 1);
    }
    const int na = tc_bm_bytes(s.a, s.ebytes) / 16, nb = tc_bm_bytes(s.b, s.ebytes) / 16,
              nc = tc_bm_bytes(s.c, s.ebytes) / 16, nt = tc_tw_count(s);
#pragma unroll 4
    for (int i = threadIdx.x; i < na; i += blockDim.x) reinterpret_cast<uint4*>(m.bm_a)[i] = __ldg(s.a.slices + i);
#pragma unroll 4
    for (int i = threadIdx.x; i < nb; i += blockDim.x) reinterpret_cast<uint4*>(m.bm_b)[i] = __ldg(s.b.slices + i);
#pragma unroll 4
    for (int i = threadIdx.x; i < nc; i += blockDim.x) reinterpret_cast<uint4*>(m.bm_c)[i] = __ldg(s.c.slices + i);
    for (int i = threadIdx.x; i < nt; i += blockDim.x) m.tw[i] = __ldg(s.tw + i);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *m.tmem_slot;
}

__device__ inline void tc_teardown(uint32_t tmem) {
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) tmem_dealloc(tmem, 512u);
}

// Barrier of the threads of one half (named barrier 1 + id, kT threads; the whole CTA when there is one half)
template <int kT>
__device__ __forceinline__ void tc_half_sync(const TcHalf& h) {
    if constexpr (kT == kTcThreads) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(1 + h.id), "r"(kT) : "memory");
    }
}

// 2^k as a float64 for k in the normal range [-1022, 1023]
__device__ __forceinline__ double tc_pow2(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }
// 2^k for k in [-1122, 1023] (below the normal range: the subnormal power of two, or zero)
__device__ __forceinline__ double tc_pow2_low(int k) {
    return k >= -1022 ? tc_pow2(k) : __dmul_rn(tc_pow2(k + 100), tc_pow2(-100));
}

// Row exponent bound E of a row whose largest magnitude has the bit pattern `maxbits`: |x| < 2^E, and E one higher
// when the top six mantissa bits are set, so that every X = rint(x 2^(55-E)) has |X| <= 2^55 - 2^48 and
// X + 0x80808080808080 stays within seven bytes.
__device__ __forceinline__ int tc_row_expo(unsigned long long maxbits) {
    const int ex = (int)(maxbits >> 52);
    return (ex ? ex - 1022 : -1022) + (((maxbits >> 46) & 0x3F) == 0x3F ? 1 : 0);
}

// Biased digits of x at row exponent E: byte i of the result is digit i of rint(x 2^(55-E)) plus 128 (bytes 0..6).
__device__ __forceinline__ unsigned long long tc_biased_digits(double x, int E) {
    const int sh = 55 - E, s1 = sh < 1000 ? sh : 1000;
    double v = __dmul_rn(x, tc_pow2(s1));  // exact: a power of two, no overflow
    if (sh > s1) v = __dmul_rn(v, tc_pow2(sh - s1));
    return (unsigned long long)(__double2ll_rn(v) + 0x80808080808080LL);
}

// 4x4 byte transpose: out[i] byte j = in[j] byte i
__device__ __forceinline__ void tc_transpose4(const uint32_t (&in)[4], uint32_t (&out)[4]) {
    const uint32_t e0 = __byte_perm(in[0], in[1], 0x5140), e1 = __byte_perm(in[0], in[1], 0x7362);
    const uint32_t e2 = __byte_perm(in[2], in[3], 0x5140), e3 = __byte_perm(in[2], in[3], 0x7362);
    out[0] = __byte_perm(e0, e2, 0x5410);
    out[1] = __byte_perm(e0, e2, 0x7632);
    out[2] = __byte_perm(e1, e3, 0x5410);
    out[3] = __byte_perm(e1, e3, 0x7632);
}

// Writes the digit slices of 8 consecutive K elements (k0 .. k0 + 7) of one row: b[v] holds the biased digits of
// value v. Slice t (top-indexed) receives digit 6 - t, as int8 or f16.
template <class S>
__device__ __forceinline__ void tc_put_digits(unsigned char* slices, int kpad, int row, int k0,
                                              const unsigned long long (&b)[8]) {
    uint32_t lo[2][4], hi[2][4];  // [values 0-3 | 4-7][digit]
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const uint32_t l[4] = {(uint32_t)b[4 * h], (uint32_t)b[4 * h + 1], (uint32_t)b[4 * h + 2], (uint32_t)b[4 * h + 3]};
        const uint32_t u[4] = {(uint32_t)(b[4 * h] >> 32), (uint32_t)(b[4 * h + 1] >> 32), (uint32_t)(b[4 * h + 2] >> 32),
                               (uint32_t)(b[4 * h + 3] >> 32)};
        tc_transpose4(l, lo[h]);
        tc_transpose4(u, hi[h]);
    }
#pragma unroll
    for (int i = 0; i < kTcDigits; i++) {
        const uint32_t w0 = i < 4 ? lo[0][i] : hi[0][i - 4], w1 = i < 4 ? lo[1][i] : hi[1][i - 4];
        unsigned char* base = slices + (kTcDigits - 1 - i) * kTcRows * kpad;
        if constexpr (S::kBytes == 1) {
            *reinterpret_cast<uint2*>(base + umma_off(row, k0, kpad)) = make_uint2(w0 ^ 0x80808080u, w1 ^ 0x80808080u);
        } else {
            // biased byte b -> the f16 of 1408 + b (bits 0x6580 + b, no carry between lanes), minus 1536 exactly
            const __half2 off = __float2half2_rn(1536.0f);
            uint32_t h[4] = {__byte_perm(w0, 0, 0x4140), __byte_perm(w0, 0, 0x4342), __byte_perm(w1, 0, 0x4140),
                             __byte_perm(w1, 0, 0x4342)};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                h[j] += 0x65806580u;
                __half2 v = *reinterpret_cast<__half2*>(&h[j]);
                v = __hsub2(v, off);
                h[j] = *reinterpret_cast<uint32_t*>(&v);
            }
            *reinterpret_cast<uint4*>(base + umma_off(row, 2 * k0, kpad)) = make_uint4(h[0], h[1], h[2], h[3]);
        }
    }
}

// y = hi 2^(E-37) + lo 2^(E-69) from the accumulators C_0..C_7 of one output column (see the top of the file)
template <class S>
__device__ __forceinline__ double tc_combine(const int32_t (&c)[kTcAcc][4], int u, double s1, double s2) {
    const long long hi = (((long long)S::acc_value(c[0][u]) * 256 + S::acc_value(c[1][u])) * 256 +
                          S::acc_value(c[2][u])) * 256 + S::acc_value(c[3][u]);
    const long long lo = (((long long)S::acc_value(c[4][u]) * 256 + S::acc_value(c[5][u])) * 256 +
                          S::acc_value(c[6][u])) * 256 + S::acc_value(c[7][u]);
    return __dadd_rn(__dmul_rn(__ll2double_rn(hi), s1), __dmul_rn(__ll2double_rn(lo), s2));
}

// One contraction stage on one half: `nrows` rows of R complex values. load(row, j) -> double2 (real, imaginary)
// for j < R; store(row, k, re, im) for output k < R. `phase` counts the half's mbarrier phases completed so far.
// Starts and ends with the half synchronised (what load reads must be visible on entry; what store writes is
// visible on return). kT: threads of the half (512 or 256); kRounds: the radix's rounds (1, or 2 with kT = 256).
//   slicing        thread t: row t / (kT/128), 8-element chunks 8 (t % (kT/128)) + 8 (kT/128) i of both halves of K;
//                  the row exponent by shuffles between the row's threads (with two chunks per thread the values
//                  are read twice, once for the exponent and once for the digits, to keep them out of registers)
//   MMA            thread 0: per round, data slice ta against matrix slices 0..7-ta side by side, accumulators ta..7
//   recombination  warp w: TMEM lanes 32 (w % 4) ..; the warpgroups take interleaved groups of 4 outputs; with two
//                  rounds the real parts wait in registers for the imaginary parts
template <class S, int kT, int kRounds, class Load, class Store>
__device__ inline void tc_stage(const TcRadix& rad, int nrows, const TcHalf& h, const unsigned char* bmat,
                                uint32_t& phase, int* err, Load load, Store store) {
    constexpr int kTPR = kT / kTcRows, kGroups = kT / 128;  // threads per row while slicing; warpgroups
    constexpr int kChunks = 32 / kTPR / 8;                  // 8-element chunks per thread, at most
    constexpr int kIters = 32 / (4 * kGroups);              // output groups of 4 per warpgroup, at most
    const int R = rad.R, kh = rad.kh, nh = rad.nh, npad = 2 * nh, kpad = 2 * kh * S::kBytes;
    const int nr = npad / kRounds;
    const int t = h.t;
    {
        const int row = t / kTPR, q = t % kTPR;
        const bool live = row < nrows;
        auto chunk = [&](int i, double2 (&v)[8]) {
            const int j0 = 8 * (q + kTPR * i);
#pragma unroll
            for (int u = 0; u < 8; u++) v[u] = live && j0 + u < R ? load(row, j0 + u) : make_double2(0.0, 0.0);
        };
        auto magnitude = [](const double2 (&v)[8], unsigned long long mx) {
#pragma unroll
            for (int u = 0; u < 8; u++) {
                mx = max(mx, (unsigned long long)__double_as_longlong(v[u].x) & 0x7FFFFFFFFFFFFFFFull);
                mx = max(mx, (unsigned long long)__double_as_longlong(v[u].y) & 0x7FFFFFFFFFFFFFFFull);
            }
            return mx;
        };
        auto put = [&](int i, const double2 (&v)[8], int E) {
            const int j0 = 8 * (q + kTPR * i);
            if (!live || j0 >= kh) return;
            unsigned long long br[8], bi[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                br[u] = tc_biased_digits(v[u].x, E);
                bi[u] = tc_biased_digits(v[u].y, E);
            }
            tc_put_digits<S>(h.slices, kpad, row, j0, br);
            tc_put_digits<S>(h.slices, kpad, row, kh + j0, bi);
        };
        double2 v[8];
        unsigned long long mx = 0;
        if constexpr (kChunks == 1) {
            chunk(0, v);
            mx = magnitude(v, mx);
        } else {
#pragma unroll 1
            for (int i = 0; i < kChunks; i++) {
                chunk(i, v);
                mx = magnitude(v, mx);
            }
        }
#pragma unroll
        for (int o = 1; o < kTPR; o <<= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        const int E = tc_row_expo(mx);
        if (q == 0) h.expo[row] = E;
        if constexpr (kChunks == 1) {
            put(0, v, E);
        } else {
#pragma unroll 1
            for (int i = 0; i < kChunks; i++) {
                chunk(i, v);
                put(i, v, E);
            }
        }
    }
    fence_async_smem();
    const int warp = t >> 5, lq = warp & 3, g = warp >> 2, row = 32 * lq + (t & 31);
    const uint32_t lane_addr = h.tmem + ((uint32_t)(32 * lq) << 16);
    double yre[kRounds == 2 ? 4 * kIters : 1];  // real outputs of round 0 while round 1 runs
#pragma unroll
    for (int rd = 0; rd < kRounds; rd++) {
        tc_fence_before();
        tc_half_sync<kT>(h);  // slices written (round 0), or the previous round's TMEM reads done (round 1)
        tc_fence_after();
        if (t == 0) {
            const uint32_t sa = smem_u32(h.slices), sb = smem_u32(bmat) + rd * kTcMats * nr * kpad,
                           sbo = 8 * kpad;
            const int bpc = 256 / nr, ksteps = kpad / 32;
            for (int ta = 0; ta < kTcDigits; ta++)
                for (int d0 = ta; d0 < kTcAcc; d0 += bpc) {
                    const int nb = min(bpc, kTcAcc - d0);
                    const uint32_t idesc = S::idesc(kTcRows, nb * nr);
                    for (int ks = 0; ks < ksteps; ks++)
                        S::mma(h.tmem + d0 * nr, umma_desc(sa + ta * kTcRows * kpad + 256 * ks, 128, sbo),
                               umma_desc(sb + (d0 - ta) * nr * kpad + 256 * ks, 128, sbo), idesc,
                               (ta || ks) ? 1u : 0u);
                }
            umma_commit(h.mbar);
        }
        bool ok = mbar_wait(h.mbar, phase & 1u, kTcWaitLimit);
        phase++;
        ok = __all_sync(0xffffffffu, ok);  // the TMEM loads below are warp-collective
        tc_fence_after();
        if (!ok) {
            if ((t & 31) == 0) atomicExch(err, 1);
            continue;
        }
        const int E = h.expo[row];
        const double s1 = tc_pow2_low(E - 37), s2 = tc_pow2_low(E - 69);
#pragma unroll
        for (int it = 0; it < kIters; it++) {
            const int k0 = 4 * g + 4 * kGroups * it;
            if (k0 >= R) break;
            if constexpr (kRounds == 1) {
                int32_t cr[kTcAcc][4], ci[kTcAcc][4];
#pragma unroll
                for (int d = 0; d < kTcAcc; d++) {
                    tmem_ld4(lane_addr + d * nr + k0, cr[d]);
                    tmem_ld4(lane_addr + d * nr + nh + k0, ci[d]);
                }
                tmem_wait_ld();
                if (row < nrows) {
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        if (k0 + u < R)
                            store(row, k0 + u, tc_combine<S>(cr, u, s1, s2), tc_combine<S>(ci, u, s1, s2));
                }
            } else {
                int32_t c[kTcAcc][4];
#pragma unroll
                for (int d = 0; d < kTcAcc; d++) tmem_ld4(lane_addr + d * nr + k0, c[d]);
                tmem_wait_ld();
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const double y = tc_combine<S>(c, u, s1, s2);
                    if (rd == 0) yre[4 * it + u] = y;
                    else if (row < nrows && k0 + u < R) store(row, k0 + u, yre[4 * it + u], y);
                }
            }
        }
    }
    tc_fence_before();
    tc_half_sync<kT>(h);
    tc_fence_after();
}

// tc_stage with the radix's rounds (two rounds only arise with two halves)
template <class S, int kT, class Load, class Store>
__device__ __forceinline__ void tc_stage_r(const TcRadix& rad, int nrows, const TcHalf& h, const unsigned char* bmat,
                                           uint32_t& phase, int* err, Load load, Store store) {
    if constexpr (kT == kTcThreads) {
        tc_stage<S, kT, 1>(rad, nrows, h, bmat, phase, err, load, store);
    } else {
        if (rad.rounds == 2) tc_stage<S, kT, 2>(rad, nrows, h, bmat, phase, err, load, store);
        else tc_stage<S, kT, 1>(rad, nrows, h, bmat, phase, err, load, store);
    }
}

__device__ __forceinline__ double2 tc_cmul(double re, double im, double2 w) {
    return make_double2(__dsub_rn(__dmul_rn(re, w.x), __dmul_rn(im, w.y)), __dadd_rn(__dmul_rn(re, w.y), __dmul_rn(im, w.x)));
}

// Sub-FFT of N points on F sequences by one half of the CTA, Cooley-Tukey through the stages of TcSub, from
// load_in(n, f) -> double2 (input n of sequence f) to store_out(k, f, re, im) (output k of sequence f, natural
// order). Intermediate stages live in the half's plane pairs Y (and X, three radices), element j of sequence f at
// j * F + f; each inter-stage twiddle is applied as the stage's outputs are stored. seq_fast: the first stage's
// rows run the sequences fastest (inputs of neighbouring rows are neighbours in a column pass) rather than the
// inputs (a row pass).
//   two radices,   n = Rb j + m, k = k1 + Ra k2: DFT_Ra over j, twiddle w_N^{m k1}, DFT_Rb over m
//   three radices, M = Rb Rc, n = M j + m, m = Rc u + v, k = k1 + Ra (c1 + Rb c2): DFT_Ra over j, w_N^{m k1},
//                  DFT_Rb over u, w_M^{v c1}, DFT_Rc over v
template <class S, int kT, class LoadIn, class StoreOut>
__device__ inline void tc_subfft(const TcSub& s, bool seq_fast, const TcHalf& h, uint32_t& phase, int* err,
                                 LoadIn load_in, StoreOut store_out) {
    const Planes<ArF64>& X = h.X;
    const Planes<ArF64>& Y = h.Y;
    const int F = s.F, Ra = s.a.R, Rb = s.b.R, Rc = s.c.R, M = Rb * (Rc > 1 ? Rc : 1);
    const FastDiv dF = fast_div(F), dM = fast_div(M);
    auto first_row = [&](int r, int& mm, int& f) {
        if (seq_fast) {
            mm = (int)fdiv(r, dF);
            f = r - mm * F;
        } else {
            f = (int)fdiv(r, dM);
            mm = r - f * M;
        }
    };
    tc_stage_r<S, kT>(s.a, M * F, h, h.bm_a, phase, err,
                [&](int r, int j) {
                    int mm, f;
                    first_row(r, mm, f);
                    return load_in(M * j + mm, f);
                },
                [&](int r, int k1, double re, double im) {
                    int mm, f;
                    first_row(r, mm, f);
                    if (Rb <= 1) {  // a single stage (a prime length of at most 32)
                        store_out(k1, f, re, im);
                        return;
                    }
                    const double2 y = tc_cmul(re, im, h.tw[k1 * M + mm]);
                    const int i = (k1 * M + mm) * F + f;
                    Y.re[i] = y.x;
                    Y.im[i] = y.y;
                });
    if (Rb <= 1) return;
    if (Rc <= 1) {
        tc_stage_r<S, kT>(s.b, Ra * F, h, h.bm_b, phase, err,
                    [&](int r, int mm) {
                        const int k1 = (int)fdiv(r, dF), f = r - k1 * F, i = (k1 * Rb + mm) * F + f;
                        return make_double2(Y.re[i], Y.im[i]);
                    },
                    [&](int r, int k2, double re, double im) {
                        const int k1 = (int)fdiv(r, dF), f = r - k1 * F;
                        store_out(k1 + Ra * k2, f, re, im);
                    });
        return;
    }
    const FastDiv dRb = fast_div(Rb), dRc = fast_div(Rc);
    tc_stage_r<S, kT>(s.b, Ra * Rc * F, h, h.bm_b, phase, err,
                [&](int r, int u) {
                    const int q = (int)fdiv(r, dF), f = r - q * F, k1 = (int)fdiv(q, dRc), v = q - k1 * Rc;
                    const int i = (k1 * M + Rc * u + v) * F + f;
                    return make_double2(Y.re[i], Y.im[i]);
                },
                [&](int r, int c1, double re, double im) {
                    const int q = (int)fdiv(r, dF), f = r - q * F, k1 = (int)fdiv(q, dRc), v = q - k1 * Rc;
                    const double2 y = tc_cmul(re, im, h.tw[s.N + c1 * Rc + v]);
                    const int i = (k1 * M + Rc * c1 + v) * F + f;
                    X.re[i] = y.x;
                    X.im[i] = y.y;
                });
    tc_stage_r<S, kT>(s.c, Ra * Rb * F, h, h.bm_c, phase, err,
                [&](int r, int v) {
                    const int q = (int)fdiv(r, dF), f = r - q * F, k1 = (int)fdiv(q, dRb), c1 = q - k1 * Rb;
                    const int i = (k1 * M + Rc * c1 + v) * F + f;
                    return make_double2(X.re[i], X.im[i]);
                },
                [&](int r, int c2, double re, double im) {
                    const int q = (int)fdiv(r, dF), f = r - q * F, k1 = (int)fdiv(q, dRb), c1 = q - k1 * Rb;
                    store_out(k1 + Ra * (c1 + Rb * c2), f, re, im);
                });
}

}  // namespace kbsrc::dev
