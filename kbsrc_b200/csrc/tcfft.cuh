// Split-precision DFT on the tensor cores: each stage of a sub-FFT is a dense DFT-matrix contraction of int8
// slices on tcgen05, accumulated exactly in int32 in TMEM and recombined in float64.
//
// A stage transforms up to 128 row vectors of R complex float64 values. Each row is scaled by its own power of
// two 2^E (the smallest above every |value| of the row) and cut into kTcSlices signed 7-bit slices,
//     x = 2^E * sum_i a_i 2^(-7(i+1)),  a_i in [-127, 127]   (56 bits: every float64 digit of the row's maximum),
// and the real form of the DFT_R matrix W (entries cos and +-sin, |w| <= 1) is cut the same way after halving,
// w = 2 * sum_j b_j 2^(-7(j+1)). The products a_i b_j with i + j = d accumulate exactly in int32 accumulator d
// for d <= 8 (43 of the 64 products; the dropped ones sum to below 2^-60 of the row's scale per term), and
//     y = 2^(E+1) * sum_d C_d 2^(-7(d+2))
// is formed from two exact int64 Horner sums, two exact conversions and one rounded float64 addition. The
// result is within float64 rounding of the exact stage output: the accuracy of a float64 engine, not the bit
// pattern of any reference engine.
//
// Shared-memory operands use the canonical K-major layout of tc.cuh: K = [real half | imaginary half] of 2*kh
// bytes, N = [real outputs | imaginary outputs] of 2*nh columns.
#pragma once
#include "fft.cuh"
#include "tc.cuh"

namespace kbsrc::dev {

constexpr int kTcSlices = 8;
constexpr int kTcAcc = kTcSlices + 1;  // accumulators d = i + j = 0..8: the triangle plus its first diagonal
constexpr int kTcMats = kTcSlices + 1; // matrix slices, the last one zero (it initialises accumulator 8)
constexpr int kTcRows = 128;          // MMA M: row vectors per stage
constexpr int kTcThreads = 512;       // four threads per row while slicing; four warpgroups while recombining
constexpr int kTcWaitLimit = 1 << 22; // mbarrier polls before a stage reports a timeout

// One radix of the split form: the sliced real DFT_R matrix (global memory, kTcMats * 2nh * 2kh bytes), stored per
// round (the output columns a round covers) with its slices one after the other, so that consecutive slices form
// one operand of kTcMats times the round's columns.
struct TcRadix {
    int R, kh, nh;
    const uint4* slices;
};

// A sub-FFT of N = a.R * b.R * c.R points (c.R == 1: two radices) on F sequences per CTA, every stage at most 128
// rows (F * N / R <= 128 for each radix R); ncols: TMEM columns to allocate. Inner twiddles, M = b.R * c.R:
// tw[k1 * M + m] = e^{-2 pi i m k1 / N}, then (three radices) tw[N + c1 * c.R + v] = e^{-2 pi i v c1 / M}.
struct TcSub {
    int N, F, ncols;
    TcRadix a, b, c;
    const double2* tw;
};
__host__ __device__ inline int tc_tw_count(const TcSub& s) { return s.c.R > 1 ? s.N + s.b.R * s.c.R : s.N; }

// Per-CTA shared memory of the split form after the two data plane pairs.
struct TcSmem {
    unsigned char* slices;  // kTcSlices * 128 * kpad_max
    unsigned char* bm_a;    // sliced DFT matrices
    unsigned char* bm_b;
    unsigned char* bm_c;
    double2* tw;            // tc_tw_count inner twiddles
    int* emax;              // row exponents (four per row while slicing)
    uint64_t* mbar;
    uint32_t* tmem_slot;
};

__host__ __device__ inline int tc_bm_bytes(const TcRadix& r) { return r.R > 1 ? kTcMats * (2 * r.nh) * (2 * r.kh) : 0; }
// Rounds of a stage: accumulators of all 2nh output columns at once when they fit TMEM's 512 columns, else the
// real and the imaginary outputs in turn.
__host__ __device__ inline int tc_rounds(int nh) { return kTcAcc * 2 * nh <= 512 ? 1 : 2; }
__host__ __device__ inline int tc_kpad(const TcSub& s) {
    const int k = s.a.kh > s.b.kh ? s.a.kh : s.b.kh;
    return 2 * (s.c.R > 1 && s.c.kh > k ? s.c.kh : k);
}
__host__ __device__ inline size_t tc_align(size_t v) { return (v + 127) & ~(size_t)127; }

// Shared bytes the split-form part of a CTA needs after its data planes.
__host__ __device__ inline size_t tc_smem_bytes(const TcSub& s) {
    return tc_align((size_t)kTcSlices * kTcRows * tc_kpad(s)) + tc_align(tc_bm_bytes(s.a)) + tc_align(tc_bm_bytes(s.b)) +
           tc_align(tc_bm_bytes(s.c)) + tc_align((size_t)tc_tw_count(s) * 16) + tc_align(4 * kTcRows * 4) + 128;
}

__device__ inline TcSmem tc_carve(unsigned char* p, const TcSub& s) {
    TcSmem m;
    m.slices = p;
    p += tc_align((size_t)kTcSlices * kTcRows * tc_kpad(s));
    m.bm_a = p;
    p += tc_align(tc_bm_bytes(s.a));
    m.bm_b = p;
    p += tc_align(tc_bm_bytes(s.b));
    m.bm_c = p;
    p += tc_align(tc_bm_bytes(s.c));
    m.tw = reinterpret_cast<double2*>(p);
    p += tc_align((size_t)tc_tw_count(s) * 16);
    m.emax = reinterpret_cast<int*>(p);
    p += tc_align(4 * kTcRows * 4);
    m.mbar = reinterpret_cast<uint64_t*>(p);
    m.tmem_slot = reinterpret_cast<uint32_t*>(p + 8);
    return m;
}

// TMEM allocation, the mbarrier, and the CTA's copies of the sliced matrices and inner twiddles. Ends with the
// CTA synchronised; returns the TMEM base address.
__device__ inline uint32_t tc_setup(const TcSmem& m, const TcSub& s) {
    if (threadIdx.x < 32) tmem_alloc(m.tmem_slot, (uint32_t)s.ncols);
    if (threadIdx.x == 0) mbar_init(m.mbar, 1);
    const int na = tc_bm_bytes(s.a) / 16, nb = tc_bm_bytes(s.b) / 16, nc = tc_bm_bytes(s.c) / 16, nt = tc_tw_count(s);
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

__device__ inline void tc_teardown(const TcSub& s, uint32_t tmem) {
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) tmem_dealloc(tmem, (uint32_t)s.ncols);
}

// Exponent bound of x: |x| < 2^tc_expo(x) (zero and subnormals: -1022)
__device__ __forceinline__ int tc_expo(double x) {
    const int ex = (int)((__double_as_longlong(x) >> 52) & 0x7ff);
    return ex ? ex - 1022 : -1022;
}
// floor(|x| * 2^(56 - e)) for |x| < 2^e: the 56-bit magnitude the slices are cut from
__device__ __forceinline__ unsigned long long tc_mag(double x, int e) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    int ex = (int)((b >> 52) & 0x7ff);
    unsigned long long m = b & ((1ull << 52) - 1);
    if (ex) m |= 1ull << 52;
    else ex = 1;
    const int sh = ex - 1019 - e;
    return sh >= 0 ? m << sh : (sh > -64 ? m >> -sh : 0ull);
}
// 2^k as a float64 for k in the normal range
__device__ __forceinline__ double tc_pow2(int k) {
    if (k < -1022 || k > 1023) return ldexp(1.0, k);
    return __longlong_as_double((long long)(k + 1023) << 52);
}

// One contraction stage: `nrows` rows of R complex values, load(row, j, part) -> double (part 0 the real, 1 the
// imaginary part); store(row, k, part, y) for output k. `phase` counts the mbarrier phases completed so far.
template <class Load, class Store>
__device__ inline void tc_stage(const TcRadix& rad, int nrows, const TcSmem& m, const unsigned char* bmat,
                                uint32_t tmem, uint32_t& phase, int* err, Load load, Store store) {
    const int R = rad.R, kh = rad.kh, nh = rad.nh, kpad = 2 * kh, npad = 2 * nh;
    const int t = threadIdx.x;
    {  // slicing: four threads per row, one per 16-column chunk of a K half (real, imaginary parts); the row
       // exponent through smem
        const int row = t & (kTcRows - 1), part = (t >> 7) & 1, c = 16 * (t >> 8);
        double vals[16];
        int e = -1022;
#pragma unroll
        for (int q = 0; q < 16; q++) {
            vals[q] = (row < nrows && c + q < R) ? load(row, c + q, part) : 0.0;
            e = max(e, tc_expo(vals[q]));
        }
        m.emax[(t >> 7) * kTcRows + row] = e;
        __syncthreads();
        e = max(max(m.emax[row], m.emax[kTcRows + row]), max(m.emax[2 * kTcRows + row], m.emax[3 * kTcRows + row]));
        if (row < nrows && c < kh) {
            unsigned long long mag[16];
            unsigned neg = 0;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                mag[q] = tc_mag(vals[q], e);
                if (__double_as_longlong(vals[q]) < 0) neg |= 1u << q;
            }
            uint32_t nm[4];  // byte k of nm[g]: 0xff where value 4g + k is negative
#pragma unroll
            for (int g = 0; g < 4; g++)
                nm[g] = ((neg >> (4 * g)) & 1 ? 0xffu : 0u) | ((neg >> (4 * g + 1)) & 1 ? 0xff00u : 0u) |
                        ((neg >> (4 * g + 2)) & 1 ? 0xff0000u : 0u) | ((neg >> (4 * g + 3)) & 1 ? 0xff000000u : 0u);
#pragma unroll
            for (int i = 0; i < kTcSlices; i++) {
                uint32_t w[4];
#pragma unroll
                for (int g = 0; g < 4; g++) {
                    uint32_t v = 0;  // 7-bit field i of value 4g + k, placed in byte k by one constant shift
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const int sh = 49 - 7 * i - 8 * k;
                        const unsigned long long x = sh >= 0 ? mag[4 * g + k] >> sh : mag[4 * g + k] << -sh;
                        v |= (uint32_t)x & (0x7fu << (8 * k));
                    }
                    // the negative values' bytes negated, four at once: -b = (0x80 - b) ^ 0x80 for b in [0, 127]
                    const uint32_t nv = (0x80808080u - v) ^ 0x80808080u;
                    w[g] = v ^ ((v ^ nv) & nm[g]);
                }
                *reinterpret_cast<uint4*>(m.slices + i * kTcRows * kpad + umma_off(row, part * kh + c, kpad)) =
                    make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        __syncthreads();
        if (t < kTcRows) m.emax[row] = e;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // Accumulators d = 0..kTcAcc-1 of nr columns each (tc_rounds).
    const int rounds = tc_rounds(nh), nr = npad / rounds;
    const uint32_t sbo = 8 * kpad;
    for (int rd = 0; rd < rounds; rd++) {
        if (t == 0) {  // the product triangle i + j <= kTcAcc - 1, accumulator d collecting every i + j = d: data
                       // slice i times matrix slices 0.. side by side lands on accumulators i.., up to 256 columns
                       // per MMA; i = 0 (with the zero slice) initialises every accumulator
            const uint32_t sa = smem_u32(m.slices), sb = smem_u32(bmat) + rd * kTcMats * nr * kpad;
            const int bpc = 256 / nr;
            for (int i = 0; i < kTcSlices; i++)
                for (int d0 = i; d0 < kTcAcc; d0 += bpc) {
                    const int nb = min(bpc, kTcAcc - d0);
                    const uint32_t idesc = umma_idesc_s8(kTcRows, nb * nr);
                    for (int ks = 0; ks < kpad / 32; ks++)
                        umma_s8(tmem + d0 * nr, umma_desc(sa + i * kTcRows * kpad + 256 * ks, 128, sbo),
                                umma_desc(sb + (d0 - i) * nr * kpad + 256 * ks, 128, sbo), idesc,
                                (i || ks) ? 1u : 0u);
                }
            umma_commit(m.mbar);
        }
        bool ok = mbar_wait(m.mbar, phase & 1u, kTcWaitLimit);
        phase++;
        ok = __all_sync(0xffffffffu, ok);  // the TMEM loads below are warp-collective
        tc_fence_after();
        if (!ok) {
            if ((t & 31) == 0) atomicExch(err, 1);
        } else {  // recombination: warp w reads TMEM lanes 32 (w % 4) ..; warpgroup w / 4 takes every fourth group
                  // of 8 columns
            const int warp = t >> 5, lane0 = 32 * (warp & 3), row = lane0 + (t & 31);
            const int e = row < nrows ? m.emax[row] : 0;
            const double s1 = tc_pow2(e - 34), s2 = tc_pow2(e - 69);
            const uint32_t lane_addr = tmem + ((uint32_t)lane0 << 16);
            for (int c0 = 8 * (warp >> 2); c0 < nr; c0 += 32) {
                long long hi[8], lo[8];
                int32_t v[5][8];
#pragma unroll
                for (int d = 0; d < 4; d++) tmem_ld8(lane_addr + d * nr + c0, v[d]);
                tmem_wait_ld();
#pragma unroll
                for (int q = 0; q < 8; q++)
                    hi[q] = (((long long)v[0][q] * 128 + v[1][q]) * 128 + v[2][q]) * 128 + v[3][q];
#pragma unroll
                for (int d = 0; d < 5; d++) tmem_ld8(lane_addr + (d + 4) * nr + c0, v[d]);
                tmem_wait_ld();
#pragma unroll
                for (int q = 0; q < 8; q++)
                    lo[q] = ((((long long)v[0][q] * 128 + v[1][q]) * 128 + v[2][q]) * 128 + v[3][q]) * 128 + v[4][q];
                if (row < nrows) {
#pragma unroll
                    for (int q = 0; q < 8; q++) {
                        const int n = rd * nr + c0 + q, part = n >= nh, k = n - part * nh;
                        if (k < R)
                            store(row, k, part, __dadd_rn(__dmul_rn(__ll2double_rn(hi[q]), s1),
                                                          __dmul_rn(__ll2double_rn(lo[q]), s2)));
                    }
                }
            }
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
}

// Sub-FFT of N = Ra * Rb points on F sequences held in X (element j of sequence f at j * F + f), Cooley-Tukey
// with n = Rb j + m, k = k1 + Ra k2: stage A (DFT_Ra over j for each m), the twiddle w_N^{m k1}, stage B (DFT_Rb
// over m for each k1). Y is scratch; the result is in X in natural order. `phase`: mbarrier phases completed so
// far by this CTA.
__device__ inline void tc_subfft3(const TcSub& s, const Planes<ArF64>& X, const Planes<ArF64>& Y, const TcSmem& m,
                                  uint32_t tmem, uint32_t& phase, int* err);

__device__ inline void tc_subfft(const TcSub& s, const Planes<ArF64>& X, const Planes<ArF64>& Y, const TcSmem& m,
                                 uint32_t tmem, uint32_t& phase, int* err) {
    if (s.c.R > 1) {
        tc_subfft3(s, X, Y, m, tmem, phase, err);
        return;
    }
    const int F = s.F, Ra = s.a.R, Rb = s.b.R;
    tc_stage(s.a, Rb * F, m, m.bm_a, tmem, phase, err,
             [&](int r, int j, int part) {
                 const int mm = r / F, f = r - mm * F, i = (Rb * j + mm) * F + f;
                 return part ? X.im[i] : X.re[i];
             },
             [&](int r, int k1, int part, double y) {
                 const int mm = r / F, f = r - mm * F, i = (k1 * Rb + mm) * F + f;
                 (part ? Y.im : Y.re)[i] = y;
             });
    for (int e = threadIdx.x; e < s.N * F; e += blockDim.x) {
        const double2 w = m.tw[e / F];
        const double re = Y.re[e], im = Y.im[e];
        Y.re[e] = __dsub_rn(__dmul_rn(re, w.x), __dmul_rn(im, w.y));
        Y.im[e] = __dadd_rn(__dmul_rn(re, w.y), __dmul_rn(im, w.x));
    }
    __syncthreads();
    tc_stage(s.b, Ra * F, m, m.bm_b, tmem, phase, err,
             [&](int r, int mm, int part) {
                 const int k1 = r / F, f = r - k1 * F, i = (k1 * Rb + mm) * F + f;
                 return part ? Y.im[i] : Y.re[i];
             },
             [&](int r, int k2, int part, double y) {
                 const int k1 = r / F, f = r - k1 * F, i = (k1 + Ra * k2) * F + f;
                 (part ? X.im : X.re)[i] = y;
             });
}

// In-place complex multiply of the N*F values of P by tw[(e / F) % period] (e the plane index)
__device__ inline void tc_twiddle(const Planes<ArF64>& P, const double2* tw, int n, int F, int period) {
    for (int e = threadIdx.x; e < n * F; e += blockDim.x) {
        const double2 w = tw[(e / F) % period];
        const double re = P.re[e], im = P.im[e];
        P.re[e] = __dsub_rn(__dmul_rn(re, w.x), __dmul_rn(im, w.y));
        P.im[e] = __dadd_rn(__dmul_rn(re, w.y), __dmul_rn(im, w.x));
    }
    __syncthreads();
}

// Sub-FFT of N = Ra * M points, M = Rb * Rc: n = M j + m, k = k1 + Ra k2, then within each k1 the M-point
// transform over m = Rc u + v, k2 = c1 + Rb c2. Stage A (DFT_Ra over j for each m, X -> Y), twiddle w_N^{m k1},
// stage B (DFT_Rb over u for each (k1, v), Y -> X in the same slots), twiddle w_M^{v c1}, stage C (DFT_Rc over v
// for each (k1, c1), X -> X in natural order: every value of a stage is read before any is written).
__device__ inline void tc_subfft3(const TcSub& s, const Planes<ArF64>& X, const Planes<ArF64>& Y, const TcSmem& m,
                                  uint32_t tmem, uint32_t& phase, int* err) {
    const int F = s.F, Ra = s.a.R, Rb = s.b.R, Rc = s.c.R, M = Rb * Rc;
    tc_stage(s.a, M * F, m, m.bm_a, tmem, phase, err,
             [&](int r, int j, int part) {
                 const int mm = r / F, f = r - mm * F, i = (M * j + mm) * F + f;
                 return part ? X.im[i] : X.re[i];
             },
             [&](int r, int k1, int part, double y) {
                 const int mm = r / F, f = r - mm * F, i = (k1 * M + mm) * F + f;
                 (part ? Y.im : Y.re)[i] = y;
             });
    tc_twiddle(Y, m.tw, s.N, F, s.N);
    tc_stage(s.b, Ra * Rc * F, m, m.bm_b, tmem, phase, err,
             [&](int r, int u, int part) {
                 const int q = r / F, f = r - q * F, k1 = q / Rc, v = q - k1 * Rc, i = (k1 * M + Rc * u + v) * F + f;
                 return part ? Y.im[i] : Y.re[i];
             },
             [&](int r, int c1, int part, double y) {
                 const int q = r / F, f = r - q * F, k1 = q / Rc, v = q - k1 * Rc, i = (k1 * M + Rc * c1 + v) * F + f;
                 (part ? X.im : X.re)[i] = y;
             });
    tc_twiddle(X, m.tw + s.N, s.N, F, M);
    tc_stage(s.c, Ra * Rb * F, m, m.bm_c, tmem, phase, err,
             [&](int r, int v, int part) {
                 const int q = r / F, f = r - q * F, k1 = q / Rb, c1 = q - k1 * Rb, i = (k1 * M + Rc * c1 + v) * F + f;
                 return part ? X.im[i] : X.re[i];
             },
             [&](int r, int c2, int part, double y) {
                 const int q = r / F, f = r - q * F, k1 = q / Rb, c1 = q - k1 * Rb, i = (k1 + Ra * (c1 + Rb * c2)) * F + f;
                 (part ? X.im : X.re)[i] = y;
             });
}

}  // namespace kbsrc::dev
