// Mixed-radix Stockham DFT passes in shared memory.
//
// A CTA transforms F independent sequences of length n at once. Element j of sequence f lives at
// smem[j*F + f], so consecutive threads (consecutive f) touch consecutive addresses. Each stage walks its
// (f, butterfly) pairs in a block-stride loop and ping-pongs between two buffers.
//
// The butterflies and the stage/twiddle indexing are the reference's (HongYue1/KBSRC src/dsp/fft.hpp:62-151):
// radix order 4s, 2s, then 3, 5, 7; stage twiddles skipped for p == 0; the odd-radix sums accumulated for
// t = 1..H in that order. Rounding is part of the output definition, so none of this may be reordered.
#pragma once
#include "dd.cuh"

namespace kbsrc::dev {

constexpr int kMaxStages = 16;

// Division by a divisor that is fixed for a loop, through its rounded-up reciprocal m = ceil(2^32 / d) =
// floor((2^32 - 1) / d) + 1: (n * m) >> 32 is floor(n / d) whenever n * d < 2^32, which every index range of the
// passes satisfies (n < 2^22, d < 2^12). One division sets it up; each use is one 64-bit multiply.
struct FastDiv {
    unsigned d;
    unsigned long long m;
};
__host__ __device__ __forceinline__ FastDiv fast_div(unsigned d) {
    return FastDiv{d, (unsigned long long)(0xFFFFFFFFu / d) + 1ull};
}
__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv& f) {
    return (unsigned)(((unsigned long long)n * f.m) >> 32);
}

struct Stage {
    int r, m, s;  // radix, butterflies per (p) group count m = n_left/r, output stride s
    int tw;       // offset of this stage's twiddles (complex table entries), laid out [p*(r-1) + u-1]
};
struct SubPlan {
    int n, nst;
    int tw0, twn;  // this plan's twiddles: entries [tw0, tw0 + twn) of the table
    Stage st[kMaxStages];
};

// cos / sin of 2 pi k / r for r = 3, 5, 7 (rows 0, 1, 2)
template <class W>
struct OddRoots {
    W c[3][7], s[3][7];
};

template <class W>
__device__ __forceinline__ cx<W> ld_tw(const cx<W>* p);
template <>
__device__ __forceinline__ cx<double> ld_tw<double>(const cx<double>* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    return cx<double>{a.x, a.y};
}
template <>
__device__ __forceinline__ cx<dd> ld_tw<dd>(const cx<dd>* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldg(q), b = __ldg(q + 1);
    return cx<dd>{dd{a.x, a.y}, dd{b.x, b.y}};
}

template <>
__device__ __forceinline__ cx<x80> ld_tw<x80>(const cx<x80>* p) {
    const longlong2* q = reinterpret_cast<const longlong2*>(p);
    const longlong2 a = __ldg(q), b = __ldg(q + 1);
    return cx<x80>{x80{(unsigned long long)a.x, (int)a.y, 0}, x80{(unsigned long long)b.x, (int)b.y, 0}};
}

// A pass's stage twiddles: entry i is table entry sp.tw0 + i, read from the CTA's shared-memory copy (double-double
// and extended by default: copied once per CTA) or, with GLOBAL, straight from the global table through the
// read-only path (float64 always: a CTA's work is too short to amortise the copy; the wide types when the launch
// shape says so, which leaves the shared memory to the sequences). A compile-time choice, so neither form pays for
// the other.
template <class Ar, bool GLOBAL = !Ar::kWide>
struct Twiddles {
    const CxW<Ar>* p;  // GLOBAL: the table at entry sp.tw0; else the shared copy
    __device__ __forceinline__ CxW<Ar> at(int i) const {
        if constexpr (GLOBAL) return ld_tw(p + i);
        else return p[i];
    }
};

// Shared-memory view of F sequences in split planes: element i = j*F + f (sample j of sequence f) has its real
// part at re[i] and its imaginary part at im[i], so consecutive threads (consecutive f) read consecutive
// 16-byte (dd) or 8-byte (f64) words of each plane without bank conflicts.
template <class Ar>
struct Planes {
    typename Ar::R* re;
    typename Ar::R* im;
    __device__ __forceinline__ CxR<Ar> ld(int i) const { return CxR<Ar>{re[i], im[i]}; }
    __device__ __forceinline__ void st(int i, const CxR<Ar>& v) const {
        re[i] = v.re;
        im[i] = v.im;
    }
};

// Carves two plane pairs of nF values each from the start of shared memory; returns the first byte after them.
template <class Ar>
__device__ __forceinline__ unsigned char* carve(unsigned char* smem, int nF, Planes<Ar>& A, Planes<Ar>& B) {
    using R = typename Ar::R;
    R* p = reinterpret_cast<R*>(smem);
    A = Planes<Ar>{p, p + nF};
    B = Planes<Ar>{p + 2 * nF, p + 3 * nF};
    return reinterpret_cast<unsigned char*>(p + 4 * nF);
}

template <class Ar, class TW>
__device__ __forceinline__ void bfly2(const Planes<Ar>& a, int ia, int sin, const Planes<Ar>& b, int ib, int sout,
                                      const TW& tw, int tk, bool p0) {
    const CxR<Ar> a0 = a.ld(ia), a1 = a.ld(ia + sin);
    b.st(ib, c_add<Ar>(a0, a1));
    b.st(ib + sout, p0 ? c_sub<Ar>(a0, a1) : c_mulw<Ar>(c_sub<Ar>(a0, a1), tw.at(tk)));
}

template <class Ar, class TW>
__device__ __forceinline__ void bfly4(const Planes<Ar>& a, int ia, int sin, const Planes<Ar>& b, int ib, int sout,
                                      const TW& tw, int tk, bool p0) {
    using C = CxR<Ar>;
    const C a0 = a.ld(ia), a1 = a.ld(ia + sin), a2 = a.ld(ia + 2 * sin), a3 = a.ld(ia + 3 * sin);
    const C t0 = c_add<Ar>(a0, a2), t1 = c_sub<Ar>(a0, a2), t2 = c_add<Ar>(a1, a3);
    const C t3 = c_mul_mi<Ar>(c_sub<Ar>(a1, a3));
    b.st(ib, c_add<Ar>(t0, t2));
    if (p0) {
        b.st(ib + sout, c_add<Ar>(t1, t3));
        b.st(ib + 2 * sout, c_sub<Ar>(t0, t2));
        b.st(ib + 3 * sout, c_sub<Ar>(t1, t3));
    } else {
        b.st(ib + sout, c_mulw<Ar>(c_add<Ar>(t1, t3), tw.at(tk)));
        b.st(ib + 2 * sout, c_mulw<Ar>(c_sub<Ar>(t0, t2), tw.at(tk + 1)));
        b.st(ib + 3 * sout, c_mulw<Ar>(c_sub<Ar>(t1, t3), tw.at(tk + 2)));
    }
}

// Odd radix R: x_u = a0 + sum_t S_t cos(2pi tu/R) -/+ i sum_t D_t sin(2pi tu/R) (fft.hpp:62-84)
template <class Ar, int R, class TW>
__device__ __forceinline__ void bfly_odd(const Planes<Ar>& a, int ia, int sin, const Planes<Ar>& b, int ib,
                                         int sout, const TW& tw, int tk, bool p0,
                                         const typename Ar::W* cr, const typename Ar::W* sr) {
    using C = CxR<Ar>;
    constexpr int H = (R - 1) / 2;
    const C a0 = a.ld(ia);
    C S[H], Df[H];
#pragma unroll
    for (int t = 1; t <= H; t++) {
        const C x = a.ld(ia + t * sin), y = a.ld(ia + (R - t) * sin);
        S[t - 1] = c_add<Ar>(x, y);
        Df[t - 1] = c_sub<Ar>(x, y);
    }
    C sum = a0;
#pragma unroll
    for (int t = 0; t < H; t++) sum = c_add<Ar>(sum, S[t]);
    b.st(ib, sum);
#pragma unroll
    for (int u = 1; u <= H; u++) {
        C A = a0, B = {Ar::zero(), Ar::zero()};
#pragma unroll
        for (int t = 1; t <= H; t++) {
            const int m = (t * u) % R;
            const typename Ar::R c = Ar::from_w(cr[m]), sn = Ar::from_w(sr[m]);
            A = {Ar::add(A.re, Ar::mul(S[t - 1].re, c)), Ar::add(A.im, Ar::mul(S[t - 1].im, c))};
            B = {Ar::add(B.re, Ar::mul(Df[t - 1].re, sn)), Ar::add(B.im, Ar::mul(Df[t - 1].im, sn))};
        }
        const C xu = {Ar::add(A.re, B.im), Ar::sub(A.im, B.re)};
        const C xr = {Ar::sub(A.re, B.im), Ar::add(A.im, B.re)};
        if (p0) {
            b.st(ib + u * sout, xu);
            b.st(ib + (R - u) * sout, xr);
        } else {
            b.st(ib + u * sout, c_mulw<Ar>(xu, tw.at(tk + u - 1)));
            b.st(ib + (R - u) * sout, c_mulw<Ar>(xr, tw.at(tk + R - u - 1)));
        }
    }
}

// Twiddles a pass reads: for the wide types unless GLOBAL, the plan's stage twiddles copied to shared memory (tws,
// sp.twn entries; the caller synchronises before use); otherwise the global table itself.
template <class Ar, bool GLOBAL = !Ar::kWide>
__device__ __forceinline__ Twiddles<Ar, GLOBAL> stage_twiddles(const SubPlan& sp, const CxW<Ar>* __restrict__ tw,
                                                               CxW<Ar>* tws) {
    if constexpr (GLOBAL) {
        return Twiddles<Ar, GLOBAL>{tw + sp.tw0};
    } else {
        for (int i = threadIdx.x; i < sp.twn; i += blockDim.x) tws[i] = ld_tw(tw + sp.tw0 + i);
        return Twiddles<Ar, GLOBAL>{tws};
    }
}

// Runs every stage of `sp` on F sequences held in `a` (element j of sequence f at j*F + f); `b` is the other
// plane pair; `tws` the plan's twiddles from stage_twiddles (entry 0 = table entry sp.tw0). Returns the planes
// that hold the result. Ends with the CTA synchronised.
template <class Ar, class TW>
__device__ __forceinline__ Planes<Ar> stockham(const SubPlan& sp, Planes<Ar> a, Planes<Ar> b, int F,
                                               const TW& tws, const OddRoots<typename Ar::W>& odd) {
    for (int g = 0; g < sp.nst; g++) {
        const int r = sp.st[g].r, m = sp.st[g].m, s = sp.st[g].s;
        const int twg = sp.st[g].tw - sp.tw0;
        const int total = m * s * F, sin = s * m * F, sout = s * F;
        const FastDiv dF = fast_div(F), ds = fast_div(s);
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            const int bf = (int)fdiv(idx, dF), f = idx - bf * F, p = (int)fdiv(bf, ds), q = bf - p * s;
            const int ia = (s * p + q) * F + f, ib = (s * r * p + q) * F + f;
            const int t = twg + p * (r - 1);
            const bool p0 = p == 0;
            if (r == 4) bfly4<Ar, TW>(a, ia, sin, b, ib, sout, tws, t, p0);
            else if (r == 2) bfly2<Ar, TW>(a, ia, sin, b, ib, sout, tws, t, p0);
            else if (r == 3) bfly_odd<Ar, 3, TW>(a, ia, sin, b, ib, sout, tws, t, p0, odd.c[0], odd.s[0]);
            else if (r == 5) bfly_odd<Ar, 5, TW>(a, ia, sin, b, ib, sout, tws, t, p0, odd.c[1], odd.s[1]);
            else bfly_odd<Ar, 7, TW>(a, ia, sin, b, ib, sout, tws, t, p0, odd.c[2], odd.s[2]);
        }
        __syncthreads();
        const Planes<Ar> t = a;
        a = b;
        b = t;
    }
    return a;
}

}  // namespace kbsrc::dev
