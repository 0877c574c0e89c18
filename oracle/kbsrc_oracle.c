/*
 * TEST INFRASTRUCTURE ONLY - the oracle. A plain-C, single-threaded CPU restatement of KBSRC 1.3.0's
 * DFT-domain rational resampling path, written from the reference's behaviour so that tests can check the
 * GPU product bit for bit. Only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg) may load
 * it, and only as the checker. Nothing in kbsrc_b200/ links or calls it.
 *
 * Parity pins: tests/test_oracle.py checks it against the reference's own pinned SHA-256 values and samples
 * (tests/test_engines.py:76-88 of the reference) and against the reference built from source
 * (oracle/_ref, tests/golden/).
 *
 * Every operation below keeps the reference's IEEE operation order; -ffp-contract=off is mandatory
 * (the reference's CMakeLists.txt:27-31 carries the same flag). The only fused multiply-add is the exact
 * product error (src/dsp/double_double.hpp:20-22), computed with libm fma(), which is correctly rounded.
 *
 * Reference files cited as path:line of HongYue1/KBSRC.
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------------------ */
/* double-double arithmetic: src/dsp/double_double.hpp:59-135, src/dsp/simd.hpp:44-66                       */
/* ------------------------------------------------------------------------------------------------------ */
typedef struct { double hi, lo; } dd;
typedef struct { dd re, im; } cdd;

static inline dd mk(double h, double l) { dd r; r.hi = h; r.lo = l; return r; }
static inline dd D(double h) { return mk(h, 0.0); }
/* quick two-sum (double_double.hpp:65) */
static inline dd qts(double a, double b) { double s = a + b; return mk(s, b - (s - a)); }
/* two-sum (double_double.hpp:66) */
static inline dd ts(double a, double b) {
    double s = a + b, bb = s - a;
    return mk(s, (a - (s - bb)) + (b - bb));
}
/* accurate add: two two-sums (double_double.hpp:67-70); also the reconstruction add (fft.hpp:318-337) */
static inline dd dadd(dd a, dd b) {
    dd s = ts(a.hi, b.hi), t = ts(a.lo, b.lo);
    s.lo = s.lo + t.hi;
    s = qts(s.hi, s.lo);
    s.lo = s.lo + t.lo;
    return qts(s.hi, s.lo);
}
static inline dd dneg(dd a) { return mk(-a.hi, -a.lo); }
static inline dd dsub(dd a, dd b) { return dadd(a, dneg(b)); }
/* short ("sloppy") add of the 4-lane type (simd.hpp:44-49 AVX2, :88-94 generic) */
static inline dd sadd(dd a, dd b) {
    double s = a.hi + b.hi, bb = s - a.hi;
    double e = (a.hi - (s - bb)) + (b.hi - bb);
    e = e + (a.lo + b.lo);
    double t = s + e;
    return mk(t, e - (t - s));
}
/* product (double_double.hpp:73-76, simd.hpp:55-59) */
static inline dd dmul(dd a, dd b) {
    double p = a.hi * b.hi, e = fma(a.hi, b.hi, -p);
    e = e + (a.hi * b.lo + a.lo * b.hi);
    return qts(p, e);
}
/* dd times double (double_double.hpp:77-79) */
static inline dd dmuld(dd a, double b) {
    double p = a.hi * b, e = fma(a.hi, b, -p);
    e = e + a.lo * b;
    return qts(p, e);
}
/* dd / double (double_double.hpp:80-84) */
static dd ddivd(dd a, double b) {
    double q1 = a.hi / b;
    dd r = dsub(a, dmuld(D(b), q1));
    double q2 = r.hi / b;
    r = dsub(r, dmuld(D(b), q2));
    double q3 = r.hi / b;
    return dadd(qts(q1, q2), D(q3));
}
/* dd / dd (double_double.hpp:88-92) */
static dd ddiv(dd a, dd b) {
    double q1 = a.hi / b.hi;
    dd r = dsub(a, dmuld(b, q1));
    double q2 = r.hi / b.hi;
    r = dsub(r, dmuld(b, q2));
    double q3 = r.hi / b.hi;
    return dadd(qts(q1, q2), D(q3));
}
/* double_double.hpp:94-98 */
static dd dsqrt(dd a) {
    if (a.hi <= 0) return D(0.0);
    double y = sqrt(a.hi);
    dd r = dsub(a, dmuld(D(y), y));
    return qts(y, r.hi / (2 * y));
}
/* modified Bessel I0 (double_double.hpp:100-107) */
static dd di0(dd x) {
    dd q = ddivd(dmul(x, x), 4.0), t = D(1.0), s = D(1.0);
    for (int k = 1; k < 2000; k++) {
        t = ddivd(dmul(t, q), (double)k * (double)k);
        s = dadd(s, t);
        if (t.hi < s.hi * 1e-34) break;
    }
    return s;
}
static const double PI_HI = 3.141592653589793116e+00, PI_LO = 1.224646799147353207e-16;
/* double_double.hpp:113-121 */
static void sincos_small(dd x, dd* c, dd* s) {
    dd x2 = dmul(x, x), t = x, ss = x, cc = D(1.0), tc = D(1.0);
    for (int k = 1; k < 40; k++) {
        tc = ddivd(dneg(dmul(tc, x2)), (double)((2 * k - 1) * (2 * k)));
        cc = dadd(cc, tc);
        t = ddivd(dneg(dmul(t, x2)), (double)((2 * k) * (2 * k + 1)));
        ss = dadd(ss, t);
        if (fabs(t.hi) < 1e-40 && fabs(tc.hi) < 1e-40) break;
    }
    *c = cc;
    *s = ss;
}
/* e^{+2 pi i k/N} with exact octant reduction (double_double.hpp:122-135) */
static void dcis(long long k, long long N, dd* c, dd* s) {
    k %= N;
    if (k < 0) k += N;
    long long m = 8 * k, oct = m / N, rem = m - oct * N;
    int odd = (int)(oct & 1);
    long long j = oct / 2;
    dd phi = ddivd(dmuld(mk(PI_HI / 4, PI_LO / 4), (double)(odd ? (N - rem) : rem)), (double)N);
    dd cc, sn;
    sincos_small(phi, &cc, &sn);
    if (odd) { sn = dneg(sn); j += 1; }
    switch (j & 3) {
        case 0: *c = cc; *s = sn; break;
        case 1: *c = dneg(sn); *s = cc; break;
        case 2: *c = dneg(cc); *s = dneg(sn); break;
        default: *c = sn; *s = dneg(cc); break;
    }
}

/* twiddle table cis(2 pi k/N) from two short tables (fft.hpp:29-43) */
typedef struct { long long N, B; dd *ac, *as, *bc, *bs; } CisTab;
static void cis_init(CisTab* t, long long n) {
    t->N = n;
    t->B = (long long)ceil(sqrt((double)n));
    long long J = n / t->B + 1;
    t->ac = malloc(sizeof(dd) * J); t->as = malloc(sizeof(dd) * J);
    t->bc = malloc(sizeof(dd) * t->B); t->bs = malloc(sizeof(dd) * t->B);
    for (long long j = 0; j < J; j++) dcis(j * t->B, n, &t->ac[j], &t->as[j]);
    for (long long l = 0; l < t->B; l++) dcis(l, n, &t->bc[l], &t->bs[l]);
}
static void cis_free(CisTab* t) { free(t->ac); free(t->as); free(t->bc); free(t->bs); }
static void cis_get(const CisTab* t, long long k, dd* c, dd* s) {
    k %= t->N;
    if (k < 0) k += t->N;
    long long j = k / t->B, l = k % t->B;
    if (l == 0) { *c = t->ac[j]; *s = t->as[j]; return; }
    if (j == 0) { *c = t->bc[l]; *s = t->bs[l]; return; }
    *c = dsub(dmul(t->ac[j], t->bc[l]), dmul(t->as[j], t->bs[l]));
    *s = dadd(dmul(t->ac[j], t->bs[l]), dmul(t->as[j], t->bc[l]));
}

/* ------------------------------------------------------------------------------------------------------ */
/* arithmetic flavours. Values are always held as dd; the f64 flavour uses .hi only (fft.hpp:16 from_dd).   */
/* ------------------------------------------------------------------------------------------------------ */
enum { A_F64 = 0, A_DDS = 1 /* short add, 4-lane DD4 */, A_DDA = 2 /* accurate scalar dd */ };

static inline dd a_add(int A, dd a, dd b) {
    if (A == A_F64) return D(a.hi + b.hi);
    return A == A_DDS ? sadd(a, b) : dadd(a, b);
}
static inline dd a_sub(int A, dd a, dd b) {
    if (A == A_F64) return D(a.hi - b.hi);
    return A == A_DDS ? sadd(a, dneg(b)) : dadd(a, dneg(b));
}
static inline dd a_mul(int A, dd a, dd b) {
    if (A == A_F64) return D(a.hi * b.hi);
    return dmul(a, b);
}
static inline cdd cx(dd re, dd im) { cdd r; r.re = re; r.im = im; return r; }
static inline cdd c_add(int A, cdd a, cdd b) { return cx(a_add(A, a.re, b.re), a_add(A, a.im, b.im)); }
static inline cdd c_sub(int A, cdd a, cdd b) { return cx(a_sub(A, a.re, b.re), a_sub(A, a.im, b.im)); }
static inline cdd c_conj(cdd a) { return cx(a.re, dneg(a.im)); }
static inline cdd c_mi(cdd a) { return cx(a.im, dneg(a.re)); } /* a * (-i), fft.hpp:52 */
/* complex product {a.re b.re - a.im b.im, a.re b.im + a.im b.re} (fft.hpp:46-51) */
static inline cdd c_mul(int A, cdd a, cdd b) {
    return cx(a_sub(A, a_mul(A, a.re, b.re), a_mul(A, a.im, b.im)),
              a_add(A, a_mul(A, a.re, b.im), a_mul(A, a.im, b.re)));
}
static inline cdd c_scale(int A, cdd a, dd h) { return cx(a_mul(A, a.re, h), a_mul(A, a.im, h)); }

/* ------------------------------------------------------------------------------------------------------ */
/* Stockham mixed-radix complex DFT, exponent sign -1 (fft.hpp:62-151)                                       */
/* ------------------------------------------------------------------------------------------------------ */
#define MAXST 64
typedef struct {
    int n, ns;
    int r[MAXST], m[MAXST], s[MAXST];
    cdd* tw[MAXST];
    dd cr[3][7], sr[3][7];
} SPlan;

static int sfft_init(SPlan* P, int n) {
    P->n = n;
    P->ns = 0;
    int t = n;
    while (t % 4 == 0) { P->r[P->ns++] = 4; t /= 4; }
    while (t % 2 == 0) { P->r[P->ns++] = 2; t /= 2; }
    static const int odd[3] = {3, 5, 7};
    for (int i = 0; i < 3; i++)
        while (t % odd[i] == 0) { P->r[P->ns++] = odd[i]; t /= odd[i]; }
    if (t != 1) return -1;
    CisTab ct;
    cis_init(&ct, n);
    int rem = n, s = 1;
    for (int g = 0; g < P->ns; g++) {
        int r = P->r[g];
        P->m[g] = rem / r;
        P->s[g] = s;
        P->tw[g] = malloc(sizeof(cdd) * (size_t)P->m[g] * (r - 1) + 1);
        for (int p = 0; p < P->m[g]; p++)
            for (int u = 1; u < r; u++) {
                dd c, sn;
                cis_get(&ct, -(long long)s * p * u, &c, &sn);
                P->tw[g][(size_t)p * (r - 1) + u - 1] = cx(c, sn);
            }
        rem /= r;
        s *= r;
    }
    cis_free(&ct);
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < odd[i]; k++) dcis(k, odd[i], &P->cr[i][k], &P->sr[i][k]);
    return 0;
}
static void sfft_free(SPlan* P) {
    for (int g = 0; g < P->ns; g++) free(P->tw[g]);
    P->ns = 0;
}

/* odd radix butterfly (fft.hpp:62-84) */
static void odd_bfly(int A, int R, const cdd* src, size_t sm, cdd* dst, int s, int q, const dd* cr, const dd* sr,
                     const cdd* tw, int p0) {
    const int H = (R - 1) / 2;
    cdd a0 = src[q], S[3], Df[3];
    for (int t = 1; t <= H; t++) {
        cdd x = src[q + t * sm], y = src[q + (R - t) * sm];
        S[t - 1] = c_add(A, x, y);
        Df[t - 1] = c_sub(A, x, y);
    }
    cdd sum = a0;
    for (int t = 0; t < H; t++) sum = c_add(A, sum, S[t]);
    dst[q] = sum;
    for (int u = 1; u <= H; u++) {
        cdd Aa = a0, B = cx(D(0.0), D(0.0));
        for (int t = 1; t <= H; t++) {
            int m = (t * u) % R;
            dd c = cr[m], sn = sr[m];
            Aa = cx(a_add(A, Aa.re, a_mul(A, S[t - 1].re, c)), a_add(A, Aa.im, a_mul(A, S[t - 1].im, c)));
            B = cx(a_add(A, B.re, a_mul(A, Df[t - 1].re, sn)), a_add(A, B.im, a_mul(A, Df[t - 1].im, sn)));
        }
        cdd xu = cx(a_add(A, Aa.re, B.im), a_sub(A, Aa.im, B.re));
        cdd xr = cx(a_sub(A, Aa.re, B.im), a_add(A, Aa.im, B.re));
        if (p0) {
            dst[q + u * s] = xu;
            dst[q + (R - u) * s] = xr;
        } else {
            dst[q + u * s] = c_mul(A, xu, tw[u - 1]);
            dst[q + (R - u) * s] = c_mul(A, xr, tw[R - u - 1]);
        }
    }
}

static cdd* sfft_run(const SPlan* P, int A, cdd* x, cdd* y) {
    cdd *a = x, *b = y;
    for (int g = 0; g < P->ns; g++) {
        const int r = P->r[g], m = P->m[g], s = P->s[g];
        for (int p = 0; p < m; p++) {
            const cdd* tw = P->tw[g] + (size_t)p * (r - 1);
            const cdd* src = a + (size_t)s * p;
            cdd* dst = b + (size_t)s * r * p;
            const size_t sm = (size_t)s * m;
            for (int q = 0; q < s; q++) {
                if (r == 4) {
                    cdd a0 = src[q], a1 = src[q + sm], a2 = src[q + 2 * sm], a3 = src[q + 3 * sm];
                    cdd t0 = c_add(A, a0, a2), t1 = c_sub(A, a0, a2), t2 = c_add(A, a1, a3);
                    cdd t3 = c_mi(c_sub(A, a1, a3));
                    dst[q] = c_add(A, t0, t2);
                    if (p == 0) {
                        dst[q + s] = c_add(A, t1, t3);
                        dst[q + 2 * s] = c_sub(A, t0, t2);
                        dst[q + 3 * s] = c_sub(A, t1, t3);
                    } else {
                        dst[q + s] = c_mul(A, c_add(A, t1, t3), tw[0]);
                        dst[q + 2 * s] = c_mul(A, c_sub(A, t0, t2), tw[1]);
                        dst[q + 3 * s] = c_mul(A, c_sub(A, t1, t3), tw[2]);
                    }
                } else if (r == 2) {
                    cdd a0 = src[q], a1 = src[q + sm];
                    dst[q] = c_add(A, a0, a1);
                    dst[q + s] = p ? c_mul(A, c_sub(A, a0, a1), tw[0]) : c_sub(A, a0, a1);
                } else {
                    int i = r == 3 ? 0 : r == 5 ? 1 : 2;
                    odd_bfly(A, r, src, sm, dst, s, q, P->cr[i], P->sr[i], tw, p == 0);
                }
            }
        }
        cdd* t = a; a = b; b = t;
    }
    return a;
}

/* ------------------------------------------------------------------------------------------------------ */
/* complex FFT of any length: direct Stockham, four-step (Bailey) or Bluestein (fft.hpp:215-314)             */
/* ------------------------------------------------------------------------------------------------------ */
/* How the reference instantiates CFFT:
 *   fast  CFFT<double,double,V4>: 4 lanes, f64 everywhere.
 *   exact CFFT<dd,dd,DD4>: 4 lanes; four-step sub-FFTs in the short add, lane results renormalised through
 *         qts on store (fft.hpp:200-204); the direct and Bluestein paths in the accurate scalar add.
 *   dd    CFFT<dd,dd,dd> (kernel design): 1 lane, accurate add; the four-step twiddle skips column 0
 *         (fft.hpp:293), where 4 lanes multiply every k1 != 0 (fft.hpp:294). */
typedef struct { int lanes4, a_sub, a_sc, store_qts; } Mode;
static const Mode MODE_FAST = {1, A_F64, A_F64, 0};
static const Mode MODE_EXACT = {1, A_DDS, A_DDA, 1};
static const Mode MODE_DD = {0, A_DDA, A_DDA, 0};

static int smooth7(long long n) {
    if (n < 1) return 0;
    static const int ps[4] = {2, 3, 5, 7};
    for (int i = 0; i < 4; i++)
        while (n % ps[i] == 0) n /= ps[i];
    return n == 1;
}
static long long next_smooth7(long long n) {
    while (!smooth7(n)) n++;
    return n;
}

typedef struct CPlan {
    int n, four, N1, N2;
    Mode md;
    SPlan s1, s2, sd;
    cdd* tw; /* tw[k1*N2 + n2] = w_n^{k1 n2} */
    int m;   /* Bluestein length, 0 if unused */
    struct CPlan* inner;
    cdd *bc, *Vf;
} CPlan;

static cdd* cplan_run(const CPlan* C, cdd* x, cdd* y);
void oracle_cplan_free(CPlan* C);

static int cplan_init(CPlan* C, int n, Mode md) {
    memset(C, 0, sizeof *C);
    C->n = n;
    C->md = md;
    if (!smooth7(n)) {
        C->m = (int)next_smooth7(2LL * n - 1);
        C->inner = malloc(sizeof(CPlan));
        if (cplan_init(C->inner, C->m, md)) return -1;
        C->bc = malloc(sizeof(cdd) * n);
        cdd* v = calloc((size_t)C->m, sizeof(cdd));
        cdd* w = calloc((size_t)C->m, sizeof(cdd));
        for (long long t = 0; t < n; t++) {
            long long e = (long long)((__int128)t * t % (2LL * n));
            dd c, sn;
            dcis(e, 2LL * n, &c, &sn);
            C->bc[t] = cx(c, sn);
            v[t] = cx(c, sn);
            if (t) v[C->m - t] = cx(c, sn);
        }
        CPlan fd;
        cplan_init(&fd, C->m, MODE_DD);
        cdd* V = cplan_run(&fd, v, w);
        C->Vf = malloc(sizeof(cdd) * C->m);
        for (int k = 0; k < C->m; k++) C->Vf[k] = cx(ddivd(V[k].re, (double)C->m), ddivd(V[k].im, (double)C->m));
        free(v);
        free(w);
        oracle_cplan_free(&fd);
        return 0;
    }
    C->four = n > 2048;
    if (!C->four) return sfft_init(&C->sd, n);
    int best = 1;
    for (int d = 1; (long long)d * d <= n; d++)
        if (n % d == 0) best = d;
    C->N1 = best;
    C->N2 = n / best;
    if (C->N1 < 8) {
        C->four = 0;
        return sfft_init(&C->sd, n);
    }
    sfft_init(&C->s1, C->N1);
    sfft_init(&C->s2, C->N2);
    C->tw = malloc(sizeof(cdd) * (size_t)n);
    CisTab ct;
    cis_init(&ct, n);
    for (int k1 = 0; k1 < C->N1; k1++)
        for (int n2 = 0; n2 < C->N2; n2++) {
            dd c, sn;
            cis_get(&ct, -(long long)k1 * n2, &c, &sn);
            C->tw[(size_t)k1 * C->N2 + n2] = cx(c, sn);
        }
    cis_free(&ct);
    return 0;
}

void oracle_cplan_free(CPlan* C) {
    if (C->m) {
        oracle_cplan_free(C->inner);
        free(C->inner);
        free(C->bc);
        free(C->Vf);
        return;
    }
    sfft_free(&C->s1);
    sfft_free(&C->s2);
    sfft_free(&C->sd);
    free(C->tw);
}

static inline dd renorm(dd v) { return qts(v.hi, v.lo); }

/* x: input (destroyed), y: output space; returns the result pointer (x or y) */
static cdd* cplan_run(const CPlan* C, cdd* x, cdd* y) {
    const int As = C->md.a_sc, Al = C->md.a_sub;
    if (C->m) { /* X_k = conj(b_k) sum_j (x_j conj(b_j)) b_{k-j} (fft.hpp:268-277) */
        cdd* u = malloc(sizeof(cdd) * C->m);
        cdd* u2 = malloc(sizeof(cdd) * C->m);
        for (int j = 0; j < C->n; j++) u[j] = c_mul(As, x[j], c_conj(C->bc[j]));
        for (int j = C->n; j < C->m; j++) u[j] = cx(D(0.0), D(0.0));
        cdd* U = cplan_run(C->inner, u, u2);
        for (int k = 0; k < C->m; k++) U[k] = c_conj(c_mul(As, U[k], C->Vf[k]));
        cdd* other = U == u ? u2 : u;
        cdd* Cc = cplan_run(C->inner, U, other);
        for (int k = 0; k < C->n; k++) y[k] = c_mul(As, c_conj(Cc[k]), c_conj(C->bc[k]));
        free(u);
        free(u2);
        return y;
    }
    if (!C->four) return sfft_run(&C->sd, As, x, y);
    const int N1 = C->N1, N2 = C->N2, M = N1 > N2 ? N1 : N2;
    cdd* tile = malloc(sizeof(cdd) * M);
    cdd* wk = malloc(sizeof(cdd) * M);
    for (int c0 = 0; c0 < N2; c0++) { /* column pass (fft.hpp:283-299) */
        for (int r = 0; r < N1; r++) tile[r] = x[(size_t)r * N2 + c0];
        cdd* res = sfft_run(&C->s1, Al, tile, wk);
        for (int k1 = 0; k1 < N1; k1++) {
            cdd v = res[k1];
            if (k1 && (C->md.lanes4 || c0)) v = c_mul(Al, v, C->tw[(size_t)k1 * N2 + c0]);
            if (C->md.store_qts) v = cx(renorm(v.re), renorm(v.im));
            x[(size_t)k1 * N2 + c0] = v;
        }
    }
    for (int r0 = 0; r0 < N1; r0++) { /* row pass, transposed store (fft.hpp:300-311) */
        for (int i = 0; i < N2; i++) tile[i] = x[(size_t)r0 * N2 + i];
        cdd* res = sfft_run(&C->s2, Al, tile, wk);
        for (int k2 = 0; k2 < N2; k2++) {
            cdd v = res[k2];
            if (C->md.store_qts) v = cx(renorm(v.re), renorm(v.im));
            y[(size_t)N1 * k2 + r0] = v;
        }
    }
    free(tile);
    free(wk);
    return y;
}

/* ------------------------------------------------------------------------------------------------------ */
/* real FFT through a half-length complex one (fft.hpp:352-461)                                              */
/* ------------------------------------------------------------------------------------------------------ */
typedef struct { int N, h, fast; CPlan c; cdd* w; } RPlan;

static int rplan_init(RPlan* R, int N, Mode md) {
    R->N = N;
    R->h = N / 2;
    R->fast = md.a_sc == A_F64;
    if (cplan_init(&R->c, R->h, md)) return -1;
    R->w = malloc(sizeof(cdd) * (R->h + 1));
    CisTab ct;
    cis_init(&ct, N);
    for (int k = 0; k <= R->h; k++) {
        dd c, s;
        cis_get(&ct, -k, &c, &s);
        R->w[k] = cx(c, s);
    }
    cis_free(&ct);
    return 0;
}
static void rplan_free(RPlan* R) {
    oracle_cplan_free(&R->c);
    free(R->w);
}

/* r: N reals as dd -> X: h+1 bins. z, y: h each */
static void rfft_forward(const RPlan* R, const dd* r, cdd* X, cdd* z, cdd* y) {
    const int h = R->h;
    const int A = R->fast ? A_F64 : A_DDA;
    for (int i = 0; i < h; i++) z[i] = cx(r[2 * i], r[2 * i + 1]);
    z = cplan_run(&R->c, z, y);
    X[0] = cx(a_add(A, z[0].re, z[0].im), D(0.0));
    X[h] = cx(a_sub(A, z[0].re, z[0].im), D(0.0));
    const dd half = D(0.5);
    if (R->fast) { /* contiguous loop (fft.hpp:366-373) */
        for (int k = 1; k < h; k++) {
            cdd a = z[k], b = c_conj(z[h - k]);
            cdd E = c_add(A, a, b), O = c_mi(c_sub(A, a, b));
            cdd v = c_add(A, E, c_mul(A, O, R->w[k]));
            X[k] = c_scale(A, v, half);
        }
    } else { /* conjugate pairs with shared E, O (fft.hpp:377-407) */
        for (int k = 1; k <= h / 2; k++) {
            const int j = h - k;
            cdd a = z[k], b = c_conj(z[j]);
            cdd E = c_add(A, a, b), O = c_mi(c_sub(A, a, b));
            cdd v = c_add(A, E, c_mul(A, O, R->w[k]));
            X[k] = c_scale(A, v, half);
            if (j != k) {
                cdd u = c_add(A, c_conj(E), c_mul(A, c_conj(O), R->w[j]));
                X[j] = c_scale(A, u, half);
            }
        }
    }
}

/* X: h+1 Hermitian bins -> r: N reals (unnormalised); z, y: h each (fft.hpp:411-461) */
static void rfft_inverse(const RPlan* R, const cdd* X, dd* r, cdd* z, cdd* y) {
    const int h = R->h;
    const int A = R->fast ? A_F64 : A_DDA;
    if (R->fast) {
        for (int k = 0; k < h; k++) {
            cdd a = X[k], b = c_conj(X[h - k]);
            cdd E = c_add(A, a, b), Dd = c_mul(A, c_sub(A, a, b), c_conj(R->w[k]));
            cdd v = cx(a_sub(A, E.re, Dd.im), a_add(A, E.im, Dd.re));
            z[k] = c_conj(v);
        }
    } else {
        for (int k = 0; k <= h / 2; k++) {
            const int j = h - k;
            cdd a = X[k], b = c_conj(X[j]);
            cdd E = c_add(A, a, b), split = c_sub(A, a, b);
            cdd Dd = c_mul(A, split, c_conj(R->w[k]));
            cdd v = cx(a_sub(A, E.re, Dd.im), a_add(A, E.im, Dd.re));
            z[k] = c_conj(v);
            if (k && j != k) {
                cdd Ej = c_conj(E), Dj = c_mul(A, cx(dneg(split.re), split.im), c_conj(R->w[j]));
                cdd u = cx(a_sub(A, Ej.re, Dj.im), a_add(A, Ej.im, Dj.re));
                z[j] = c_conj(u);
            }
        }
    }
    z = cplan_run(&R->c, z, y);
    for (int i = 0; i < h; i++) {
        r[2 * i] = z[i].re;
        r[2 * i + 1] = dneg(z[i].im);
    }
}

/* ------------------------------------------------------------------------------------------------------ */
/* kernel design (src/design.cpp:17-49), Burg edges (src/lpc.cpp:13-42)                                       */
/* ------------------------------------------------------------------------------------------------------ */
static dd* kernel_taps(int L, long long a, long long b, double beta) {
    dd* h = malloc(sizeof(dd) * (size_t)(L + 1));
    const dd ib = di0(D(beta)), ab = ddivd(D((double)a), (double)b);
    const dd PI = mk(PI_HI, PI_LO);
    for (int n = 0; n <= L; n++) {
        dd s = D(1.0);
        if (n) {
            long long m = (long long)(((__int128)n * a) % (2 * (__int128)b));
            dd c, sn;
            dcis(m, 2 * b, &c, &sn);
            s = ddiv(sn, ddivd(dmul(PI, dmuld(D((double)n), (double)a)), (double)b));
        }
        dd u = ddivd(D((double)n), (double)L);
        dd w = ddiv(di0(dmul(D(beta), dsqrt(dsub(D(1.0), dmul(u, u))))), ib);
        h[n] = dmul(dmul(ab, s), w);
    }
    return h;
}

static dd* kernel_spectrum(const dd* h, int Lk, int Nlen, double scale_den) {
    RPlan R;
    rplan_init(&R, Nlen, MODE_DD);
    dd* r = calloc((size_t)Nlen, sizeof(dd));
    r[0] = h[0];
    for (int n = 1; n <= Lk; n++) {
        r[n] = h[n];
        r[Nlen - n] = h[n];
    }
    cdd* X = malloc(sizeof(cdd) * (Nlen / 2 + 1));
    cdd* z = malloc(sizeof(cdd) * (Nlen / 2 + 1));
    cdd* y = malloc(sizeof(cdd) * (Nlen / 2 + 1));
    rfft_forward(&R, r, X, z, y);
    dd* H = malloc(sizeof(dd) * (Nlen / 2 + 1));
    for (int k = 0; k <= Nlen / 2; k++) H[k] = ddivd(X[k].re, scale_den);
    free(r); free(X); free(z); free(y);
    rplan_free(&R);
    return H;
}

static double* burg_extrap(const double* x, long long len, long long n) {
    const int order = 32, train = 4096;
    double* out = calloc((size_t)n + 1, sizeof(double));
    long long m = len < train ? len : train;
    const double* seg = x + len - m;
    if (m < 2 * order + 8) return out;
    int nz = 0;
    double mx = 0;
    for (long long i = 0; i < m; i++) {
        if (seg[i] != 0) nz = 1;
        mx = fmax(mx, fabs(seg[i]));
    }
    if (!nz) return out;
    long long nf = m - 1;
    dd* f = malloc(sizeof(dd) * nf);
    dd* bk = malloc(sizeof(dd) * nf);
    for (long long i = 0; i < nf; i++) { f[i] = D(seg[i + 1]); bk[i] = D(seg[i]); }
    dd a[40], ar[40];
    int na = 1;
    a[0] = D(1.0);
    for (int it = 0; it < order; it++) {
        dd num = D(0.0), den = D(0.0);
        for (long long i = 0; i < nf; i++) {
            num = dadd(num, dmul(f[i], bk[i]));
            den = dadd(den, dadd(dmul(f[i], f[i]), dmul(bk[i], bk[i])));
        }
        if (den.hi <= 0) break;
        dd k = ddiv(dneg(dmuld(num, 2.0)), den);
        a[na++] = D(0.0);
        for (int i = 0; i < na; i++) ar[i] = a[na - 1 - i];
        for (int i = 0; i < na; i++) a[i] = dadd(a[i], dmul(k, ar[i]));
        for (long long i = 0; i + 1 < nf; i++) {
            dd f2 = dadd(f[i + 1], dmul(k, bk[i + 1]));
            dd b2 = dadd(bk[i], dmul(k, f[i]));
            f[i] = f2; /* in place: step i reads f[i], f[i+1], bk[i], bk[i+1] before any of them changes */
            bk[i] = b2;
        }
        nf -= 1;
    }
    int p = na - 1;
    double* c = malloc(sizeof(double) * (p + 1));
    for (int i = 0; i < p; i++) c[i] = -(a[p - i].hi + a[p - i].lo);
    double* buf = malloc(sizeof(double) * (size_t)(p + n));
    for (int i = 0; i < p; i++) buf[i] = seg[m - p + i];
    for (long long i = 0; i < n; i++) {
        double s = 0;
        for (int j = 0; j < p; j++) s += c[j] * buf[i + j];
        buf[p + i] = s;
    }
    double lim = 4 * mx;
    int ok = 1;
    for (long long i = 0; i < n; i++)
        if (!isfinite(buf[p + i]) || fabs(buf[p + i]) > lim) { ok = 0; break; }
    if (ok)
        for (long long i = 0; i < n; i++) out[i] = buf[p + i];
    free(f); free(bk); free(c); free(buf);
    return out;
}

/* ------------------------------------------------------------------------------------------------------ */
/* planning (src/resampler.cpp:92-209)                                                                       */
/* ------------------------------------------------------------------------------------------------------ */
typedef struct {
    long long P, Q, nout, Lk, E, pre, span, nblk, base, tot, o, c2, fk, fi, fo, mn;
    int up, nb, marg, hop, Nb, Mb, Jg, gen;
    double fml;
    long long blk0, blk1; /* the blocks the engine runs: [0, nblk) unless a caller restricts them */
} Plan;

static long long gcdll(long long a, long long b) {
    while (b) { long long t = a % b; a = b; b = t; }
    return a < 0 ? -a : a;
}
static unsigned long long gcdull(unsigned long long a, unsigned long long b) {
    while (b) { unsigned long long t = a % b; a = b; b = t; }
    return a;
}
static int fixblk(int v) {
    while (v % 2 || !smooth7(v / 2)) v++;
    return v;
}
static int round_blk(int v, int fast_auto) {
    while (v % 2 || !smooth7(v / 2) || (fast_auto && (v / 2) % 7 == 0)) v++;
    return v;
}

enum { E_BAD_INPUT = -1, E_RATES = -2, E_RANGE = -3, E_TOO_LONG = -4, E_TOO_SHORT = -5, E_TOO_LARGE = -6 };

/* returns 0, 1 (equal rates: copy), or a negative error */
static int make_plan(Plan* pl, const double* in, long long frames, int ch, int rate_in, int rate_out, int fast,
                     double length, double beta, int block) {
    memset(pl, 0, sizeof *pl);
    if (ch < 1 || frames < 0 || (frames > 0 && !in)) return E_BAD_INPUT;
    if (rate_in < 1 || rate_out < 1) return E_RATES;
    if (!(length > 0 && length <= 10) || !(beta > 0 && beta <= 200) || block < 0) return E_RANGE;
    long long fo = rate_out, fi = rate_in, g = gcdll(fi, fo);
    pl->P = fo / g;
    pl->Q = fi / g;
    pl->up = fo > fi;
    pl->fi = fi;
    pl->fo = fo;
    const long long nin = frames, cap = LLONG_MAX / 16;
    __int128 n128 = ((__int128)nin * pl->P + pl->Q - 1) / pl->Q;
    if (nin > cap || n128 > cap) return E_TOO_LONG;
    pl->nout = (long long)n128;
    if (fo == fi) return 1;
    const long long P = pl->P, Q = pl->Q;
    long long fk = pl->up ? fo : fi, mn = fi < fo ? fi : fo;
    pl->fk = fk;
    pl->mn = mn;
    const double lk = floor(length * (double)fk);
    if (!(lk >= 1 && lk <= INT_MAX)) return E_RANGE;
    long long Lk = (long long)lk;
    pl->Lk = Lk;
    const double fml = sqrt(beta * beta + 9.8696044010893586) / (2 * 3.14159265358979323846 * length);
    const double drop = ceil(2 * fml);
    if (!((double)mn - drop > 2 * fml)) return E_TOO_SHORT;
    pl->fml = fml;
    pl->c2 = mn - (long long)drop;
    long long L = (Lk * fi + fk - 1) / fk + 1;
    long long m1 = (L + Q + Q - 1) / Q, m2 = pl->up ? (Lk + P + P - 1) / P : 0;
    long long margl = m1 > m2 ? m1 : m2;
    long long PQ = P > Q ? P : Q;
    if ((block ? block : 10 * margl) > INT_MAX / 2 / PQ) return E_TOO_LARGE;
    long long E = L + Q, pre = (E + 64 + Q - 1) / Q * Q, span = pre + nin + E + 64;
    const int fast_auto = !block && fast;
    long long v0 = 10 * margl;
    if (fast_auto) {
        long long t = 51200 / PQ;
        v0 = t < 4 * margl ? 4 * margl : t > 10 * margl ? 10 * margl : t;
    }
    int nb = block ? fixblk(block) : round_blk((int)v0, fast_auto);
    if (nb <= 2 * margl) return E_RANGE;
    const int marg = (int)margl;
    while (!block && nb > 4 * marg) {
        long long nbk = (span + (long long)(nb - 2 * marg) * Q - 1) / ((long long)(nb - 2 * marg) * Q);
        if ((long long)ch * ((nbk + 3) / 4) >= 16) break;
        int want = nb * 3 / 4;
        int nn = round_blk(4 * marg > want ? 4 * marg : want, fast_auto);
        if (nn >= nb) break;
        nb = nn;
    }
    pl->nb = nb;
    pl->marg = marg;
    pl->Nb = (int)(nb * Q);
    pl->Mb = (int)(nb * P);
    pl->hop = nb - 2 * marg;
    pl->nblk = (span + (long long)pl->hop * Q - 1) / ((long long)pl->hop * Q);
    pl->blk0 = 0;
    pl->blk1 = pl->nblk;
    pl->base = (long long)marg * Q;
    pl->tot = pl->base + pl->nblk * pl->hop * Q + pl->Nb;
    pl->E = E;
    pl->pre = pre;
    pl->span = span;
    pl->o = pre / Q * P;
    long long mx = fi > fo ? fi : fo;
    pl->gen = (double)(mx - mn) / 2 < 3 * fml;
    return 0;
}

/* ------------------------------------------------------------------------------------------------------ */
/* the block engine (src/resampler.cpp:34-88) and the whole conversion                                      */
/* ------------------------------------------------------------------------------------------------------ */
static void engine(const Plan* pl, double** xx, double** out, int ch, const dd* H, int fast) {
    const long long P = pl->P, Q = pl->Q;
    const int Nb = pl->Nb, Mb = pl->Mb, K = Mb / 2 + 1, up = pl->up, Jg = pl->Jg;
    const Mode md = fast ? MODE_FAST : MODE_EXACT;
    const int A = fast ? A_F64 : A_DDA;
    RPlan Fw, Iv;
    rplan_init(&Fw, Nb, md);
    rplan_init(&Iv, Mb, md);
    const int mx = Nb > Mb ? Nb : Mb;
    dd* rin = malloc(sizeof(dd) * (size_t)Nb);
    dd* r = malloc(sizeof(dd) * (size_t)Mb);
    cdd* X = malloc(sizeof(cdd) * (size_t)(Nb / 2 + 1));
    cdd* Y = malloc(sizeof(cdd) * (size_t)K);
    cdd* z = malloc(sizeof(cdd) * (size_t)(mx / 2 + 1));
    cdd* y = malloc(sizeof(cdd) * (size_t)(mx / 2 + 1));
    const cdd zero = cx(D(0.0), D(0.0));
    for (int c = 0; c < ch; c++)
        for (long long b = pl->blk0; b < pl->blk1; b++) {
            const double* s = xx[c] + b * pl->hop * Q;
            for (int i = 0; i < Nb; i++) rin[i] = D(s[i]);
            rfft_forward(&Fw, rin, X, z, y);
            if (Jg) { /* general fold (resampler.cpp:53-63) */
                for (int k = 0; k < K; k++) Y[k] = zero;
                for (int j = 0; j <= Jg; j++) {
                    int jj = j % Nb;
                    cdd x = jj <= Nb / 2 ? X[jj] : c_conj(X[Nb - jj]);
                    cdd v = c_scale(A, x, H[j]);
                    int k = j % Mb;
                    if (j == 0) Y[0] = c_add(A, Y[0], v);
                    else if (k == 0 || 2 * k == Mb) Y[k].re = a_add(A, Y[k].re, a_mul(A, D(2.0), v.re));
                    else if (2 * k < Mb) Y[k] = c_add(A, Y[k], v);
                    else Y[Mb - k] = c_add(A, Y[Mb - k], c_conj(v));
                }
                Y[0].im = D(0.0);
                Y[Mb / 2].im = D(0.0);
            } else if (!up) { /* downsampling fold (resampler.cpp:64-71) */
                for (int k = 0; k < K; k++) Y[k] = c_scale(A, X[k], H[k]);
                int jmax = Nb / 2 < Mb - 1 ? Nb / 2 : Mb - 1;
                for (int j = K; j <= jmax; j++) {
                    cdd v = c_scale(A, X[j], H[j]);
                    Y[Mb - j] = c_add(A, Y[Mb - j], c_conj(v));
                }
                Y[Mb / 2] = cx(a_mul(A, a_mul(A, D(2.0), X[Mb / 2].re), H[Mb / 2]), D(0.0));
            } else { /* upsampling: periodic extension (resampler.cpp:72-78) */
                for (int k = 0; k < K; k++) {
                    int kk = k % Nb;
                    cdd v = kk <= Nb / 2 ? X[kk] : c_conj(X[Nb - kk]);
                    Y[k] = c_scale(A, v, H[k]);
                }
                Y[Mb / 2].im = D(0.0);
            }
            rfft_inverse(&Iv, Y, r, z, y);
            double* dst = out[c];
            for (long long i = 0; i < (long long)pl->hop * P; i++) {
                long long d = b * pl->hop * P + i - pl->o;
                dd v = r[pl->marg * P + i];
                if (d >= 0 && d < pl->nout) dst[d] = fast ? v.hi : v.hi + v.lo;
            }
        }
    free(rin); free(r); free(X); free(Y); free(z); free(y);
    rplan_free(&Fw);
    rplan_free(&Iv);
}

/* ------------------------------------------------------------------------------------------------------ */
/* the long double engine: run_engine<long double, long double, long double> (resampler.cpp:214-215)         */
/* ------------------------------------------------------------------------------------------------------ */
/* Every value is an x87 extended real and every +, -, * one x87 operation (long double on x86-64: 64-bit
 * significand, round to nearest). Tables are the dd tables above converted by from_dd<long double>, i.e.
 * (long double)hi + (long double)lo (fft.hpp:17). CFFT<LD,LD,LD> has one lane, so its four-step twiddle skips
 * column 0 (fft.hpp:293); the RFFT split and merge run conjugate pairs (fft.hpp:397-407,447-457). */
typedef long double LD;
typedef struct { LD re, im; } cld;
static inline LD ld_of(dd v) { return (LD)v.hi + (LD)v.lo; }
static inline cld lc(LD re, LD im) { cld r; r.re = re; r.im = im; return r; }
static inline cld lc_of(cdd v) { return lc(ld_of(v.re), ld_of(v.im)); }
static inline cld l_add(cld a, cld b) { return lc(a.re + b.re, a.im + b.im); }
static inline cld l_sub(cld a, cld b) { return lc(a.re - b.re, a.im - b.im); }
static inline cld l_mul(cld a, cld b) { return lc(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cld l_conj(cld a) { return lc(a.re, -a.im); }
static inline cld l_mi(cld a) { return lc(a.im, -a.re); } /* a * (-i) */
static inline cld l_scale(cld a, LD h) { return lc(a.re * h, a.im * h); }

typedef struct {
    SPlan sp; /* radices and dd tables */
    cld* tw[MAXST];
    LD cr[3][7], sr[3][7];
} LSPlan;

static int lsfft_init(LSPlan* L, int n) {
    if (sfft_init(&L->sp, n)) return -1;
    for (int g = 0; g < L->sp.ns; g++) {
        const size_t cnt = (size_t)L->sp.m[g] * (L->sp.r[g] - 1);
        L->tw[g] = malloc(sizeof(cld) * cnt + 1);
        for (size_t i = 0; i < cnt; i++) L->tw[g][i] = lc_of(L->sp.tw[g][i]);
    }
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 7; k++) {
            L->cr[i][k] = ld_of(L->sp.cr[i][k]);
            L->sr[i][k] = ld_of(L->sp.sr[i][k]);
        }
    return 0;
}
static void lsfft_free(LSPlan* L) {
    for (int g = 0; g < L->sp.ns; g++) free(L->tw[g]);
    sfft_free(&L->sp);
}

static void l_odd_bfly(int R, const cld* src, size_t sm, cld* dst, int s, int q, const LD* cr, const LD* sr,
                       const cld* tw, int p0) {
    const int H = (R - 1) / 2;
    cld a0 = src[q], S[3], Df[3];
    for (int t = 1; t <= H; t++) {
        cld x = src[q + t * sm], y = src[q + (R - t) * sm];
        S[t - 1] = l_add(x, y);
        Df[t - 1] = l_sub(x, y);
    }
    cld sum = a0;
    for (int t = 0; t < H; t++) sum = l_add(sum, S[t]);
    dst[q] = sum;
    for (int u = 1; u <= H; u++) {
        cld Aa = a0, B = lc(0.0L, 0.0L);
        for (int t = 1; t <= H; t++) {
            int m = (t * u) % R;
            LD c = cr[m], sn = sr[m];
            Aa = lc(Aa.re + S[t - 1].re * c, Aa.im + S[t - 1].im * c);
            B = lc(B.re + Df[t - 1].re * sn, B.im + Df[t - 1].im * sn);
        }
        cld xu = lc(Aa.re + B.im, Aa.im - B.re), xr = lc(Aa.re - B.im, Aa.im + B.re);
        if (p0) {
            dst[q + u * s] = xu;
            dst[q + (R - u) * s] = xr;
        } else {
            dst[q + u * s] = l_mul(xu, tw[u - 1]);
            dst[q + (R - u) * s] = l_mul(xr, tw[R - u - 1]);
        }
    }
}

static cld* lsfft_run(const LSPlan* L, cld* x, cld* y) {
    const SPlan* P = &L->sp;
    cld *a = x, *b = y;
    for (int g = 0; g < P->ns; g++) {
        const int r = P->r[g], m = P->m[g], s = P->s[g];
        for (int p = 0; p < m; p++) {
            const cld* tw = L->tw[g] + (size_t)p * (r - 1);
            const cld* src = a + (size_t)s * p;
            cld* dst = b + (size_t)s * r * p;
            const size_t sm = (size_t)s * m;
            for (int q = 0; q < s; q++) {
                if (r == 4) {
                    cld a0 = src[q], a1 = src[q + sm], a2 = src[q + 2 * sm], a3 = src[q + 3 * sm];
                    cld t0 = l_add(a0, a2), t1 = l_sub(a0, a2), t2 = l_add(a1, a3), t3 = l_mi(l_sub(a1, a3));
                    dst[q] = l_add(t0, t2);
                    if (p == 0) {
                        dst[q + s] = l_add(t1, t3);
                        dst[q + 2 * s] = l_sub(t0, t2);
                        dst[q + 3 * s] = l_sub(t1, t3);
                    } else {
                        dst[q + s] = l_mul(l_add(t1, t3), tw[0]);
                        dst[q + 2 * s] = l_mul(l_sub(t0, t2), tw[1]);
                        dst[q + 3 * s] = l_mul(l_sub(t1, t3), tw[2]);
                    }
                } else if (r == 2) {
                    cld a0 = src[q], a1 = src[q + sm];
                    dst[q] = l_add(a0, a1);
                    dst[q + s] = p ? l_mul(l_sub(a0, a1), tw[0]) : l_sub(a0, a1);
                } else {
                    int i = r == 3 ? 0 : r == 5 ? 1 : 2;
                    l_odd_bfly(r, src, sm, dst, s, q, L->cr[i], L->sr[i], tw, p == 0);
                }
            }
        }
        cld* t = a; a = b; b = t;
    }
    return a;
}

typedef struct LCPlan {
    int n, four, N1, N2, m;
    LSPlan s1, s2, sd;
    cld* tw;
    struct LCPlan* inner;
    cld *bc, *Vf;
} LCPlan;

static void lcplan_free(LCPlan* C) {
    if (C->m) {
        lcplan_free(C->inner);
        free(C->inner);
        free(C->bc);
        free(C->Vf);
        return;
    }
    if (C->four) {
        lsfft_free(&C->s1);
        lsfft_free(&C->s2);
        free(C->tw);
    } else {
        lsfft_free(&C->sd);
    }
}

static int lcplan_init(LCPlan* C, int n) {
    memset(C, 0, sizeof *C);
    C->n = n;
    if (!smooth7(n)) { /* Bluestein (fft.hpp:228-240); Vf from the scalar dd transform, then from_dd */
        C->m = (int)next_smooth7(2LL * n - 1);
        C->inner = malloc(sizeof(LCPlan));
        if (lcplan_init(C->inner, C->m)) return -1;
        C->bc = malloc(sizeof(cld) * n);
        cdd* v = calloc((size_t)C->m, sizeof(cdd));
        cdd* w = calloc((size_t)C->m, sizeof(cdd));
        for (long long t = 0; t < n; t++) {
            long long e = (long long)((__int128)t * t % (2LL * n));
            dd c, sn;
            dcis(e, 2LL * n, &c, &sn);
            C->bc[t] = lc(ld_of(c), ld_of(sn));
            v[t] = cx(c, sn);
            if (t) v[C->m - t] = cx(c, sn);
        }
        CPlan fd;
        cplan_init(&fd, C->m, MODE_DD);
        cdd* V = cplan_run(&fd, v, w);
        C->Vf = malloc(sizeof(cld) * C->m);
        for (int k = 0; k < C->m; k++)
            C->Vf[k] = lc(ld_of(ddivd(V[k].re, (double)C->m)), ld_of(ddivd(V[k].im, (double)C->m)));
        free(v);
        free(w);
        oracle_cplan_free(&fd);
        return 0;
    }
    C->four = n > 2048;
    if (C->four) {
        int best = 1;
        for (int d = 1; (long long)d * d <= n; d++)
            if (n % d == 0) best = d;
        C->N1 = best;
        C->N2 = n / best;
        if (C->N1 < 8) C->four = 0;
    }
    if (!C->four) return lsfft_init(&C->sd, n);
    lsfft_init(&C->s1, C->N1);
    lsfft_init(&C->s2, C->N2);
    C->tw = malloc(sizeof(cld) * (size_t)n);
    CisTab ct;
    cis_init(&ct, n);
    for (int k1 = 0; k1 < C->N1; k1++)
        for (int n2 = 0; n2 < C->N2; n2++) {
            dd c, sn;
            cis_get(&ct, -(long long)k1 * n2, &c, &sn);
            C->tw[(size_t)k1 * C->N2 + n2] = lc(ld_of(c), ld_of(sn));
        }
    cis_free(&ct);
    return 0;
}

static cld* lcplan_run(const LCPlan* C, cld* x, cld* y) {
    if (C->m) { /* X_k = conj(b_k) sum_j (x_j conj(b_j)) b_{k-j} (fft.hpp:268-277) */
        cld* u = malloc(sizeof(cld) * C->m);
        cld* u2 = malloc(sizeof(cld) * C->m);
        for (int j = 0; j < C->n; j++) u[j] = l_mul(x[j], l_conj(C->bc[j]));
        for (int j = C->n; j < C->m; j++) u[j] = lc(0.0L, 0.0L);
        cld* U = lcplan_run(C->inner, u, u2);
        for (int k = 0; k < C->m; k++) U[k] = l_conj(l_mul(U[k], C->Vf[k]));
        cld* other = U == u ? u2 : u;
        cld* Cc = lcplan_run(C->inner, U, other);
        for (int k = 0; k < C->n; k++) y[k] = l_mul(l_conj(Cc[k]), l_conj(C->bc[k]));
        free(u);
        free(u2);
        return y;
    }
    if (!C->four) return lsfft_run(&C->sd, x, y);
    const int N1 = C->N1, N2 = C->N2, M = N1 > N2 ? N1 : N2;
    cld* tile = malloc(sizeof(cld) * M);
    cld* wk = malloc(sizeof(cld) * M);
    for (int c0 = 0; c0 < N2; c0++) { /* column pass, one lane: column 0 keeps its values (fft.hpp:283-299) */
        for (int r = 0; r < N1; r++) tile[r] = x[(size_t)r * N2 + c0];
        cld* res = lsfft_run(&C->s1, tile, wk);
        for (int k1 = 0; k1 < N1; k1++) {
            cld v = res[k1];
            if (k1 && c0) v = l_mul(v, C->tw[(size_t)k1 * N2 + c0]);
            x[(size_t)k1 * N2 + c0] = v;
        }
    }
    for (int r0 = 0; r0 < N1; r0++) { /* row pass, transposed store (fft.hpp:300-311) */
        for (int i = 0; i < N2; i++) tile[i] = x[(size_t)r0 * N2 + i];
        cld* res = lsfft_run(&C->s2, tile, wk);
        for (int k2 = 0; k2 < N2; k2++) y[(size_t)N1 * k2 + r0] = res[k2];
    }
    free(tile);
    free(wk);
    return y;
}

static void engine_ld(const Plan* pl, double** xx, double** out, int ch, const dd* Hd, long long Hn) {
    const long long P = pl->P, Q = pl->Q;
    const int Nb = pl->Nb, Mb = pl->Mb, K = Mb / 2 + 1, up = pl->up, Jg = pl->Jg, h = Nb / 2, hi = Mb / 2;
    LCPlan Fw, Iv;
    lcplan_init(&Fw, h);
    lcplan_init(&Iv, hi);
    cld* wf = malloc(sizeof(cld) * (h + 1));
    cld* wi = malloc(sizeof(cld) * (hi + 1));
    CisTab ct;
    cis_init(&ct, Nb);
    for (int k = 0; k <= h; k++) { dd c, s; cis_get(&ct, -k, &c, &s); wf[k] = lc(ld_of(c), ld_of(s)); }
    cis_free(&ct);
    cis_init(&ct, Mb);
    for (int k = 0; k <= hi; k++) { dd c, s; cis_get(&ct, -k, &c, &s); wi[k] = lc(ld_of(c), ld_of(s)); }
    cis_free(&ct);
    LD* H = malloc(sizeof(LD) * (size_t)Hn);
    for (long long k = 0; k < Hn; k++) H[k] = ld_of(Hd[k]);
    const int mx = Nb > Mb ? Nb : Mb;
    cld* X = malloc(sizeof(cld) * (size_t)(h + 1));
    cld* Y = malloc(sizeof(cld) * (size_t)K);
    cld* z = malloc(sizeof(cld) * (size_t)(mx / 2 + 1));
    cld* y = malloc(sizeof(cld) * (size_t)(mx / 2 + 1));
    LD* r = malloc(sizeof(LD) * (size_t)Mb);
    for (int c = 0; c < ch; c++)
        for (long long b = pl->blk0; b < pl->blk1; b++) {
            const double* s = xx[c] + b * pl->hop * Q;
            /* forward real FFT (fft.hpp:362-408): pack, transform, conjugate-pair split */
            for (int i = 0; i < h; i++) z[i] = lc((LD)s[2 * i], (LD)s[2 * i + 1]);
            cld* Z = lcplan_run(&Fw, z, y);
            X[0] = lc(Z[0].re + Z[0].im, 0.0L);
            X[h] = lc(Z[0].re - Z[0].im, 0.0L);
            for (int k = 1; k <= h / 2; k++) {
                const int j = h - k;
                cld A = Z[k], B = l_conj(Z[j]);
                cld E = l_add(A, B), O = l_mi(l_sub(A, B));
                cld v = l_add(E, l_mul(O, wf[k]));
                X[k] = lc(v.re * 0.5L, v.im * 0.5L);
                if (j != k) {
                    cld u = l_add(l_conj(E), l_mul(l_conj(O), wf[j]));
                    X[j] = lc(u.re * 0.5L, u.im * 0.5L);
                }
            }
            /* spectrum (resampler.cpp:53-78) */
            if (Jg) {
                for (int k = 0; k < K; k++) Y[k] = lc(0.0L, 0.0L);
                for (int j = 0; j <= Jg; j++) {
                    int jj = j % Nb;
                    cld x = jj <= Nb / 2 ? X[jj] : l_conj(X[Nb - jj]);
                    cld v = l_scale(x, H[j]);
                    int k = j % Mb;
                    if (j == 0) Y[0] = l_add(Y[0], v);
                    else if (k == 0 || 2 * k == Mb) Y[k].re = Y[k].re + 2.0L * v.re;
                    else if (2 * k < Mb) Y[k] = l_add(Y[k], v);
                    else Y[Mb - k] = l_add(Y[Mb - k], l_conj(v));
                }
                Y[0].im = 0.0L;
                Y[Mb / 2].im = 0.0L;
            } else if (!up) {
                for (int k = 0; k < K; k++) Y[k] = l_scale(X[k], H[k]);
                int jmax = Nb / 2 < Mb - 1 ? Nb / 2 : Mb - 1;
                for (int j = K; j <= jmax; j++) Y[Mb - j] = l_add(Y[Mb - j], l_conj(l_scale(X[j], H[j])));
                Y[Mb / 2] = lc(2.0L * X[Mb / 2].re * H[Mb / 2], 0.0L);
            } else {
                for (int k = 0; k < K; k++) {
                    int kk = k % Nb;
                    cld v = kk <= Nb / 2 ? X[kk] : l_conj(X[Nb - kk]);
                    Y[k] = l_scale(v, H[k]);
                }
                Y[Mb / 2].im = 0.0L;
            }
            /* inverse real FFT (fft.hpp:411-461): conjugate-pair merge, transform, unpack */
            for (int k = 0; k <= hi / 2; k++) {
                const int j = hi - k;
                cld A = Y[k], B = l_conj(Y[j]);
                cld E = l_add(A, B), split = l_sub(A, B);
                cld Dd = l_mul(split, l_conj(wi[k]));
                z[k] = l_conj(lc(E.re - Dd.im, E.im + Dd.re));
                if (k && j != k) {
                    cld Ej = l_conj(E), Dj = l_mul(lc(-split.re, split.im), l_conj(wi[j]));
                    z[j] = l_conj(lc(Ej.re - Dj.im, Ej.im + Dj.re));
                }
            }
            cld* Zi = lcplan_run(&Iv, z, y);
            for (int i = 0; i < hi; i++) {
                r[2 * i] = Zi[i].re;
                r[2 * i + 1] = -Zi[i].im;
            }
            double* dst = out[c];
            for (long long i = 0; i < (long long)pl->hop * P; i++) {
                long long d = b * pl->hop * P + i - pl->o;
                if (d >= 0 && d < pl->nout) dst[d] = (double)r[pl->marg * P + i];
            }
        }
    free(X); free(Y); free(z); free(y); free(r); free(H); free(wf); free(wi);
    lcplan_free(&Fw);
    lcplan_free(&Iv);
}

/* 32-sample raised-cosine fade (resampler.cpp:170-171) */
static void fade32(double fd[32]) {
    for (int i = 0; i < 32; i++) {
        dd co, sn;
        dcis(i, 64, &co, &sn);
        fd[i] = dmuld(dadd(D(1.0), co), 0.5).hi;
    }
}

/* Public oracle entry points -------------------------------------------------------------------------- */

/* info (>= 16 slots): P Q taps nb marg hop nblk Nb Mb pre o E tot gen Jg up */
static void fill_info(const Plan* pl, long long* info) {
    if (!info) return;
    long long v[16] = {pl->P, pl->Q, 2 * pl->Lk + 1, pl->nb, pl->marg, pl->hop, pl->nblk, pl->Nb, pl->Mb,
                       pl->pre, pl->o, pl->E, pl->tot, pl->gen, pl->Jg, pl->up};
    memcpy(info, v, sizeof v);
}

long long oracle_plan(long long frames, int ch, int rate_in, int rate_out, int fast, double length, double beta,
                      int block, long long* info) {
    Plan pl;
    static const double dummy = 0;
    int rc = make_plan(&pl, frames ? &dummy : NULL, frames, ch, rate_in, rate_out, fast, length, beta, block);
    if (rc < 0) return rc;
    fill_info(&pl, info);
    return pl.nout;
}

/* Full conversion. mode: 0 exact, 1 fast, 2 long double. out: ch * out_cap doubles, planar. Returns nout, or a
 * negative error code. */
/* The conversion with its block loop restricted to blocks [blk0, blk1) of every channel (blk1 < 0: all blocks);
 * output samples no block of the range writes stay as the caller left them. Test infrastructure for shares of a
 * conversion split across devices; the reference runs all blocks (src/resampler.cpp:41-48). */
long long oracle_resample_blocks(const double* in, long long frames, int ch, int rate_in, int rate_out, int mode,
                                 double length, double beta, int block, int lpc, long long blk0, long long blk1,
                                 double* out, long long out_cap, long long* info) {
    Plan pl;
    const int fast = mode == 1;
    int rc = make_plan(&pl, in, frames, ch, rate_in, rate_out, fast, length, beta, block);
    if (rc < 0) return rc;
    if (blk1 >= 0) {
        if (blk0 < 0 || blk1 < blk0 || blk1 > pl.nblk) return -101;
        pl.blk0 = blk0;
        pl.blk1 = blk1;
    }
    if (pl.nout > out_cap) return -100;
    if (rc == 1) {
        for (int c = 0; c < ch; c++)
            for (long long i = 0; i < frames; i++) out[(size_t)c * out_cap + i] = in[i * ch + c];
        fill_info(&pl, info);
        return pl.nout;
    }
    const long long nin = frames, Q = pl.Q, P = pl.P;
    double fd[32];
    fade32(fd);
    double** xx = malloc(sizeof(double*) * ch);
    for (int c = 0; c < ch; c++) {
        xx[c] = calloc((size_t)pl.tot, sizeof(double));
        double* X = xx[c] + pl.base + pl.pre;
        for (long long i = 0; i < nin; i++) X[i] = in[i * ch + c];
        if (lpc) {
            long long ext = pl.E + 32;
            double* tl = burg_extrap(X, nin, ext);
            for (int i = 0; i < 32; i++) tl[ext - 32 + i] *= fd[i];
            long long m = nin < 4096 ? nin : 4096;
            double* xr = malloc(sizeof(double) * (size_t)(m + 1));
            for (long long i = 0; i < m; i++) xr[i] = X[m - 1 - i];
            double* hd = burg_extrap(xr, m, ext);
            for (int i = 0; i < 32; i++) hd[ext - 32 + i] *= fd[i];
            for (long long i = 0; i < ext; i++) {
                X[nin + i] = tl[i];
                X[-1 - i] = hd[i];
            }
            free(tl); free(xr); free(hd);
        }
    }
    /* kernel (resampler.cpp:187-206) */
    dd* H;
    long long Hn;
    if (pl.gen) {
        long long Nk = (long long)(pl.Nb > pl.Mb ? pl.Nb : pl.Mb) * 5LL / 4;
        Nk += Nk & 1;
        while (!smooth7(Nk / 2)) Nk += 2;
        __int128 A = (__int128)pl.c2 * pl.Nb, B = (__int128)Nk * pl.fi;
        long long g2 = (long long)gcdull((unsigned long long)pl.c2 * (unsigned long long)pl.Nb,
                                         (unsigned long long)Nk * (unsigned long long)pl.fi);
        double fk2 = (double)Nk * pl.fi / pl.Nb;
        int L2 = (int)floor(length * fk2);
        dd* h2 = kernel_taps(L2, (long long)(A / g2), (long long)(B / g2), beta);
        H = kernel_spectrum(h2, L2, (int)Nk, (double)pl.Nb);
        Hn = Nk / 2 + 1;
        free(h2);
        long long jg = (long long)ceil((pl.mn / 2.0 + 4 * pl.fml) * pl.Nb / pl.fi);
        pl.Jg = (int)(Nk / 2 < jg ? Nk / 2 : jg);
    } else {
        long long gc = gcdll(pl.c2, pl.fk);
        dd* h = kernel_taps((int)pl.Lk, pl.c2 / gc, pl.fk / gc, beta);
        H = kernel_spectrum(h, (int)pl.Lk, pl.up ? pl.Mb : pl.Nb, (double)pl.Nb);
        Hn = (pl.up ? pl.Mb : pl.Nb) / 2 + 1;
        free(h);
    }
    double** op = malloc(sizeof(double*) * ch);
    for (int c = 0; c < ch; c++) op[c] = out + (size_t)c * out_cap;
    if (mode == 2) engine_ld(&pl, xx, op, ch, H, Hn);
    else engine(&pl, xx, op, ch, H, fast);
    (void)P;
    (void)Q;
    fill_info(&pl, info);
    for (int c = 0; c < ch; c++) free(xx[c]);
    free(xx); free(op); free(H);
    return pl.nout;
}

long long oracle_resample(const double* in, long long frames, int ch, int rate_in, int rate_out, int mode,
                          double length, double beta, int block, int lpc, double* out, long long out_cap,
                          long long* info) {
    return oracle_resample_blocks(in, frames, ch, rate_in, rate_out, mode, length, beta, block, lpc, 0, -1, out,
                                  out_cap, info);
}

/* Pieces for unit checks ------------------------------------------------------------------------------- */

/* Forward real FFT of N points. mode: 0 fast, 1 exact, 2 dd (kernel design). in: N dd (hi, lo pairs);
 * out: (N/2+1) complex dd as (re.hi, re.lo, im.hi, im.lo). */
int oracle_rfft_forward(int mode, int N, const double* in, double* out) {
    Mode md = mode == 0 ? MODE_FAST : mode == 1 ? MODE_EXACT : MODE_DD;
    RPlan R;
    if (N < 2 || N % 2 || rplan_init(&R, N, md)) return -1;
    dd* r = malloc(sizeof(dd) * N);
    for (int i = 0; i < N; i++) r[i] = mk(in[2 * i], in[2 * i + 1]);
    cdd* X = malloc(sizeof(cdd) * (N / 2 + 1));
    cdd* z = malloc(sizeof(cdd) * (N / 2 + 1));
    cdd* y = malloc(sizeof(cdd) * (N / 2 + 1));
    rfft_forward(&R, r, X, z, y);
    memcpy(out, X, sizeof(cdd) * (N / 2 + 1));
    free(r); free(X); free(z); free(y);
    rplan_free(&R);
    return 0;
}

/* Inverse real FFT: in (N/2+1) complex dd -> out N dd (hi, lo) */
int oracle_rfft_inverse(int mode, int N, const double* in, double* out) {
    Mode md = mode == 0 ? MODE_FAST : mode == 1 ? MODE_EXACT : MODE_DD;
    RPlan R;
    if (N < 2 || N % 2 || rplan_init(&R, N, md)) return -1;
    cdd* X = malloc(sizeof(cdd) * (N / 2 + 1));
    memcpy(X, in, sizeof(cdd) * (N / 2 + 1));
    dd* r = malloc(sizeof(dd) * N);
    cdd* z = malloc(sizeof(cdd) * (N / 2 + 1));
    cdd* y = malloc(sizeof(cdd) * (N / 2 + 1));
    rfft_inverse(&R, X, r, z, y);
    memcpy(out, r, sizeof(dd) * N);
    free(r); free(X); free(z); free(y);
    rplan_free(&R);
    return 0;
}

/* Complex FFT of n points in a given mode; in/out n complex dd */
int oracle_cfft(int mode, int n, const double* in, double* out) {
    Mode md = mode == 0 ? MODE_FAST : mode == 1 ? MODE_EXACT : MODE_DD;
    CPlan C;
    if (cplan_init(&C, n, md)) return -1;
    cdd* x = malloc(sizeof(cdd) * n);
    cdd* y = malloc(sizeof(cdd) * n);
    memcpy(x, in, sizeof(cdd) * n);
    cdd* r = cplan_run(&C, x, y);
    memcpy(out, r, sizeof(cdd) * n);
    free(x); free(y);
    oracle_cplan_free(&C);
    return 0;
}

/* Kernel spectrum for a plan: H (len n/2+1 dd). Returns its length. */
long long oracle_kernel(int rate_in, int rate_out, int fast, double length, double beta, int block, long long frames,
                        int ch, double* H_out, long long cap) {
    Plan pl;
    static const double dummy = 0;
    int rc = make_plan(&pl, frames ? &dummy : NULL, frames, ch, rate_in, rate_out, fast, length, beta, block);
    if (rc != 0) return rc < 0 ? rc : 0;
    if (pl.gen) return -200;
    long long gc = gcdll(pl.c2, pl.fk);
    dd* h = kernel_taps((int)pl.Lk, pl.c2 / gc, pl.fk / gc, beta);
    int n = pl.up ? pl.Mb : pl.Nb;
    dd* H = kernel_spectrum(h, (int)pl.Lk, n, (double)pl.Nb);
    long long len = n / 2 + 1;
    if (len <= cap) memcpy(H_out, H, sizeof(dd) * len);
    free(h); free(H);
    return len;
}

/* Burg extrapolation of n samples after x[0..len) */
int oracle_burg(const double* x, long long len, long long n, double* out) {
    double* r = burg_extrap(x, len, n);
    memcpy(out, r, sizeof(double) * n);
    free(r);
    return 0;
}
