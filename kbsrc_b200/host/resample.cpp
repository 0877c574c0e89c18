// Host side of the converter: argument checks, block planning, Burg LPC edges, Kaiser taps, and the calls into
// the GPU engine through the C ABI (include/kbsrc_gpu.h). Replaces HongYue1/KBSRC src/resampler.cpp:92-228
// (resample_impl), src/design.cpp:17-37 (kernel_taps), src/lpc.cpp:13-42 (burg_extrap) and src/dispatch.cpp
// (the round-to-nearest guard). The block loop itself (resampler.cpp:34-88) runs on the GPU.
//
// Block planning, tap values and LPC edges are part of the output definition: the integer formulas, the
// double-double operation order and the 16-task shrink rule are the reference's, so the engine sees the
// same blocks and kernel and the output is byte-identical.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <future>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>
#if defined(__x86_64__) || defined(__i386__)
#include <xmmintrin.h>
#else
#include <cfenv>
#endif

#include "ddh.hpp"
#include "kbsrc/kbsrc.hpp"
#include "kbsrc/kbsrc_c.h"
#include "kbsrc_gpu.h"

#ifndef KBSRC_VERSION
#define KBSRC_VERSION "1.3.0-b200"
#endif

namespace kbsrc {
namespace {

using host::dd;

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

// Exact and the split-precision forms (which keep Exact's plan and kernel) run their host arithmetic in
// round-to-nearest.
bool is_split_or_exact(Precision p) {
    return p == Precision::Exact || p == Precision::SplitTC || p == Precision::SplitTC16;
}

// Runs Exact's host arithmetic in round-to-nearest and restores the caller's rounding mode on exit; only the
// SSE rounding-control bits are touched on x86 (the reference's dispatch.cpp:37-67 contract).
class RoundToNearest {
public:
    explicit RoundToNearest(bool on) {
        if (!on) return;
#if defined(__x86_64__) || defined(__i386__)
        saved_ = _mm_getcsr() & kRC;
        if (saved_) _mm_setcsr(_mm_getcsr() & ~kRC);
#else
        const int m = std::fegetround();
        if (m >= 0 && m != FE_TONEAREST && std::fesetround(FE_TONEAREST) == 0) saved_ = m;
#endif
    }
    ~RoundToNearest() {
#if defined(__x86_64__) || defined(__i386__)
        if (saved_) _mm_setcsr((_mm_getcsr() & ~kRC) | saved_);
#else
        if (saved_ != kNone) std::fesetround(saved_);
#endif
    }
    RoundToNearest(const RoundToNearest&) = delete;
    RoundToNearest& operator=(const RoundToNearest&) = delete;

private:
#if defined(__x86_64__) || defined(__i386__)
    static constexpr unsigned kRC = 0x6000;
    unsigned saved_ = 0;
#else
    static constexpr int kNone = -1;
    int saved_ = kNone;
#endif
};

// Runs body(i) for i in [0, n) on up to `threads` threads, each taking indices from a shared counter.
template <class F>
void parallel_for(int threads, long long n, long long chunk, F body) {
    std::atomic<long long> next(0);
    auto work = [&] {
        for (long long c; (c = next.fetch_add(chunk)) < n;)
            for (long long i = c; i < std::min(n, c + chunk); i++) body(i);
    };
    threads = (int)std::max<long long>(1, std::min<long long>(threads, (n + chunk - 1) / chunk));
    std::vector<std::thread> pool;
    try {
        for (int t = 1; t < threads; t++) pool.emplace_back(work);
    } catch (...) {
        // fewer threads: the ones started and this one share the work
    }
    work();
    for (auto& t : pool) t.join();
}

bool block_ok(int v, bool avoid7) { return v % 2 == 0 && host::smooth7(v / 2) && !(avoid7 && (v / 2) % 7 == 0); }

// The overlap-save plan of one conversion (resampler.cpp:98-209).
struct Plan {
    long long P = 0, Q = 0, nout = 0, Lk = 0, E = 0, pre = 0, nblk = 0, base = 0, c2 = 0, fk = 0, mn = 0;
    long long fi = 0, fo = 0;
    int nb = 0, marg = 0, hop = 0;
    bool up = false, general = false, copy = false;
    double fml = 0;
};

Plan make_plan(const void* in, long long frames, int ch, int rate_in, int rate_out, const Options& opt) {
    if (ch < 1 || frames < 0 || (frames > 0 && !in)) throw std::invalid_argument("bad input buffer");
    if (rate_in < 1 || rate_out < 1) throw std::invalid_argument("sample rates must be positive");
    if (!(opt.length > 0 && opt.length <= 10) || !(opt.beta > 0 && opt.beta <= 200) || opt.threads < 0 ||
        opt.block < 0)
        throw std::invalid_argument("option out of range");
    Plan pl;
    pl.fi = rate_in;
    pl.fo = rate_out;
    const long long g = std::gcd(pl.fi, pl.fo);
    pl.P = pl.fo / g;
    pl.Q = pl.fi / g;
    pl.up = pl.fo > pl.fi;
    const long long cap = LLONG_MAX / 16;
    const __int128 n128 = ((__int128)frames * pl.P + pl.Q - 1) / pl.Q;
    if (frames > cap || n128 > cap) throw std::invalid_argument("input too long");
    pl.nout = (long long)n128;
    if (pl.fo == pl.fi) {
        pl.copy = true;
        return pl;
    }
    const long long P = pl.P, Q = pl.Q;
    pl.fk = pl.up ? pl.fo : pl.fi;
    pl.mn = std::min(pl.fi, pl.fo);
    const double lk = std::floor(opt.length * (double)pl.fk);
    if (!(lk >= 1 && lk <= INT_MAX)) throw std::invalid_argument("option out of range");
    pl.Lk = (long long)lk;
    // transition band 2*fml wide; its top edge must fit below the lower Nyquist frequency
    pl.fml = std::sqrt(opt.beta * opt.beta + 9.8696044010893586) / (2 * 3.14159265358979323846 * opt.length);
    const double drop = std::ceil(2 * pl.fml);
    if (!((double)pl.mn - drop > 2 * pl.fml)) throw std::invalid_argument("length too short for these sample rates");
    pl.c2 = pl.mn - (long long)drop;
    const long long reach = (pl.Lk * pl.fi + pl.fk - 1) / pl.fk + 1;
    const long long margl = std::max((reach + Q + Q - 1) / Q, pl.up ? (pl.Lk + P + P - 1) / P : 0LL);
    if ((opt.block ? opt.block : 10 * margl) > INT_MAX / 2 / std::max(P, Q))
        throw std::invalid_argument("block, rates or length too large");
    pl.E = reach + Q;
    pl.pre = (pl.E + 64 + Q - 1) / Q * Q;
    const long long span = pl.pre + frames + pl.E + 64;
    // Fast's automatic block: about 51200 points in the larger transform, 4..10 margins, no factor 7
    const bool fast_auto = !opt.block && opt.precision == Precision::Fast;
    auto next_block = [](int v, bool avoid7) {
        while (!block_ok(v, avoid7)) v++;
        return v;
    };
    int nb = opt.block ? next_block(opt.block, false)
                       : next_block((int)(fast_auto ? std::clamp(51200 / std::max(P, Q), 4 * margl, 10 * margl)
                                                    : 10 * margl),
                                    fast_auto);
    if (nb <= 2 * margl) throw std::invalid_argument("option out of range");
    const int marg = (int)margl;
    // Short inputs: smaller blocks until there are at least 16 quarter-block task groups. Machine-independent
    // by design, since the block size sets the rounding.
    while (!opt.block && nb > 4 * marg) {
        const long long hq = (long long)(nb - 2 * marg) * Q;
        const long long nbk = (span + hq - 1) / hq;
        if ((long long)ch * ((nbk + 3) / 4) >= 16) break;
        const int nn = next_block(std::max(4 * marg, nb * 3 / 4), fast_auto);
        if (nn >= nb) break;
        nb = nn;
    }
    pl.nb = nb;
    pl.marg = marg;
    pl.hop = nb - 2 * marg;
    pl.nblk = (span + (long long)pl.hop * Q - 1) / ((long long)pl.hop * Q);
    pl.base = (long long)marg * Q;
    pl.general = (double)(std::max(pl.fi, pl.fo) - pl.mn) / 2 < 3 * pl.fml;
    return pl;
}

// One-sided Kaiser-windowed sinc taps h[0..L], relative cutoff a/b, in dd (design.cpp:17-37). The sinc
// argument is reduced exactly: sin(pi n a/b) from the root e^{2 pi i (n a mod 2b) / 2b}.
std::vector<dd> kaiser_taps(int L, long long a, long long b, double beta, int threads) {
    std::vector<dd> h((size_t)L + 1);
    const dd i0b = host::bessel_i0(dd(beta)), ab = dd((double)a) / (double)b;
    parallel_for(threads, (long long)L + 1, 256, [&](long long n) {
        dd s(1.0);
        if (n) {
            const long long m = (long long)(((__int128)n * a) % (2 * (__int128)b));
            dd c, sn;
            host::unit_root(m, 2 * b, c, sn);
            s = sn / (host::kPi * (dd((double)n) * (double)a) / (double)b);
        }
        const dd u = dd((double)n) / (double)L;
        const dd w = host::bessel_i0(dd(beta) * host::sqrt_dd(dd(1.0) - u * u)) / i0b;
        h[n] = ab * s * w;
    });
    return h;
}

// Burg LPC (order 32, trained on the last 4096 samples) predicting n samples after x[0..len) (lpc.cpp:13-42).
// Zeros when the segment is too short, silent, or the prediction leaves 4x the segment's peak.
std::vector<double> burg_predict(const double* x, long long len, long long n) {
    constexpr int order = 32, train = 4096;
    std::vector<double> out((size_t)n, 0.0);
    const long long m = std::min<long long>(len, train);
    const double* seg = x + len - m;
    if (m < 2 * order + 8) return out;
    bool nonzero = false;
    double peak = 0;
    for (long long i = 0; i < m; i++) {
        nonzero |= seg[i] != 0;
        peak = std::max(peak, std::fabs(seg[i]));
    }
    if (!nonzero) return out;
    std::vector<dd> fw(seg + 1, seg + m), bw(seg, seg + m - 1), a{dd(1.0)};
    for (int it = 0; it < order; it++) {
        dd num(0.0), den(0.0);
        for (size_t i = 0; i < fw.size(); i++) {
            num = num + fw[i] * bw[i];
            den = den + (fw[i] * fw[i] + bw[i] * bw[i]);
        }
        if (den.hi <= 0) break;
        const dd k = -(num * 2.0) / den;
        a.push_back(dd(0.0));
        const std::vector<dd> rev(a.rbegin(), a.rend());
        for (size_t i = 0; i < a.size(); i++) a[i] = a[i] + k * rev[i];
        for (size_t i = 0; i + 1 < fw.size(); i++) {  // in place: reads i and i+1 before they change
            const dd f2 = fw[i + 1] + k * bw[i + 1], b2 = bw[i] + k * fw[i];
            fw[i] = f2;
            bw[i] = b2;
        }
        fw.pop_back();
        bw.pop_back();
    }
    const int p = (int)a.size() - 1;
    std::vector<double> c(p), buf((size_t)(p + n));
    for (int i = 0; i < p; i++) c[i] = -(a[p - i].hi + a[p - i].lo);
    for (int i = 0; i < p; i++) buf[i] = seg[m - p + i];
    for (long long i = 0; i < n; i++) {
        double s = 0;
        for (int j = 0; j < p; j++) s += c[j] * buf[i + j];
        buf[p + i] = s;
    }
    const double lim = 4 * peak;
    for (long long i = 0; i < n; i++)
        if (!std::isfinite(buf[p + i]) || std::fabs(buf[p + i]) > lim) return out;
    std::copy(buf.begin() + p, buf.end(), out.begin());
    return out;
}

void gpu_check(int rc, const char* what) {
    if (rc == KBSRC_GPU_OK) return;
    if (rc == KBSRC_GPU_E_NOMEM) throw std::bad_alloc();
    throw std::runtime_error(std::string(what) + ": " + kbsrc_gpu_last_error());
}

struct EngineHandle {
    kbsrc_gpu_engine* e = nullptr;
    EngineHandle() = default;
    EngineHandle(const EngineHandle&) = delete;
    EngineHandle& operator=(const EngineHandle&) = delete;
    ~EngineHandle() { kbsrc_gpu_engine_destroy(e); }
};

// A planned conversion: everything but the block loop, ready to run on new input of the same shape.
struct Conversion {
    Plan pl;
    Options opt;
    int ch = 0;
    long long frames = 0;
    std::vector<double> head, tail;  // LPC edges, ch * ext each
    long long ext = 0;
    std::vector<double> H;           // kernel spectrum (hi, lo) pairs
    kbsrc_gpu_desc desc{};           // the engine's plan (desc.H points into H); desc.shard: its share, if any
    EngineHandle eng;
    double design_seconds = 0;
};

// Kernel spectra shared by the conversions of a batch: the same taps and transform give the same spectrum.
struct SpectrumCache {
    std::map<std::tuple<int, long long, long long, double, int, long long>, std::vector<double>> m;
    std::mutex mu;
};

// CUDA start-up (context creation and kernel attributes take a good fraction of a second) runs on its own thread
// from the first conversion (or warm_up()) on, overlapping the host's LPC and kernel taps; gpu_ready() waits.
// The status travels with its message: kbsrc_gpu_last_error() belongs to the thread that failed.
std::shared_future<std::pair<int, std::string>>& gpu_init_future() {
    static std::mutex mu;
    static std::shared_future<std::pair<int, std::string>> f;
    std::lock_guard<std::mutex> lock(mu);
    if (!f.valid())
        f = std::async(std::launch::async, [] {
                const int rc = kbsrc_gpu_init();
                return std::make_pair(rc, std::string(rc ? kbsrc_gpu_last_error() : ""));
            }).share();
    return f;
}
void gpu_ready() {
    const auto& r = gpu_init_future().get();
    if (r.first == KBSRC_GPU_E_NOMEM) throw std::bad_alloc();
    if (r.first) throw std::runtime_error("GPU initialisation: " + r.second);
}

// KBSRC_TRACE=1: the host phases of each preparation on stderr
bool trace_on() {
    static const bool on = [] {
        const char* v = std::getenv("KBSRC_TRACE");
        return v && *v && *v != '0';
    }();
    return on;
}

// Input sample i (= frame * ch + channel) of interleaved data in a KBSRC_GPU_IN_* format, decoded as the WAV
// reader decodes it (src/io/wav.cpp:299-362); the GPU gather decodes the same way.
double input_sample(const void* p, int fmt, long long i) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    switch (fmt) {
        case KBSRC_GPU_IN_F32: { float v; std::memcpy(&v, b + 4 * i, 4); return v; }
        case KBSRC_GPU_IN_S32: { int32_t v; std::memcpy(&v, b + 4 * i, 4); return v / 2147483648.0; }
        case KBSRC_GPU_IN_S24: {
            int32_t v = b[3 * i] | b[3 * i + 1] << 8 | b[3 * i + 2] << 16;
            if (v & 0x800000) v -= 1 << 24;
            return v / 8388608.0;
        }
        case KBSRC_GPU_IN_S16: { int16_t v; std::memcpy(&v, b + 2 * i, 2); return v / 32768.0; }
        case KBSRC_GPU_IN_U8: return ((int)b[i] - 128) / 128.0;
        default: { double v; std::memcpy(&v, b + 8 * i, 8); return v; }
    }
}

// Plans a conversion, predicts its LPC edges, designs its kernel and creates its engine. `in`: interleaved
// input in format in_fmt (KBSRC_GPU_IN_*); only the first and last 4096 frames are read here.
std::unique_ptr<Conversion> prepare(const void* in, long long frames, int ch, int rate_in, int rate_out,
                                    const Options& opt, bool make_engine = true, SpectrumCache* cache = nullptr,
                                    int in_fmt = KBSRC_GPU_IN_F64) {
    auto cv = std::make_unique<Conversion>();
    cv->pl = make_plan(in, frames, ch, rate_in, rate_out, opt);
    cv->opt = opt;
    cv->ch = ch;
    cv->frames = frames;
    const Plan& pl = cv->pl;
    if (pl.copy) return cv;
    const double t0 = now();
    gpu_init_future();  // start CUDA while the host works
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int threads = opt.threads ? opt.threads : std::min(hw, 8);
    const long long Q = pl.Q, P = pl.P, Nb = (long long)pl.nb * Q, Mb = (long long)pl.nb * P;
    // LPC edges: the tail predicted from the last 4096 samples, the head from the first 4096 reversed, each
    // faded out over its last 32 samples (resampler.cpp:168-186)
    const long long ext = opt.lpc_edges ? pl.E + 32 : 0;
    cv->ext = ext;
    cv->head.assign((size_t)(ext * ch), 0.0);
    cv->tail.assign((size_t)(ext * ch), 0.0);
    if (ext) {
        double fade[32];
        for (int i = 0; i < 32; i++) {
            dd co, sn;
            host::unit_root(i, 64, co, sn);
            fade[i] = ((dd(1.0) + co) * 0.5).hi;
        }
        parallel_for(threads, 2LL * ch, 1, [&](long long job) {
            const int c = (int)(job / 2);
            const long long m = std::min<long long>(frames, 4096);
            std::vector<double> seg((size_t)m);
            if (job % 2 == 0)  // tail: the channel's last m samples in order
                for (long long i = 0; i < m; i++) seg[i] = input_sample(in, in_fmt, (frames - m + i) * ch + c);
            else  // head: the first m samples reversed
                for (long long i = 0; i < m; i++) seg[i] = input_sample(in, in_fmt, (m - 1 - i) * ch + c);
            std::vector<double> pred = burg_predict(seg.data(), m, ext);
            for (int i = 0; i < 32; i++) pred[ext - 32 + i] *= fade[i];
            std::copy(pred.begin(), pred.end(), (job % 2 == 0 ? cv->tail : cv->head).begin() + c * ext);
        });
    }
    // kernel: taps on the host, spectrum on the GPU (design.cpp:40-49)
    int L, nspec, Jg = 0;
    long long ta, tb;
    if (pl.general) {
        // Near-unity ratios: the kernel sampled on a finer grid of Nk points (rate Nk*fi/Nb) so its spectrum is
        // the true continuous response, folded modulo Mb by the engine (resampler.cpp:187-202).
        long long Nk = std::max(Nb, Mb) * 5LL / 4;
        Nk += Nk & 1;
        while (!host::smooth7(Nk / 2)) Nk += 2;
        const __int128 A = (__int128)pl.c2 * Nb, B = (__int128)Nk * pl.fi;
        const long long g2 = (long long)std::gcd((unsigned long long)pl.c2 * (unsigned long long)Nb,
                                                 (unsigned long long)Nk * (unsigned long long)pl.fi);
        const double fk2 = (double)Nk * pl.fi / Nb;
        L = (int)std::floor(opt.length * fk2);
        ta = (long long)(A / g2);
        tb = (long long)(B / g2);
        nspec = (int)Nk;
        Jg = (int)std::min<long long>(Nk / 2, (long long)std::ceil((pl.mn / 2.0 + 4 * pl.fml) * Nb / pl.fi));
    } else {
        const long long gc = std::gcd(pl.c2, pl.fk);
        L = (int)pl.Lk;
        ta = pl.c2 / gc;
        tb = pl.fk / gc;
        nspec = (int)(pl.up ? Mb : Nb);
    }
    const auto key = std::make_tuple(L, ta, tb, opt.beta, nspec, Nb);
    bool cached = false;
    if (cache) {
        std::lock_guard<std::mutex> lock(cache->mu);
        auto it = cache->m.find(key);
        if (it != cache->m.end()) {
            cv->H = it->second;
            cached = true;
        }
    }
    const double t_lpc = now();
    double t_taps = t_lpc;
    if (!cached) {
        const std::vector<dd> taps = kaiser_taps(L, ta, tb, opt.beta, threads);
        t_taps = now();
        gpu_ready();
        cv->H.assign((size_t)(nspec / 2 + 1) * 2, 0.0);
        gpu_check(kbsrc_gpu_kernel_spectrum(reinterpret_cast<const double*>(taps.data()), L, nspec, (double)Nb,
                                            cv->H.data()),
                  "kernel spectrum");
        if (cache) {
            std::lock_guard<std::mutex> lock(cache->mu);
            cache->m.emplace(key, cv->H);
        }
    }
    kbsrc_gpu_desc& d = cv->desc;
    d.precision = opt.precision == Precision::Fast         ? KBSRC_GPU_FAST
                  : opt.precision == Precision::LongDouble ? KBSRC_GPU_LD
                  : opt.precision == Precision::SplitTC    ? KBSRC_GPU_SPLIT
                  : opt.precision == Precision::SplitTC16  ? KBSRC_GPU_SPLIT_F16
                                                           : KBSRC_GPU_EXACT;
    d.channels = ch;
    d.P = P;
    d.Q = Q;
    d.nb = pl.nb;
    d.marg = pl.marg;
    d.nblk = pl.nblk;
    d.lead = pl.base + pl.pre;
    d.o = pl.pre / Q * P;
    d.frames = frames;
    d.nout = pl.nout;
    d.up = pl.up;
    d.Jg = Jg;
    d.edge_len = ext;
    d.H = cv->H.data();
    d.H_len = (long long)cv->H.size() / 2;
    d.in_format = in_fmt;
    const double t_spec = now();
    if (make_engine) {
        gpu_ready();
        gpu_check(kbsrc_gpu_engine_create(&d, &cv->eng.e), "GPU engine");
    }
    cv->design_seconds = now() - t0;
    if (trace_on())
        std::fprintf(stderr, "kbsrc trace: lpc %.3fs  taps %.3fs  spectrum (incl. GPU start) %.3fs  engine %.3fs\n",
                     t_lpc - t0, t_taps - t_lpc, t_spec - t_taps, now() - t_spec);
    return cv;
}

void fill_stats(const Conversion& cv, Stats* stats, double process_seconds) {
    if (!stats) return;
    const Plan& pl = cv.pl;
    stats->p = pl.P;
    stats->q = pl.Q;
    if (pl.copy) {
        stats->isa = "generic";
        stats->threads = 1;
        return;
    }
    stats->isa = kbsrc_gpu_engine_name();
    stats->taps = 2 * pl.Lk + 1;
    stats->block = pl.nb;
    stats->threads = 1;
    stats->general_fold = pl.general;
    stats->design_seconds = cv.design_seconds;
    stats->process_seconds = process_seconds;
    stats->passband = (double)pl.c2 / 2 - pl.fml;
    stats->stopband = (double)pl.c2 / 2 + pl.fml;
}

// Runs a prepared conversion on input of its shape (the whole interleaved input); out: planar ch * nout, or for a
// share ch * shard.nout (its output samples from shard.out0).
void run_conversion(Conversion& cv, const double* in, double* out) {
    const Plan& pl = cv.pl;
    if (pl.copy) {
        for (int c = 0; c < cv.ch; c++)
            for (long long i = 0; i < cv.frames; i++) out[c * pl.nout + i] = in[i * cv.ch + c];
        return;
    }
    const double* span = in ? in + cv.desc.shard.frame0 * cv.ch : in;
    gpu_check(kbsrc_gpu_engine_run_host(cv.eng.e, span, cv.head.data(), cv.tail.data(), out), "GPU engine");
}

// The shares of a prepared (engine-less) conversion over `count` devices: contiguous block ranges.
std::vector<kbsrc_gpu_shard> plan_shares(const Conversion& cv, int count) {
    if (count < 1) throw std::invalid_argument("no devices given");
    const int n = (int)std::min<long long>(count, std::max<long long>(1, cv.pl.nblk));
    std::vector<kbsrc_gpu_shard> sh((size_t)n);
    gpu_check(kbsrc_gpu_shard_plan(&cv.desc, n, sh.data()), "shard plan");
    return sh;
}

// Plans a conversion and creates the engine of share `index` of `count` on the current device.
std::unique_ptr<Conversion> prepare_share(const double* in, long long frames, int ch, int rate_in, int rate_out,
                                          const Options& opt, int index, int count) {
    auto cv = prepare(in, frames, ch, rate_in, rate_out, opt, false);
    if (cv->pl.copy) return cv;
    const std::vector<kbsrc_gpu_shard> sh = plan_shares(*cv, count);
    if (index < 0 || index >= (int)sh.size()) throw std::invalid_argument("share index out of range");
    cv->desc.shard = sh[(size_t)index];
    gpu_ready();
    gpu_check(kbsrc_gpu_engine_create(&cv->desc, &cv->eng.e), "GPU engine");
    return cv;
}

std::vector<std::vector<double>> resample_gpu(const double* in, long long frames, int ch, int rate_in, int rate_out,
                                              const Options& opt, Stats* stats) {
    auto cv = prepare(in, frames, ch, rate_in, rate_out, opt);
    const double t1 = now();
    const long long nout = cv->pl.nout;
    std::vector<double> planar((size_t)(nout * ch));
    run_conversion(*cv, in, planar.data());
    std::vector<std::vector<double>> out(ch);
    for (int c = 0; c < ch; c++) out[c].assign(planar.begin() + c * nout, planar.begin() + (c + 1) * nout);
    fill_stats(*cv, stats, now() - t1);
    return out;
}

}  // namespace

std::vector<std::vector<double>> resample(const double* in, long long frames, int channels, int rate_in, int rate_out,
                                          const Options& opt, Stats* stats) {
    RoundToNearest rn(is_split_or_exact(opt.precision));
    return resample_gpu(in, frames, channels, rate_in, rate_out, opt, stats);
}

std::vector<std::vector<double>> resample_devices(const double* in, long long frames, int channels, int rate_in,
                                                  int rate_out, const int* devices, int ndevices, const Options& opt,
                                                  Stats* stats) {
    if (!devices || ndevices < 1) throw std::invalid_argument("no devices given");
    RoundToNearest rn(is_split_or_exact(opt.precision));
    auto cv = prepare(in, frames, channels, rate_in, rate_out, opt, false);
    const double t1 = now();
    const long long nout = cv->pl.nout;
    std::vector<std::vector<double>> out((size_t)channels, std::vector<double>((size_t)nout));
    if (cv->pl.copy) {
        for (int c = 0; c < channels; c++)
            for (long long i = 0; i < frames; i++) out[c][i] = in[i * channels + c];
        fill_stats(*cv, stats, now() - t1);
        return out;
    }
    const std::vector<kbsrc_gpu_shard> sh = plan_shares(*cv, ndevices);
    // one host thread per share: select its device, create its engine, copy its input span up, run its blocks,
    // copy its output range down into the result; no data moves between devices
    std::vector<std::string> errors(sh.size());
    std::vector<int> nomem(sh.size(), 0);
    std::vector<std::thread> workers;
    for (size_t k = 0; k < sh.size(); k++)
        workers.emplace_back([&, k] {
            try {
                gpu_check(kbsrc_gpu_use_device(devices[k]), "device");
                kbsrc_gpu_desc d = cv->desc;
                d.shard = sh[k];
                EngineHandle e;
                gpu_check(kbsrc_gpu_engine_create(&d, &e.e), "GPU engine");
                std::vector<double> part((size_t)(channels * sh[k].nout));
                gpu_check(kbsrc_gpu_engine_run_host(e.e, in + sh[k].frame0 * channels, cv->head.data(),
                                                    cv->tail.data(), part.data()),
                          "GPU engine");
                for (int c = 0; c < channels; c++)
                    std::copy(part.begin() + c * sh[k].nout, part.begin() + (c + 1) * sh[k].nout,
                              out[c].begin() + sh[k].out0);
            } catch (const std::bad_alloc&) {
                nomem[k] = 1;
            } catch (const std::exception& x) {
                errors[k] = x.what();
            }
        });
    for (auto& w : workers) w.join();
    for (size_t k = 0; k < sh.size(); k++) {
        if (nomem[k]) throw std::bad_alloc();
        if (!errors[k].empty()) throw std::runtime_error("share " + std::to_string(k) + ": " + errors[k]);
    }
    fill_stats(*cv, stats, now() - t1);
    return out;
}

std::vector<unsigned char> resample_wav_data(const double* in, long long frames, int channels, int rate_in,
                                             int rate_out, const char* format, bool dither, long long& clipped,
                                             const Options& opt, Stats* stats) {
    const std::string f = format ? format : "";
    const int fmt = f == "f64" ? 0 : f == "f32" ? 1 : f == "s32" ? 2 : f == "s24" ? 3 : f == "s16" ? 4 : -1;
    if (fmt < 0) throw std::invalid_argument("format must be f64, f32, s32, s24 or s16");
    RoundToNearest rn(is_split_or_exact(opt.precision));
    auto cv = prepare(in, frames, channels, rate_in, rate_out, opt);
    if (cv->pl.copy) throw std::invalid_argument("equal rates: nothing to convert");
    const double t1 = now();
    const int bps = fmt == 0 ? 8 : fmt == 3 ? 3 : fmt == 4 ? 2 : 4;
    std::vector<unsigned char> data((size_t)(cv->pl.nout * channels * bps));
    gpu_check(kbsrc_gpu_engine_run_host_packed(cv->eng.e, in, cv->head.data(), cv->tail.data(), fmt, dither ? 1 : 0,
                                               data.data(), &clipped),
              "GPU engine");
    fill_stats(*cv, stats, now() - t1);
    return data;
}

std::vector<unsigned char> resample_wav_pcm(const void* pcm, const char* sample_format, long long frames,
                                            int channels, int rate_in, int rate_out, const char* format, bool dither,
                                            long long& clipped, const Options& opt, Stats* stats) {
    const std::string f = format ? format : "", sf = sample_format ? sample_format : "";
    const int fmt = f == "f64" ? 0 : f == "f32" ? 1 : f == "s32" ? 2 : f == "s24" ? 3 : f == "s16" ? 4 : -1;
    if (fmt < 0) throw std::invalid_argument("format must be f64, f32, s32, s24 or s16");
    const int in_fmt = sf == "f64"   ? KBSRC_GPU_IN_F64
                       : sf == "f32" ? KBSRC_GPU_IN_F32
                       : sf == "s32" ? KBSRC_GPU_IN_S32
                       : sf == "s24" ? KBSRC_GPU_IN_S24
                       : sf == "s16" ? KBSRC_GPU_IN_S16
                       : sf == "u8"  ? KBSRC_GPU_IN_U8
                                     : -1;
    if (in_fmt < 0) throw std::invalid_argument("sample format must be f64, f32, s32, s24, s16 or u8");
    RoundToNearest rn(is_split_or_exact(opt.precision));
    auto cv = prepare(pcm, frames, channels, rate_in, rate_out, opt, true, nullptr, in_fmt);
    if (cv->pl.copy) throw std::invalid_argument("equal rates: nothing to convert");
    const double t1 = now();
    const int bps = fmt == 0 ? 8 : fmt == 3 ? 3 : fmt == 4 ? 2 : 4;
    std::vector<unsigned char> data((size_t)(cv->pl.nout * channels * bps));
    gpu_check(kbsrc_gpu_engine_run_host_packed(cv->eng.e, static_cast<const double*>(pcm), cv->head.data(),
                                               cv->tail.data(), fmt, dither ? 1 : 0, data.data(), &clipped),
              "GPU engine");
    fill_stats(*cv, stats, now() - t1);
    return data;
}

void warm_up() { gpu_init_future(); }

const char* version() { return KBSRC_VERSION; }

}  // namespace kbsrc

// ---- C form -----------------------------------------------------------------------------------------------
namespace {
long long report(const char* msg, long long code, char* err, int err_len) {
    if (err && err_len > 0) {
        std::strncpy(err, msg, (size_t)err_len - 1);
        err[err_len - 1] = 0;
    }
    return code;
}
}  // namespace

extern "C" long long kbsrc_output_frames(long long frames, int rate_in, int rate_out) {
    if (frames < 0 || rate_in < 1 || rate_out < 1) return -1;
    const long long g = std::gcd((long long)rate_in, (long long)rate_out), P = rate_out / g, Q = rate_in / g;
    const __int128 n = ((__int128)frames * P + Q - 1) / Q;
    return n > LLONG_MAX / 16 ? -1 : (long long)n;
}

extern "C" long long kbsrc_resample_c(const double* in, long long frames, int channels, int rate_in, int rate_out,
                                      const kbsrc_options_c* copt, double* out, long long out_cap,
                                      kbsrc_stats_c* cst, char* err, int err_len) {
    try {
        kbsrc::Options o;
        if (copt) {
            o.precision = copt->precision == 0   ? kbsrc::Precision::Fast
                          : copt->precision == 2 ? kbsrc::Precision::LongDouble
                          : copt->precision == 3 ? kbsrc::Precision::SplitTC
                      : copt->precision == 4 ? kbsrc::Precision::SplitTC16
                          : copt->precision == 4 ? kbsrc::Precision::SplitTC16
                                                 : kbsrc::Precision::Exact;
            o.length = copt->length;
            o.beta = copt->beta;
            o.threads = copt->threads;
            o.block = copt->block;
            o.lpc_edges = copt->lpc_edges != 0;
        }
        kbsrc::Stats st;
        auto y = kbsrc::resample(in, frames, channels, rate_in, rate_out, o, &st);
        const long long n = y.empty() ? 0 : (long long)y[0].size();
        if (n > out_cap || (n > 0 && !out)) return report("output buffer too small", -2, err, err_len);
        for (int c = 0; c < channels; c++)
            if (n) std::memcpy(out + (size_t)c * out_cap, y[c].data(), (size_t)n * sizeof(double));
        if (cst) {
            cst->p = st.p; cst->q = st.q; cst->taps = st.taps; cst->block = st.block; cst->threads = st.threads;
            cst->general_fold = st.general_fold; cst->design_seconds = st.design_seconds;
            cst->process_seconds = st.process_seconds; cst->passband = st.passband; cst->stopband = st.stopband;
            cst->isa = st.isa;
        }
        return n;
    } catch (const std::invalid_argument& x) {
        return report(x.what(), -1, err, err_len);
    } catch (const std::bad_alloc&) {
        return report("out of memory", -4, err, err_len);
    } catch (const std::exception& x) {
        return report(x.what(), -3, err, err_len);
    }
}

extern "C" const char* kbsrc_version_c(void) { return kbsrc::version(); }

namespace {
kbsrc::Options options_from_c(const kbsrc_options_c* copt) {
    kbsrc::Options o;
    if (copt) {
        o.precision = copt->precision == 0   ? kbsrc::Precision::Fast
                      : copt->precision == 2 ? kbsrc::Precision::LongDouble
                      : copt->precision == 3 ? kbsrc::Precision::SplitTC
                      : copt->precision == 4 ? kbsrc::Precision::SplitTC16
                                             : kbsrc::Precision::Exact;
        o.length = copt->length;
        o.beta = copt->beta;
        o.threads = copt->threads;
        o.block = copt->block;
        o.lpc_edges = copt->lpc_edges != 0;
    }
    return o;
}
}  // namespace

extern "C" int kbsrc_prepare_c(const double* in, long long frames, int channels, int rate_in, int rate_out,
                               const kbsrc_options_c* copt, kbsrc_conversion** out, char* err, int err_len) {
    if (!out) return (int)report("null output pointer", -1, err, err_len);
    *out = nullptr;
    try {
        const kbsrc::Options o = options_from_c(copt);
        kbsrc::RoundToNearest rn(kbsrc::is_split_or_exact(o.precision));
        *out = reinterpret_cast<kbsrc_conversion*>(kbsrc::prepare(in, frames, channels, rate_in, rate_out, o).release());
        return 0;
    } catch (const std::invalid_argument& x) {
        return (int)report(x.what(), -1, err, err_len);
    } catch (const std::bad_alloc&) {
        return (int)report("out of memory", -4, err, err_len);
    } catch (const std::exception& x) {
        return (int)report(x.what(), -3, err, err_len);
    }
}

extern "C" long long kbsrc_resample_devices_c(const double* in, long long frames, int channels, int rate_in,
                                              int rate_out, const int* devices, int ndevices,
                                              const kbsrc_options_c* copt, double* out, long long out_cap,
                                              kbsrc_stats_c* cst, char* err, int err_len) {
    try {
        kbsrc::Stats st;
        auto y = kbsrc::resample_devices(in, frames, channels, rate_in, rate_out, devices, ndevices,
                                         options_from_c(copt), &st);
        const long long n = y.empty() ? 0 : (long long)y[0].size();
        if (n > out_cap || (n > 0 && !out)) return report("output buffer too small", -2, err, err_len);
        for (int c = 0; c < channels; c++)
            if (n) std::memcpy(out + (size_t)c * out_cap, y[c].data(), (size_t)n * sizeof(double));
        if (cst) {
            cst->p = st.p; cst->q = st.q; cst->taps = st.taps; cst->block = st.block; cst->threads = st.threads;
            cst->general_fold = st.general_fold; cst->design_seconds = st.design_seconds;
            cst->process_seconds = st.process_seconds; cst->passband = st.passband; cst->stopband = st.stopband;
            cst->isa = st.isa;
        }
        return n;
    } catch (const std::invalid_argument& x) {
        return report(x.what(), -1, err, err_len);
    } catch (const std::bad_alloc&) {
        return report("out of memory", -4, err, err_len);
    } catch (const std::exception& x) {
        return report(x.what(), -3, err, err_len);
    }
}

extern "C" int kbsrc_prepare_share_c(const double* in, long long frames, int channels, int rate_in, int rate_out,
                                     const kbsrc_options_c* copt, int index, int count, kbsrc_conversion** out,
                                     char* err, int err_len) {
    if (!out) return (int)report("null output pointer", -1, err, err_len);
    *out = nullptr;
    try {
        const kbsrc::Options o = options_from_c(copt);
        kbsrc::RoundToNearest rn(kbsrc::is_split_or_exact(o.precision));
        *out = reinterpret_cast<kbsrc_conversion*>(
            kbsrc::prepare_share(in, frames, channels, rate_in, rate_out, o, index, count).release());
        return 0;
    } catch (const std::invalid_argument& x) {
        return (int)report(x.what(), -1, err, err_len);
    } catch (const std::bad_alloc&) {
        return (int)report("out of memory", -4, err, err_len);
    } catch (const std::exception& x) {
        return (int)report(x.what(), -3, err, err_len);
    }
}

extern "C" int kbsrc_conversion_share_c(const kbsrc_conversion* cvp, long long* share6) {
    if (!cvp || !share6) return -1;
    const kbsrc_gpu_shard& s = reinterpret_cast<const kbsrc::Conversion*>(cvp)->desc.shard;
    const long long v[6] = {s.blk0, s.blk1, s.frame0, s.frames, s.out0, s.nout};
    std::memcpy(share6, v, sizeof v);
    return 0;
}

extern "C" int kbsrc_conversion_run_c(kbsrc_conversion* cv, const double* in, double* out, char* err, int err_len) {
    if (!cv) return (int)report("null conversion", -1, err, err_len);
    try {
        kbsrc::run_conversion(*reinterpret_cast<kbsrc::Conversion*>(cv), in, out);
        return 0;
    } catch (const std::bad_alloc&) {
        return (int)report("out of memory", -4, err, err_len);
    } catch (const std::exception& x) {
        return (int)report(x.what(), -3, err, err_len);
    }
}

extern "C" int kbsrc_conversion_info_c(const kbsrc_conversion* cvp, long long* nout, long long* edge_len,
                                       const double** head, const double** tail, kbsrc_gpu_engine** engine,
                                       kbsrc_stats_c* st) {
    if (!cvp) return -1;
    const auto& cv = *reinterpret_cast<const kbsrc::Conversion*>(cvp);
    if (nout) *nout = cv.pl.nout;
    if (edge_len) *edge_len = cv.ext;
    if (head) *head = cv.head.data();
    if (tail) *tail = cv.tail.data();
    if (engine) *engine = cv.eng.e;
    if (st) {
        kbsrc::Stats s;
        kbsrc::fill_stats(cv, &s, 0);
        st->p = s.p; st->q = s.q; st->taps = s.taps; st->block = s.block; st->threads = s.threads;
        st->general_fold = s.general_fold; st->design_seconds = s.design_seconds; st->process_seconds = 0;
        st->passband = s.passband; st->stopband = s.stopband; st->isa = s.isa;
    }
    return 0;
}

extern "C" void kbsrc_conversion_free_c(kbsrc_conversion* cv) { delete reinterpret_cast<kbsrc::Conversion*>(cv); }

// ---- diagnostics: the host-side pieces on their own ---------------------------------------------------------

// Block plan: info[16] = P Q taps nb marg hop nblk Nb Mb pre o E lead general up nout. Returns 0, 1 (equal rates)
// or -1 (invalid argument, message in err).
extern "C" int kbsrc_plan_c(long long frames, int channels, int rate_in, int rate_out, const kbsrc_options_c* copt,
                            long long* info, char* err, int err_len) {
    try {
        static const double dummy = 0;
        const kbsrc::Options o = options_from_c(copt);
        const kbsrc::Plan pl = kbsrc::make_plan(frames ? &dummy : nullptr, frames, channels, rate_in, rate_out, o);
        const long long v[16] = {pl.P, pl.Q, 2 * pl.Lk + 1, pl.nb, pl.marg, pl.hop, pl.nblk, (long long)pl.nb * pl.Q,
                                 (long long)pl.nb * pl.P, pl.pre, pl.Q ? pl.pre / pl.Q * pl.P : 0, pl.E,
                                 pl.base + pl.pre, pl.general, pl.up, pl.nout};
        if (info) std::memcpy(info, v, sizeof v);
        return pl.copy ? 1 : 0;
    } catch (const std::exception& x) {
        return (int)report(x.what(), -1, err, err_len);
    }
}

// Kaiser taps h[0..L] as (hi, lo) pairs (2L+2 doubles)
extern "C" int kbsrc_kernel_taps_c(int L, long long a, long long b, double beta, int threads, double* out) {
    if (L < 1 || a < 1 || b < 1 || !out) return -1;
    try {
        kbsrc::RoundToNearest rn(true);
        const auto h = kbsrc::kaiser_taps(L, a, b, beta, threads < 1 ? 1 : threads);
        std::memcpy(out, h.data(), h.size() * sizeof(kbsrc::host::dd));
        return 0;
    } catch (...) {
        return -4;
    }
}

// Burg LPC prediction of n samples following x[0..len)
extern "C" int kbsrc_burg_c(const double* x, long long len, long long n, double* out) {
    if (len < 0 || n < 0 || (len > 0 && !x) || (n > 0 && !out)) return -1;
    try {
        kbsrc::RoundToNearest rn(true);
        const auto p = kbsrc::burg_predict(x, len, n);
        std::copy(p.begin(), p.end(), out);
        return 0;
    } catch (...) {
        return -4;
    }
}

// ---- batches of conversions ------------------------------------------------------------------------------------
namespace kbsrc {
namespace {
struct BatchRun {
    std::vector<std::unique_ptr<Conversion>> convs;
    std::vector<int> gpu_index;  // conversion -> position in the GPU batch, -1 for equal-rate copies
    kbsrc_gpu_batch* gb = nullptr;
    ~BatchRun() { kbsrc_gpu_batch_destroy(gb); }
};
}  // namespace
}  // namespace kbsrc

extern "C" int kbsrc_batch_prepare_c(const kbsrc_batch_item_c* items, int count, const kbsrc_options_c* copt,
                                     kbsrc_batch** out, char* err, int err_len) {
    if (!out || !items || count < 1) return (int)report("empty batch", -1, err, err_len);
    *out = nullptr;
    try {
        const kbsrc::Options o = options_from_c(copt);
        kbsrc::RoundToNearest rn(kbsrc::is_split_or_exact(o.precision));
        auto b = std::make_unique<kbsrc::BatchRun>();
        b->convs.resize(count);
        kbsrc::SpectrumCache cache;
        std::vector<std::string> errors(count);
        std::vector<int> kinds(count, 0);  // 1 invalid argument, 3 runtime, 4 memory
        const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
        kbsrc::Options inner = o;
        inner.threads = 1;  // parallel over conversions instead
        kbsrc::parallel_for(o.threads ? o.threads : hw, count, 1, [&](long long i) {
            kbsrc::RoundToNearest rn_worker(kbsrc::is_split_or_exact(o.precision));
            try {
                b->convs[i] = kbsrc::prepare(items[i].in, items[i].frames, items[i].channels, items[i].rate_in,
                                             items[i].rate_out, inner, false, &cache);
            } catch (const std::invalid_argument& x) {
                errors[i] = x.what();
                kinds[i] = 1;
            } catch (const std::bad_alloc&) {
                errors[i] = "out of memory";
                kinds[i] = 4;
            } catch (const std::exception& x) {
                errors[i] = x.what();
                kinds[i] = 3;
            }
        });
        for (int i = 0; i < count; i++)
            if (kinds[i])
                return (int)report(("conversion " + std::to_string(i) + ": " + errors[i]).c_str(), -kinds[i], err,
                                   err_len);
        std::vector<kbsrc_gpu_desc> descs;
        b->gpu_index.assign(count, -1);
        for (int i = 0; i < count; i++)
            if (!b->convs[i]->pl.copy) {
                b->gpu_index[i] = (int)descs.size();
                descs.push_back(b->convs[i]->desc);
            }
        if (!descs.empty())
            kbsrc::gpu_check(kbsrc_gpu_batch_create(descs.data(), (int)descs.size(), &b->gb), "GPU batch");
        *out = reinterpret_cast<kbsrc_batch*>(b.release());
        return 0;
    } catch (const std::invalid_argument& x) {
        return (int)report(x.what(), -1, err, err_len);
    } catch (const std::bad_alloc&) {
        return (int)report("out of memory", -4, err, err_len);
    } catch (const std::exception& x) {
        return (int)report(x.what(), -3, err, err_len);
    }
}

extern "C" int kbsrc_batch_run_c(kbsrc_batch* bp, const double* const* in, double* const* out, char* err,
                                 int err_len) {
    if (!bp || !in || !out) return (int)report("null batch or buffer array", -1, err, err_len);
    try {
        auto& b = *reinterpret_cast<kbsrc::BatchRun*>(bp);
        const int count = (int)b.convs.size();
        std::vector<const double*> gi, gh, gt;
        std::vector<double*> go;
        for (int i = 0; i < count; i++) {
            const kbsrc::Conversion& cv = *b.convs[i];
            if (b.gpu_index[i] < 0) {  // equal rates: the host copy
                for (int c = 0; c < cv.ch; c++)
                    for (long long f = 0; f < cv.frames; f++) out[i][c * cv.pl.nout + f] = in[i][f * cv.ch + c];
                continue;
            }
            gi.push_back(in[i]);
            gh.push_back(cv.head.data());
            gt.push_back(cv.tail.data());
            go.push_back(out[i]);
        }
        if (b.gb)
            kbsrc::gpu_check(kbsrc_gpu_batch_run_host(b.gb, gi.data(), gh.data(), gt.data(), go.data()), "GPU batch");
        return 0;
    } catch (const std::bad_alloc&) {
        return (int)report("out of memory", -4, err, err_len);
    } catch (const std::exception& x) {
        return (int)report(x.what(), -3, err, err_len);
    }
}

extern "C" int kbsrc_batch_info_c(const kbsrc_batch* bp, int i, long long* nout, long long* edge_len,
                                  const double** head, const double** tail, int* gpu_index) {
    if (!bp) return -1;
    const auto& b = *reinterpret_cast<const kbsrc::BatchRun*>(bp);
    if (i < 0 || i >= (int)b.convs.size()) return -1;
    const kbsrc::Conversion& cv = *b.convs[i];
    if (nout) *nout = cv.pl.nout;
    if (edge_len) *edge_len = cv.ext;
    if (head) *head = cv.head.data();
    if (tail) *tail = cv.tail.data();
    if (gpu_index) *gpu_index = b.gpu_index[i];
    return 0;
}

extern "C" kbsrc_gpu_batch* kbsrc_batch_gpu_c(kbsrc_batch* bp) {
    return bp ? reinterpret_cast<kbsrc::BatchRun*>(bp)->gb : nullptr;
}

extern "C" void kbsrc_batch_free_c(kbsrc_batch* bp) { delete reinterpret_cast<kbsrc::BatchRun*>(bp); }
