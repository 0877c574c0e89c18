// Rounding-mode check of kbsrc::resample (tests/test_gpu_fenv.py). The reference's contract
// (include/kbsrc/kbsrc.hpp:37-40, src/dispatch.cpp:31-67): an Exact conversion gives the round-to-nearest result
// whatever rounding mode the caller is in, and every conversion, a rejected one included, hands the caller's mode
// back unchanged.
//
// usage: fenv_check <exact|fast|ld> <rate_in> <rate_out> <channels> <length> <beta> <threads> <in.f64> <out_prefix>
//   in.f64  interleaved little-endian doubles (frames = bytes / 8 / channels)
// Converts the input once in each caller mode (nearest, up, down, toward zero). For each it writes the planar output
// to <out_prefix>.<mode>.f64 (channel after channel) and prints one line
//   mode=<name> kept=<0|1> threw=<0|1> samples=<n> engine=<Stats::isa>
// kept: fegetround() and, on x86, the SSE and x87 rounding-control fields read back equal after the call. Exit status
// 0 when the lines were printed, 2 on usage or I/O errors.
#include <cfenv>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>
#if defined(__x86_64__) || defined(__i386__)
#include <xmmintrin.h>
#endif

#include "kbsrc/kbsrc.hpp"

namespace {

// Everything a caller's rounding state consists of on this machine.
struct RoundingState {
    int fe;
    unsigned sse_rc, x87_rc;
};

RoundingState read_state() {
    RoundingState s{std::fegetround(), 0u, 0u};
#if defined(__x86_64__) || defined(__i386__)
    s.sse_rc = _mm_getcsr() & 0x6000u;
    unsigned short cw = 0;
    __asm__ volatile("fnstcw %0" : "=m"(cw));
    s.x87_rc = cw & 0x0C00u;
#endif
    return s;
}

bool same(const RoundingState& a, const RoundingState& b) {
    return a.fe == b.fe && a.sse_rc == b.sse_rc && a.x87_rc == b.x87_rc;
}

bool read_file(const char* path, std::vector<double>& v) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize((size_t)n / 8);
    const bool ok = std::fread(v.data(), 8, v.size(), f) == v.size();
    std::fclose(f);
    return ok;
}

bool write_file(const std::string& path, const std::vector<std::vector<double>>& y) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = true;
    for (const auto& c : y) ok = ok && std::fwrite(c.data(), 8, c.size(), f) == c.size();
    return std::fclose(f) == 0 && ok;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 10) {
        std::fprintf(stderr, "usage: fenv_check <exact|fast|ld> <rate_in> <rate_out> <channels> <length> <beta> "
                             "<threads> <in.f64> <out_prefix>\n");
        return 2;
    }
    // every argument is parsed in round-to-nearest, before any mode is changed
    const std::string prec = argv[1];
    kbsrc::Options opt;
    opt.precision = prec == "fast" ? kbsrc::Precision::Fast
                    : prec == "ld" ? kbsrc::Precision::LongDouble
                                   : kbsrc::Precision::Exact;
    const int rate_in = std::atoi(argv[2]), rate_out = std::atoi(argv[3]), ch = std::atoi(argv[4]);
    opt.length = std::strtod(argv[5], nullptr);
    opt.beta = std::strtod(argv[6], nullptr);
    opt.threads = std::atoi(argv[7]);
    std::vector<double> x;
    if (ch < 1 || !read_file(argv[8], x)) {
        std::fprintf(stderr, "fenv_check: cannot read %s\n", argv[8]);
        return 2;
    }
    const long long frames = (long long)x.size() / ch;
    const struct {
        const char* name;
        int fe;
    } modes[] = {{"nearest", FE_TONEAREST}, {"up", FE_UPWARD}, {"down", FE_DOWNWARD}, {"zero", FE_TOWARDZERO}};
    for (const auto& m : modes) {
        std::vector<std::vector<double>> y;
        kbsrc::Stats st;
        bool threw = false;
        std::fesetround(m.fe);
        const RoundingState before = read_state();
        try {
            y = kbsrc::resample(x.data(), frames, ch, rate_in, rate_out, opt, &st);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        const RoundingState after = read_state();
        std::fesetround(FE_TONEAREST);
        const std::string out = std::string(argv[9]) + "." + m.name + ".f64";
        if (!threw && !write_file(out, y)) {
            std::fprintf(stderr, "fenv_check: cannot write %s\n", out.c_str());
            return 2;
        }
        long long n = 0;
        for (const auto& c : y) n += (long long)c.size();
        std::printf("mode=%s kept=%d threw=%d samples=%lld engine=%s\n", m.name, same(before, after) ? 1 : 0,
                    threw ? 1 : 0, n, threw || !st.isa ? "-" : st.isa);
    }
    return 0;
}
