// kbsrc command-line tool on the GPU engine. Options, messages, exit codes (0 ok, 1 runtime error, 2 usage)
// and the -v plan line are those of HongYue1/KBSRC app/main.cpp:84-165, so scripts and the reference's own
// test suites drive it unchanged.
#include <algorithm>
#include <cerrno>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <iterator>
#include <type_traits>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kbsrc/kbsrc.hpp"
#include "wav.hpp"

namespace {

// A command line the tool cannot act on: reported as "kbsrc: <text> (see --help)" with exit status 2.
struct BadCommandLine {
    std::string text;
};

double seconds_now() {
    using clock = std::chrono::steady_clock;
    return std::chrono::duration_cast<std::chrono::duration<double>>(clock::now().time_since_epoch()).count();
}

// Whole-string decimal numbers: leading blanks and a sign are accepted, trailing characters are not; an integer
// must fit an int and a real number must be finite.
bool whole_int(const std::string& text, int& out) {
    const char* s = text.c_str();
    char* end = nullptr;
    errno = 0;
    const long v = std::strtol(s, &end, 10);
    if (end == s || *end != '\0' || errno == ERANGE || v < INT_MIN || v > INT_MAX) return false;
    out = (int)v;
    return true;
}
bool whole_real(const std::string& text, double& out) {
    const char* s = text.c_str();
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(s, &end);
    if (end == s || *end != '\0' || errno == ERANGE || !std::isfinite(v)) return false;
    out = v;
    return true;
}

template <class T>
T option_value(const std::string& text, const char* option) {
    T v{};
    bool ok;
    if constexpr (std::is_same_v<T, int>) ok = whole_int(text, v);
    else ok = whole_real(text, v);
    if (!ok) throw BadCommandLine{std::string("invalid value for ") + option + ": " + text};
    return v;
}

void help() {
    std::printf(
        "kbsrc %s - Kaiser-Bessel sample-rate converter (B200 engine)\n"
        "\n"
        "usage: kbsrc [options] input.wav output.wav\n"
        "\n"
        "  -r, --rate N        output sample rate in Hz (default 44100)\n"
        "  -m, --mode M        exact (default), fast, ld, split or split16 (tensor-core forms, float64 accuracy)\n"
        "  -f, --format F      f64 (default), f32, s32, s24 or s16\n"
        "      --dither        TPDF dither for integer formats\n"
        "  -t, --threads N     host threads for kernel design and LPC (default: up to 8)\n"
        "      --len S         one-sided kernel length in seconds (default 0.2)\n"
        "      --beta B        Kaiser beta (default 40)\n"
        "      --block N       block size factor (default: automatic)\n"
        "      --no-lpc        zero-pad edges instead of LPC extrapolation\n"
        "  -v, --verbose       print plan and timing\n"
        "  -h, --help          show this help\n"
        "      --version       show version\n",
        kbsrc::version());
}

int run(int argc, char** argv) {
    kbsrc::Options opt;
    int rate = 44100;
    std::string format = "f64", in_path, out_path;
    bool dither = false, verbose = false;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto value = [&]() -> std::string {
            if (i + 1 >= argc) throw BadCommandLine{"missing value for " + a};
            return argv[++i];
        };
        if (a == "-r" || a == "--rate") rate = option_value<int>(value(), "--rate");
        else if (a == "-m" || a == "--mode") {
            const std::string m = value();
            if (m == "exact") opt.precision = kbsrc::Precision::Exact;
            else if (m == "fast") opt.precision = kbsrc::Precision::Fast;
            else if (m == "ld") opt.precision = kbsrc::Precision::LongDouble;
            else if (m == "split") opt.precision = kbsrc::Precision::SplitTC;
            else if (m == "split16") opt.precision = kbsrc::Precision::SplitTC16;
            else throw BadCommandLine{"mode must be exact, fast or ld"};
        } else if (a == "-f" || a == "--format") format = value();
        else if (a == "-t" || a == "--threads") opt.threads = option_value<int>(value(), "--threads");
        else if (a == "--block") opt.block = option_value<int>(value(), "--block");
        else if (a == "--len") opt.length = option_value<double>(value(), "--len");
        else if (a == "--beta") opt.beta = option_value<double>(value(), "--beta");
        else if (a == "--dither") dither = true;
        else if (a == "--no-lpc") opt.lpc_edges = false;
        else if (a == "-v" || a == "--verbose") verbose = true;
        else if (a == "-h" || a == "--help") { help(); return 0; }
        else if (a == "--version") { std::printf("kbsrc %s\n", kbsrc::version()); return 0; }
        else if (a.size() > 1 && a[0] == '-') throw BadCommandLine{"unknown option " + a};
        else if (in_path.empty()) in_path = a;
        else if (out_path.empty()) out_path = a;
        else throw BadCommandLine{"too many arguments"};
    }
    if (in_path.empty() || out_path.empty()) throw BadCommandLine{"expected input and output paths"};
    if (rate < 1 || rate > 10000000) throw BadCommandLine{"--rate must be between 1 and 10000000"};
    static const char* const kFormats[] = {"f64", "f32", "s32", "s24", "s16"};
    if (std::find(std::begin(kFormats), std::end(kFormats), format) == std::end(kFormats))
        throw BadCommandLine{"format must be f64, f32, s32, s24 or s16"};

    const double t0 = seconds_now();
    kbsrc::warm_up();  // the GPU starts while the file is read
    kbsrc::io::Audio a = kbsrc::io::read_wav_raw(in_path.c_str());  // decoded on the GPU while converting
    if (a.rate > 10000000) throw std::runtime_error("input sample rate above 10000000 Hz");
    kbsrc::io::check_wav_output(a.ch, rate, format);  // fail before converting
    const double t1 = seconds_now();
    kbsrc::Stats st;
    long long clipped = 0, nout = 0;
    double t2, t3;
    if (a.rate == rate) {  // equal rates: the host copy and the host writer
        kbsrc::io::decode_wav(a);
        auto y = kbsrc::resample(a.d.data(), a.frames, a.ch, a.rate, rate, opt, &st);
        t2 = seconds_now();
        nout = y.empty() ? 0 : (long long)y[0].size();
        kbsrc::io::write_wav(out_path.c_str(), y, a.ch, nout, rate, format, dither, clipped);
    } else {  // the input decode, the conversion and the output step (scale, dither, round, clip) on the GPU
        const auto data = kbsrc::resample_wav_pcm(a.bytes(), a.sample_format.c_str(), a.frames, a.ch, a.rate,
                                                  rate, format.c_str(), dither, clipped, opt, &st);
        t2 = seconds_now();
        const long long bps = format == "f64" ? 8 : format == "s24" ? 3 : format == "s16" ? 2 : 4;
        nout = (long long)data.size() / (a.ch * bps);
        kbsrc::io::write_wav_data(out_path.c_str(), a.ch, nout, rate, format, data.data(), data.size());
    }
    t3 = seconds_now();
    if (clipped) std::fprintf(stderr, "kbsrc: warning: %lld samples clipped\n", clipped);
    if (verbose) {
        std::fprintf(stderr, "%d Hz -> %d Hz, %d ch, %lld -> %lld frames\n", a.rate, rate, a.ch, a.frames, nout);
        std::fprintf(stderr, "P/Q=%lld/%lld taps=%lld block=%d threads=%d engine=%s%s\n", st.p, st.q, st.taps,
                     st.block, st.threads, st.isa, st.general_fold ? " (general fold)" : "");
        if (st.stopband > 0) std::fprintf(stderr, "passband 0-%.1f Hz, stopband from %.1f Hz\n", st.passband, st.stopband);
        std::fprintf(stderr, "read %.3fs  design %.3fs  resample %.3fs  write %.3fs  total %.3fs\n", t1 - t0,
                     st.design_seconds, t2 - t1 - st.design_seconds, t3 - t2, t3 - t0);
    }
    return 0;
}

}  // namespace

// Exit status 0 on success, 2 for a command line the tool cannot act on, 1 for any failure while converting; the
// reason goes to stderr after "kbsrc: " and no output file is left behind.
int main(int argc, char** argv) {
    std::string reason;
    int status = 1;
    try {
        return run(argc, argv);
    } catch (const BadCommandLine& e) {
        reason = e.text + " (see --help)";
        status = 2;
    } catch (const std::bad_alloc&) {
        reason = "out of memory";
    } catch (const std::exception& e) {
        reason = e.what();
    }
    std::fprintf(stderr, "kbsrc: %s\n", reason.c_str());
    return status;
}
