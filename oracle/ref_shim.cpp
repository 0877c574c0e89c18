// Test infrastructure: a C entry point over the reference library's public C++ API
// (include/kbsrc/kbsrc.hpp:41-45 in HongYue1/KBSRC), so Python tests and the CPU baseline can call the
// unmodified reference engine through ctypes. Built only into oracle/_ref/libkbsrc_ref.so; nothing in the
// product links it.
#include <cstring>
#include <exception>
#include <new>
#include <stdexcept>

#include "kbsrc/kbsrc.hpp"

extern "C" {

// precision: 0 fast, 1 exact, 2 long double. out: channels * out_cap doubles, planar.
// Returns the output frames per channel (>= 0), -1 on std::invalid_argument (message in err), -2 when out_cap
// is too small, -3 on any other error.
long long kbsrc_ref_resample(const double* in, long long frames, int channels, int rate_in, int rate_out,
                             int precision, double length, double beta, int threads, int block, int lpc,
                             double* out, long long out_cap, long long* plan /* p q taps block threads */,
                             double* seconds /* design, process */, char* err, int err_len) {
    kbsrc::Options o;
    o.precision = precision == 0 ? kbsrc::Precision::Fast
                  : precision == 2 ? kbsrc::Precision::LongDouble : kbsrc::Precision::Exact;
    o.length = length;
    o.beta = beta;
    o.threads = threads;
    o.block = block;
    o.lpc_edges = lpc != 0;
    kbsrc::Stats st;
    try {
        auto y = kbsrc::resample(in, frames, channels, rate_in, rate_out, o, &st);
        long long n = y.empty() ? 0 : (long long)y[0].size();
        if (n > out_cap) return -2;
        for (int c = 0; c < channels; c++) std::memcpy(out + (size_t)c * out_cap, y[c].data(), (size_t)n * 8);
        if (plan) {
            plan[0] = st.p; plan[1] = st.q; plan[2] = st.taps; plan[3] = st.block; plan[4] = st.threads;
        }
        if (seconds) { seconds[0] = st.design_seconds; seconds[1] = st.process_seconds; }
        return n;
    } catch (const std::invalid_argument& e) {
        if (err && err_len > 0) { std::strncpy(err, e.what(), err_len - 1); err[err_len - 1] = 0; }
        return -1;
    } catch (const std::exception& e) {
        if (err && err_len > 0) { std::strncpy(err, e.what(), err_len - 1); err[err_len - 1] = 0; }
        return -3;
    }
}

const char* kbsrc_ref_version() { return kbsrc::version(); }
}
