// KBSRC on B200 - Kaiser-Bessel sample-rate converter, public C++ API.
//
// Same API as HongYue1/KBSRC 1.3.0 include/kbsrc/kbsrc.hpp:8-45 (Precision, Options, Stats, resample,
// version), so code written against the reference library builds unchanged. The block engine runs on the
// GPU (sm_100a); its output is byte-identical to the reference CPU engines in all three precisions.
#pragma once

#include <vector>

namespace kbsrc {

enum class Precision {
    Fast,        // float64 pipeline
    Exact,       // double-double (~106-bit) pipeline
    LongDouble,  // x87 80-bit extended; the GPU emulates its arithmetic in integers, bit for bit
    SplitTC,     // not in the reference: the Exact plan with its FFT stages as tensor-core contractions of 8-bit
                 // digit slices in int8 (split precision); within float64 rounding of Exact, not byte-identical
    SplitTC16,   // not in the reference: the same with the digit slices in f16 (f32 accumulation); same output
};

struct Options {
    Precision precision = Precision::Exact;
    double length = 0.2;    // one-sided kernel length, seconds; the transition band is inversely proportional
    double beta = 40.0;     // Kaiser window beta
    int threads = 0;        // host threads for kernel design and LPC, 0 = automatic
    int block = 0;          // block size factor, 0 = automatic
    bool lpc_edges = true;  // Burg LPC extrapolation at the signal edges
};

struct Stats {
    long long p = 0, q = 0;     // rate ratio P/Q
    long long taps = 0;         // kernel taps at the kernel rate
    int block = 0, threads = 0;
    bool general_fold = false;  // near-unity ratio path
    double design_seconds = 0, process_seconds = 0;
    double passband = 0, stopband = 0;  // band edges in Hz
    const char* isa = "";       // engine used: "sm_100a" (GPU), "generic" for the equal-rate copy
};

// Resamples interleaved input (frames x channels) from rate_in to rate_out and returns planar output, one
// vector per channel of ceil(frames * rate_out / rate_in) samples. Throws std::invalid_argument on bad
// arguments (same messages as the reference) and std::runtime_error when the GPU engine cannot run the plan.
// Exact computes in round-to-nearest whatever the caller's mode, which is restored on return or throw.
std::vector<std::vector<double>> resample(const double* interleaved, long long frames, int channels,
                                          int rate_in, int rate_out, const Options& options = {},
                                          Stats* stats = nullptr);

// The same conversion followed by the output step of a WAV writer, on the GPU: returns the data section of a WAV
// file in `format` ("f64", "f32", "s32", "s24" or "s16"), interleaved little-endian; integer formats are scaled,
// TPDF-dithered when `dither` (std::mt19937_64 seeded 12345, two uniform(-0.5, 0.5) draws per sample), rounded and
// clipped, with the clipped count in `clipped` - byte for byte what the reference's kbsrc tool writes. Equal rates
// (no conversion) throw std::invalid_argument.
std::vector<unsigned char> resample_wav_data(const double* interleaved, long long frames, int channels, int rate_in,
                                             int rate_out, const char* format, bool dither, long long& clipped,
                                             const Options& options = {}, Stats* stats = nullptr);

// resample_wav_data on the data section of a PCM or float WAV file as it is stored: `pcm` holds frames x channels
// samples of `sample_format` ("u8", "s16", "s24", "s32", "f32" or "f64", little-endian). The GPU decodes every
// sample as the reference's WAV reader does while it gathers blocks (a 24-bit file moves 3 bytes per sample to
// the device instead of 8); the host decodes only the frames the LPC edges need. Output and exceptions as
// resample_wav_data.
std::vector<unsigned char> resample_wav_pcm(const void* pcm, const char* sample_format, long long frames,
                                            int channels, int rate_in, int rate_out, const char* format, bool dither,
                                            long long& clipped, const Options& options = {}, Stats* stats = nullptr);

// Not in the reference: the same conversion with its block loop split across CUDA devices in contiguous block
// ranges, one engine and one host thread per device; each device receives only its input span (its blocks' inputs,
// halo included) and returns its output range, and nothing moves between devices. `devices` lists CUDA device
// indices (one may appear more than once). Output, exceptions and rounding-mode handling as resample().
std::vector<std::vector<double>> resample_devices(const double* interleaved, long long frames, int channels,
                                                  int rate_in, int rate_out, const int* devices, int ndevices,
                                                  const Options& options = {}, Stats* stats = nullptr);

// Starts the GPU's initialisation (CUDA context, kernel attributes) on a background thread and returns at once.
// Optional: the first conversion starts it too, overlapped with its host-side LPC and kernel taps; a caller that
// knows a conversion is coming (a tool about to read its input file) can start it earlier. Not in the reference.
void warm_up();

const char* version();

}  // namespace kbsrc
