// WAV reading and writing for the kbsrc command-line tool (PCM 8/16/24/32, IEEE float 32/64,
// WAVE_FORMAT_EXTENSIBLE). Same formats, header layout and error messages as HongYue1/KBSRC src/io/wav.hpp,
// since the tool's output file is compared byte for byte.
#pragma once

#include <memory>
#include <string>
#include <vector>

namespace kbsrc::io {

struct Audio {
    int rate = 0, ch = 0;
    long long frames = 0;
    std::vector<double> d;  // interleaved, decoded (read_wav)
    int fmt_bits = 0;
    bool fmt_float = false;
    std::vector<unsigned char> raw;  // the data section as stored (read_wav_raw), frames * ch samples,
    std::shared_ptr<const void> map;  // unless it is read in place from a mapping of the file
    const unsigned char* mapped = nullptr;
    std::string sample_format;      // its sample format: "u8", "s16", "s24", "s32", "f32" or "f64"
    const unsigned char* bytes() const { return map ? mapped : raw.data(); }
};

Audio read_wav(const char* path);
// The same checks and header parsing as read_wav, but the samples stay as stored in the file (bytes(),
// sample_format); decode_wav fills d from them. The data section is mapped read-only where the file can be
// mapped (the copies to the GPU then read the page cache directly), else read into raw. A file truncated by
// another process while it is mapped ends the process with SIGBUS.
Audio read_wav_raw(const char* path);
void decode_wav(Audio& a);
// Fails when a WAV header in `format` cannot describe ch channels at this rate.
void check_wav_output(int ch, int rate, const std::string& format);
// y: planar samples. Integer formats are scaled, optionally TPDF-dithered (two uniform draws per sample from
// std::mt19937_64 seeded 12345, frame-major order), rounded in the current rounding mode and clipped.
void write_wav(const char* path, const std::vector<std::vector<double>>& y, int ch, long long frames, int rate,
               const std::string& format, bool dither, long long& clipped);

// Writes a WAV file of `frames` frames whose data section (interleaved samples in `format`) was produced
// elsewhere (the GPU packer); the header is the one write_wav produces.
void write_wav_data(const char* path, int ch, long long frames, int rate, const std::string& format,
                    const unsigned char* data, size_t bytes);

}  // namespace kbsrc::io
