// WAV file I/O for the command-line tool; behaviour of HongYue1/KBSRC src/io/wav.cpp:274-418.
#include "wav.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>

#include <sys/mman.h>
#include <unistd.h>

namespace kbsrc::io {
namespace {

[[noreturn]] void fail(const char* m) { throw std::runtime_error(m); }

struct FileCloser {
    FILE* f = nullptr;
    ~FileCloser() {
        if (f) std::fclose(f);
    }
};

unsigned le16(const uint8_t* p) { return (unsigned)p[0] | (unsigned)p[1] << 8; }
uint32_t le32(const uint8_t* p) { return (uint32_t)le16(p) | (uint32_t)le16(p + 2) << 16; }

int bytes_per_sample(const std::string& fmt) { return fmt == "f64" ? 8 : fmt == "s24" ? 3 : fmt == "s16" ? 2 : 4; }

}  // namespace

namespace {
// Decodes m samples of `bps` bytes (tag 1 PCM or tag 3 IEEE float) from p into o.
void decode_samples(const uint8_t* p, size_t m, bool is_float, int bits, int bps, double* o) {
    if (is_float && bits == 64) {
        std::memcpy(o, p, 8 * m);
    } else if (is_float) {
        for (size_t k = 0; k < m; k++) {
            float v;
            std::memcpy(&v, p + 4 * k, 4);
            o[k] = v;
        }
    } else if (bps == 1) {
        for (size_t k = 0; k < m; k++) o[k] = ((int)p[k] - 128) / 128.0;
    } else if (bps == 2) {
        for (size_t k = 0; k < m; k++) o[k] = (int16_t)(p[2 * k] | p[2 * k + 1] << 8) / 32768.0;
    } else if (bps == 3) {
        for (size_t k = 0; k < m; k++) {
            int32_t v = p[3 * k] | p[3 * k + 1] << 8 | p[3 * k + 2] << 16;
            if (v & 0x800000) v -= 1 << 24;
            o[k] = v / 8388608.0;
        }
    } else {
        for (size_t k = 0; k < m; k++) {
            const uint8_t* q = p + 4 * k;
            o[k] = (int32_t)(q[0] | q[1] << 8 | q[2] << 16 | (uint32_t)q[3] << 24) / 2147483648.0;
        }
    }
}

int sample_bytes(const Audio& a) { return a.fmt_float ? a.fmt_bits / 8 : (a.fmt_bits + 7) / 8; }

// Header checks and the data section; raw: keep the bytes, else decode them.
Audio read_impl(const char* path, bool raw) {
    FileCloser fc{std::fopen(path, "rb")};
    FILE* f = fc.f;
    if (!f) fail("cannot open input");
    fseeko(f, 0, SEEK_END);
    const long long size = ftello(f);
    fseeko(f, 0, SEEK_SET);
    uint8_t riff[12];
    if (size < 12 || std::fread(riff, 1, 12, f) != 12 || std::memcmp(riff, "RIFF", 4) ||
        std::memcmp(riff + 8, "WAVE", 4))
        fail("not a RIFF/WAVE file");
    long long pos = 12, data_pos = -1, data_len = 0;
    int tag = 0, ch = 0, bits = 0, align = 0;
    uint32_t rate = 0;
    bool have_fmt = false;
    while (pos + 8 <= size) {
        uint8_t hdr[8];
        fseeko(f, pos, SEEK_SET);
        if (std::fread(hdr, 1, 8, f) != 8) break;
        const uint32_t len = le32(hdr + 4);
        const long long body = pos + 8;
        if (!std::memcmp(hdr, "fmt ", 4)) {
            uint8_t fm[40] = {};
            const size_t n = std::fread(fm, 1, std::min<uint32_t>(len, 40), f);
            if (n < 16) fail("bad fmt chunk");
            have_fmt = true;
            tag = (int)le16(fm);
            ch = (int)le16(fm + 2);
            rate = le32(fm + 4);
            align = (int)le16(fm + 12);
            bits = (int)le16(fm + 14);
            if (tag == 0xFFFE && n >= 26) tag = (int)le16(fm + 24);
        } else if (!std::memcmp(hdr, "data", 4)) {
            data_pos = body;
            data_len = std::min<long long>(len, size - body);
            if (len == 0xFFFFFFFFu || len == 0) data_len = size - body;
            break;
        }
        pos = body + len + (len & 1);
    }
    if (!have_fmt || data_pos < 0) fail("missing fmt/data chunk");
    if (!ch) fail("invalid WAV channel count");
    if (!rate || rate > INT_MAX) fail("invalid WAV sample rate");
    if (align <= 0 || align % ch) fail("invalid WAV block alignment");
    if (!(tag == 1 || (tag == 3 && (bits == 32 || bits == 64)))) fail("unsupported WAV format (need PCM or IEEE float)");
    const int bps = align / ch;
    if (tag == 1 && (bps < 1 || bps > 4 || (bits + 7) / 8 != bps)) fail("unsupported PCM width");
    if (tag == 3 && bits != 8 * bps) fail("IEEE float sample size does not match the block alignment");
    Audio a;
    a.rate = (int)rate;
    a.ch = ch;
    a.fmt_bits = bits;
    a.fmt_float = tag == 3;
    a.frames = data_len / align;
    static const char* const pcm[] = {"u8", "s16", "s24", "s32"};
    a.sample_format = a.fmt_float ? (bits == 64 ? "f64" : "f32") : pcm[bps - 1];
    const size_t n = (size_t)a.frames * ch;
    fseeko(f, data_pos, SEEK_SET);
    if (raw) {
        if (n) {
            const long long page = sysconf(_SC_PAGESIZE), off = data_pos / page * page;
            const size_t len = (size_t)(data_pos - off) + n * bps;
            void* m = mmap(nullptr, len, PROT_READ, MAP_PRIVATE, fileno(f), (off_t)off);
            if (m != MAP_FAILED) {
                madvise(m, len, MADV_SEQUENTIAL);
                a.map = std::shared_ptr<const void>(m, [len](const void* q) { munmap(const_cast<void*>(q), len); });
                a.mapped = static_cast<const unsigned char*>(m) + (data_pos - off);
                return a;
            }
        }
        a.raw.resize(n * bps);
        if (n && std::fread(a.raw.data(), (size_t)bps, n, f) != n) fail("read error");
        return a;
    }
    a.d.resize(n);
    const size_t chunk = (size_t)1 << 20;
    std::vector<uint8_t> buf(chunk * bps);
    for (size_t k0 = 0; k0 < n; k0 += chunk) {
        const size_t m = std::min(chunk, n - k0);
        if (std::fread(buf.data(), (size_t)bps, m, f) != m) fail("read error");
        decode_samples(buf.data(), m, a.fmt_float, bits, bps, a.d.data() + k0);
    }
    return a;
}
}  // namespace

Audio read_wav(const char* path) { return read_impl(path, false); }
Audio read_wav_raw(const char* path) { return read_impl(path, true); }

void decode_wav(Audio& a) {
    const size_t n = (size_t)a.frames * a.ch;
    a.d.resize(n);
    if (n) decode_samples(a.bytes(), n, a.fmt_float, a.fmt_bits, sample_bytes(a), a.d.data());
}

void check_wav_output(int ch, int rate, const std::string& fmt) {
    const long long frame = (long long)ch * bytes_per_sample(fmt);
    if (ch < 1 || frame > 0xFFFF) fail("too many channels for a WAV file in this format");
    if (rate < 1 || rate * frame > 0xFFFFFFFFLL) fail("sample rate too high for a WAV file with this many channels");
}

namespace {
// The RIFF/WAVE header for `frames` frames of `ch` channels in `fmt` (reference wav.cpp:355-371)
std::vector<uint8_t> wav_header(int ch, long long frames, int rate, const std::string& fmt, size_t& data_bytes) {
    check_wav_output(ch, rate, fmt);
    const bool is_float = fmt == "f64" || fmt == "f32";
    const int bits = fmt == "f64" ? 64 : fmt == "f32" ? 32 : fmt == "s32" ? 32 : fmt == "s24" ? 24 : 16;
    const int bps = bits / 8, align = ch * bps;
    if (frames < 0 || frames > (0xFFFFFFFFLL - 80) / align) fail("output too large for WAV (4 GB limit)");
    data_bytes = (size_t)frames * align;
    std::vector<uint8_t> hdr;
    auto put16 = [&](unsigned v) { hdr.push_back(v & 255); hdr.push_back(v >> 8 & 255); };
    auto put32 = [&](uint32_t v) { put16(v & 0xFFFF); put16(v >> 16); };
    auto tag = [&](const char* s) { hdr.insert(hdr.end(), s, s + 4); };
    const bool extensible = ch > 2 || (!is_float && bits > 16);
    const unsigned fmt_len = extensible ? 40 : (is_float ? 18 : 16);
    const uint32_t riff = 4 + 8 + fmt_len + (is_float ? 12 : 0) + 8 + (uint32_t)data_bytes + (data_bytes & 1);
    tag("RIFF"); put32(riff); tag("WAVE"); tag("fmt "); put32(fmt_len);
    put16(extensible ? 0xFFFE : is_float ? 3 : 1);
    put16(ch); put32(rate); put32((uint32_t)rate * align); put16(align); put16(bits);
    if (fmt_len >= 18) put16(extensible ? 22 : 0);
    if (extensible) {
        put16(bits);
        put32(ch == 1 ? 4 : ch == 2 ? 3 : 0);  // channel mask: mono = FC, stereo = FL|FR, else unassigned
        put16(is_float ? 3 : 1);
        static const uint8_t guid_tail[14] = {0x00, 0x00, 0x00, 0x00, 0x10, 0x00, 0x80,
                                              0x00, 0x00, 0xAA, 0x00, 0x38, 0x9B, 0x71};
        hdr.insert(hdr.end(), guid_tail, guid_tail + 14);
    }
    if (is_float) { tag("fact"); put32(4); put32((uint32_t)frames); }
    tag("data"); put32((uint32_t)data_bytes);
    return hdr;
}
}  // namespace

void write_wav(const char* path, const std::vector<std::vector<double>>& y, int ch, long long frames, int rate,
               const std::string& fmt, bool dither, long long& clipped) {
    size_t data_bytes = 0;
    const std::vector<uint8_t> hdr = wav_header(ch, frames, rate, fmt, data_bytes);
    const int bps = fmt == "f64" ? 8 : fmt == "f32" ? 4 : fmt == "s32" ? 4 : fmt == "s24" ? 3 : 2;
    const int align = ch * bps;
    FileCloser fc{std::fopen(path, "wb")};
    FILE* f = fc.f;
    if (!f) fail("cannot open output");
    if (std::fwrite(hdr.data(), 1, hdr.size(), f) != hdr.size()) fail("write error");
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> U(-0.5, 0.5);
    const double scale = bps == 2 ? 32768.0 : bps == 3 ? 8388608.0 : 2147483648.0;
    clipped = 0;
    const long long chunk = std::max(1, std::min(1 << 16, (4 << 20) / align));
    std::vector<uint8_t> buf((size_t)chunk * align);
    for (long long f0 = 0; f0 < frames; f0 += chunk) {
        const long long nf = std::min(chunk, frames - f0);
        uint8_t* p = buf.data();
        for (long long i = f0; i < f0 + nf; ++i)
            for (int c = 0; c < ch; ++c, p += bps) {
                const double x = y[c][i];
                if (fmt == "f64") {
                    std::memcpy(p, &x, 8);
                } else if (fmt == "f32") {
                    const float v = (float)x;
                    std::memcpy(p, &v, 4);
                } else {
                    double v = x * scale;
                    if (dither) v += U(rng) + U(rng);
                    v = std::nearbyint(v);
                    if (v > scale - 1) { v = scale - 1; ++clipped; }
                    else if (v < -scale) { v = -scale; ++clipped; }
                    const int64_t iv = std::isnan(v) ? 0 : (int64_t)v;  // NaN is written as zero
                    for (int t = 0; t < bps; ++t) p[t] = (iv >> (8 * t)) & 255;
                }
            }
        const size_t nb = (size_t)(p - buf.data());
        if (std::fwrite(buf.data(), 1, nb, f) != nb) fail("write error");
    }
    if (data_bytes & 1) std::fputc(0, f);
    fc.f = nullptr;
    if (std::fclose(f)) fail("write error");
}

void write_wav_data(const char* path, int ch, long long frames, int rate, const std::string& fmt,
                    const unsigned char* data, size_t bytes) {
    size_t data_bytes = 0;
    const std::vector<uint8_t> hdr = wav_header(ch, frames, rate, fmt, data_bytes);
    if (bytes != data_bytes) fail("internal error: WAV data size");
    FileCloser fc{std::fopen(path, "wb")};
    FILE* f = fc.f;
    if (!f) fail("cannot open output");
    if (std::fwrite(hdr.data(), 1, hdr.size(), f) != hdr.size()) fail("write error");
    if (bytes && std::fwrite(data, 1, bytes, f) != bytes) fail("write error");
    if (data_bytes & 1) std::fputc(0, f);
    fc.f = nullptr;
    if (std::fclose(f)) fail("write error");
}

}  // namespace kbsrc::io
