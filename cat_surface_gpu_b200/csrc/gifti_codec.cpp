// GIFTI payload decoding on the host: the base64 text of a Base64Binary or
// GZipBase64Binary DataArray to the array's bytes.  A GZipBase64Binary payload
// is one zlib stream (RFC 1950); when its writer recorded the raw-deflate chunk
// lengths of a chunked stream (each chunk ended by a sync flush, the last by the
// final block), the chunks inflate on several threads and their Adler-32 sums
// are combined for the stream's check.  Plain C++ and zlib: the caller's
// interpreter lock is not held, so several files decode at once.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/catsurf_b200.h"
#include "errors.h"

namespace {

constexpr int8_t kBad = -1, kSpace = -2, kPad = -3;

struct Base64Table {
    int8_t value[256];
    Base64Table() {
        for (int c = 0; c < 256; ++c) value[c] = kBad;
        const char* alphabet = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
        for (int k = 0; k < 64; ++k) value[static_cast<unsigned char>(alphabet[k])] = static_cast<int8_t>(k);
        value[static_cast<unsigned char>(' ')] = value[static_cast<unsigned char>('\t')] = kSpace;
        value[static_cast<unsigned char>('\r')] = value[static_cast<unsigned char>('\n')] = kSpace;
        value[static_cast<unsigned char>('=')] = kPad;
    }
};

const Base64Table& table() {
    static const Base64Table t;
    return t;
}

// The sextet of each character pre-shifted to its place in a group of four;
// anything but the alphabet sets bit 24, so one test clears a whole group.
struct GroupTables {
    uint32_t shifted[4][256];
    GroupTables() {
        const int8_t* T = table().value;
        for (int c = 0; c < 256; ++c)
            for (int p = 0; p < 4; ++p)
                shifted[p][c] = T[c] >= 0 ? static_cast<uint32_t>(T[c]) << (18 - 6 * p) : 0x01000000u;
    }
};

const GroupTables& groups() {
    static const GroupTables g;
    return g;
}

// Decodes text[0, n) into out (capacity cap).  Whitespace may stand anywhere;
// '=' only as the last one or two characters of the last group of four.
// Returns the decoded length, or -1 with *why set.
long long base64_decode(const unsigned char* text, size_t n, unsigned char* out, size_t cap, std::string* why) {
    const int8_t* T = table().value;
    const uint32_t(*G)[256] = groups().shifted;
    uint32_t acc = 0;
    int have = 0, pads = 0;
    size_t o = 0;
    for (size_t i = 0; i < n;) {
        if (have == 0 && pads == 0) {
            // whole groups of four alphabet characters (the bulk of a payload)
            while (i + 4 <= n && o + 3 <= cap) {
                const uint32_t x = G[0][text[i]] | G[1][text[i + 1]] | G[2][text[i + 2]] | G[3][text[i + 3]];
                if (x >> 24) break;
                out[o] = static_cast<unsigned char>(x >> 16);
                out[o + 1] = static_cast<unsigned char>(x >> 8);
                out[o + 2] = static_cast<unsigned char>(x);
                o += 3;
                i += 4;
            }
            if (i >= n) break;
        }
        const int t = T[text[i]];
        if (t == kSpace) {
            ++i;
            continue;
        }
        if (t == kBad) {
            *why = "invalid base64 character at offset " + std::to_string(i);
            return -1;
        }
        if (t == kPad) {
            if (have < 2) {
                *why = "misplaced base64 padding at offset " + std::to_string(i);
                return -1;
            }
            ++pads;
            acc <<= 6;
        } else {
            if (pads) {
                *why = "base64 data after padding at offset " + std::to_string(i);
                return -1;
            }
            acc = (acc << 6) | static_cast<uint32_t>(t);
        }
        if (++have == 4) {
            const int bytes = 3 - pads;
            if (o + bytes > cap) {
                *why = "base64 payload longer than the array";
                return -1;
            }
            for (int k = 0; k < bytes; ++k) out[o++] = static_cast<unsigned char>(acc >> (16 - 8 * k));
            acc = 0;
            have = 0;
            if (pads) {
                for (++i; i < n; ++i)
                    if (T[text[i]] != kSpace) {
                        *why = "base64 data after padding at offset " + std::to_string(i);
                        return -1;
                    }
                return static_cast<long long>(o);
            }
        }
        ++i;
    }
    if (have != 0) {
        *why = "incorrect base64 padding";
        return -1;
    }
    return static_cast<long long>(o);
}

uInt piece(size_t left) { return static_cast<uInt>(std::min<size_t>(left, UINT_MAX)); }

// One zlib stream (header, deflate data, Adler-32) into exactly out_n bytes.
bool inflate_stream(const unsigned char* z, size_t zn, unsigned char* out, size_t out_n, uLong* check, std::string* why) {
    z_stream s;
    std::memset(&s, 0, sizeof(s));
    if (inflateInit(&s) != Z_OK) {
        *why = "zlib: cannot start an inflater";
        return false;
    }
    size_t in_left = zn, out_left = out_n;
    const unsigned char* ip = z;
    unsigned char* op = out;
    bool ok = false;
    for (;;) {
        if (s.avail_in == 0 && in_left) {
            s.next_in = const_cast<Bytef*>(ip);
            s.avail_in = piece(in_left);
            ip += s.avail_in;
            in_left -= s.avail_in;
        }
        if (s.avail_out == 0 && out_left) {
            s.next_out = op;
            s.avail_out = piece(out_left);
            op += s.avail_out;
            out_left -= s.avail_out;
        }
        const int r = inflate(&s, Z_NO_FLUSH);
        if (r == Z_STREAM_END) {
            ok = s.total_out == out_n;
            *check = s.adler;  // the stream's Adler-32, which inflate has verified
            if (!ok) *why = "GIFTI array holds " + std::to_string(s.total_out) + " bytes, header says " + std::to_string(out_n);
            break;
        }
        if (r == Z_OK) continue;
        if (r == Z_BUF_ERROR && s.avail_out == 0 && out_left == 0) {
            *why = "GIFTI array holds more than the " + std::to_string(out_n) + " bytes the header says";
        } else if (r == Z_BUF_ERROR && s.avail_in == 0 && in_left == 0) {
            *why = "zlib: truncated stream";
        } else {
            *why = std::string("zlib: ") + (s.msg ? s.msg : "invalid stream");
        }
        break;
    }
    inflateEnd(&s);
    return ok;
}

// One raw-deflate chunk into exactly out_n bytes; `last` chunks end the deflate
// stream, the others end at a block boundary with no output pending.
bool inflate_chunk(const unsigned char* z, size_t zn, unsigned char* out, size_t out_n, bool last) {
    if (zn > UINT_MAX || out_n > UINT_MAX) return false;
    z_stream s;
    std::memset(&s, 0, sizeof(s));
    if (inflateInit2(&s, -15) != Z_OK) return false;
    s.next_in = const_cast<Bytef*>(z);
    s.avail_in = static_cast<uInt>(zn);
    s.next_out = out;
    s.avail_out = static_cast<uInt>(out_n);
    int r = Z_OK;
    while (r == Z_OK) r = inflate(&s, Z_SYNC_FLUSH);
    bool ok = s.avail_in == 0 && s.avail_out == 0 && (last ? r == Z_STREAM_END : r == Z_BUF_ERROR);
    if (ok && !last) {
        unsigned char probe;
        s.next_out = &probe;
        s.avail_out = 1;
        r = inflate(&s, Z_SYNC_FLUSH);
        ok = s.avail_out == 1 && r != Z_STREAM_END;
    }
    inflateEnd(&s);
    return ok;
}

// The chunked form when the index fits the stream and the array size, else false
// (the caller inflates the one stream).
bool chunks_fit(const unsigned char* z, size_t zn, const long long* lengths, int n_chunks, long long chunk_bytes,
                size_t out_n) {
    if (!lengths || n_chunks < 2 || chunk_bytes <= 0 || zn < 6) return false;
    if ((z[0] * 256 + z[1]) % 31 != 0 || (z[0] & 0x0f) != 8 || (z[1] & 0x20)) return false;
    unsigned long long sum = 0;
    for (int k = 0; k < n_chunks; ++k) {
        if (lengths[k] <= 0) return false;
        sum += static_cast<unsigned long long>(lengths[k]);
    }
    const unsigned long long full = static_cast<unsigned long long>(n_chunks - 1) * static_cast<unsigned long long>(chunk_bytes);
    return sum == zn - 6 && out_n > full && out_n <= full + static_cast<unsigned long long>(chunk_bytes);
}

}  // namespace

extern "C" {

int csg_gifti_decode(const char* text, size_t text_bytes, int gzip, const long long* chunk_lengths, int n_chunks,
                     long long chunk_bytes, void* out, size_t out_bytes, unsigned int* adler32_out) {
    if ((text_bytes && !text) || (out_bytes && !out) || (gzip != 0 && gzip != 1) || n_chunks < 0)
        return csg::fail(CSG_ERR_ARG, "csg_gifti_decode: null buffer or bad gzip / chunk arguments");
    const unsigned char* src = reinterpret_cast<const unsigned char*>(text);
    unsigned char* dst = static_cast<unsigned char*>(out);
    std::string why;
    if (!gzip) {
        const long long n = base64_decode(src, text_bytes, dst, out_bytes, &why);
        if (n < 0) return csg::fail(CSG_ERR_FORMAT, "%s", why.c_str());
        if (static_cast<size_t>(n) != out_bytes)
            return csg::fail(CSG_ERR_FORMAT, "GIFTI array holds %lld bytes, header says %zu", n, out_bytes);
        if (adler32_out) {
            uLong sum = adler32(0L, Z_NULL, 0);
            for (size_t at = 0; at < out_bytes; at += UINT_MAX)
                sum = adler32(sum, dst + at, piece(out_bytes - at));
            *adler32_out = static_cast<unsigned int>(sum);
        }
        return CSG_OK;
    }
    // the compressed bytes, in a per-thread buffer that repeated reads reuse
    thread_local std::vector<unsigned char> buffer;
    if (buffer.size() < text_bytes / 4 * 3 + 3) buffer.resize(text_bytes / 4 * 3 + 3);
    const unsigned char* z = buffer.data();  // helper threads below read it through this pointer
    const long long zn = base64_decode(src, text_bytes, buffer.data(), buffer.size(), &why);
    if (zn < 0) return csg::fail(CSG_ERR_FORMAT, "%s", why.c_str());
    if (!chunks_fit(z, static_cast<size_t>(zn), chunk_lengths, n_chunks, chunk_bytes, out_bytes)) {
        uLong check = 0;
        if (!inflate_stream(z, static_cast<size_t>(zn), dst, out_bytes, &check, &why))
            return csg::fail(CSG_ERR_FORMAT, "%s", why.c_str());
        if (adler32_out) *adler32_out = static_cast<unsigned int>(check);
        return CSG_OK;
    }
    std::vector<size_t> start(n_chunks);
    start[0] = 2;
    for (int k = 1; k < n_chunks; ++k) start[k] = start[k - 1] + static_cast<size_t>(chunk_lengths[k - 1]);
    std::vector<uLong> sums(n_chunks);
    std::vector<char> good(n_chunks, 0);
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int k; (k = next.fetch_add(1)) < n_chunks;) {
            const size_t at = static_cast<size_t>(k) * static_cast<size_t>(chunk_bytes);
            const size_t size = k == n_chunks - 1 ? out_bytes - at : static_cast<size_t>(chunk_bytes);
            good[k] = inflate_chunk(z + start[k], static_cast<size_t>(chunk_lengths[k]), dst + at, size,
                                    k == n_chunks - 1);
            if (good[k]) sums[k] = adler32(adler32(0L, Z_NULL, 0), dst + at, static_cast<uInt>(size));
        }
    };
    // helpers beyond the calling thread come out of one budget of (cores - 1) shared by
    // every call in flight, so files decoded side by side do not oversubscribe the cores
    static std::atomic<int> helpers_in_use{0};
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int want = std::min({n_chunks, hw, 8}) - 1;
    int granted = 0;
    while (granted < want) {
        int used = helpers_in_use.load();
        if (used >= hw - 1) break;
        if (helpers_in_use.compare_exchange_weak(used, used + 1)) ++granted;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < granted; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    helpers_in_use.fetch_sub(granted);
    uLong sum = adler32(0L, Z_NULL, 0);
    for (int k = 0; k < n_chunks; ++k) {
        if (!good[k]) return csg::fail(CSG_ERR_FORMAT, "zlib: chunk %d does not match the deflate stream", k);
        const size_t at = static_cast<size_t>(k) * static_cast<size_t>(chunk_bytes);
        const size_t size = k == n_chunks - 1 ? out_bytes - at : static_cast<size_t>(chunk_bytes);
        sum = adler32_combine(sum, sums[k], static_cast<z_off_t>(size));
    }
    const unsigned char* tail = z + zn - 4;
    const uLong check = (static_cast<uLong>(tail[0]) << 24) | (static_cast<uLong>(tail[1]) << 16) |
                        (static_cast<uLong>(tail[2]) << 8) | tail[3];
    if (sum != check) return csg::fail(CSG_ERR_FORMAT, "zlib: incorrect data check");
    if (adler32_out) *adler32_out = static_cast<unsigned int>(sum);
    return CSG_OK;
}

}  // extern "C"
