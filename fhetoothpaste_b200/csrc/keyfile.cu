// Key files: a versioned, self-describing container for the keys this library
// consumes (blind-rotation keys, RLWE/automorphism/packing key-switching keys,
// LWE key-switching keys), in the reference's own in-memory layouts, and for
// batches of LWE / RLWE ciphertexts. The
// reference keeps keys only in memory; this lets a key be generated once on a
// host, stored, shipped and uploaded to a GPU context with its parameters and
// integrity checked. Host code only.
//
// File layout (little-endian), 128-byte header then the payload:
//   0   char[8]  magic "TPKEYv1\0"
//   8   u32      header bytes (128)
//   12  u32      kind (tp_key_kind)
//   16  u32      variant (blind rotation: tp_br_variant; RLWE batch: 0 coefficients,
//                1 NTT domain; else 0)
//   20  u32      ring dimension N (LWE key switch: n_in)
//   24  u32      LWE dimension (blind rotation: n; LWE key switch: n_out; else 0)
//   28  u32      gadget digits
//   32  u64      modulus
//   40  u64      gadget basis
//   48  u32      automorphism index (kind TP_KEY_AUTOMORPHISM), ciphertext count (TP_CT_*);
//                else 0
//   52  u32      layout tag (1: the reference's layout, NTT-domain words in
//                Solinas bit-reversed slot order)
//   56  u64      payload words
//   64  u8[32]   SHA-256 of the payload bytes
//   96  u8[32]   zero
//   128 u64[words] payload
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "br_launch.h"
#include "toothpaste_gpu.h"

namespace {

// SHA-256 as specified in FIPS 180-4 (sections 4.1.2, 4.2.2, 5.1.1, 6.2).
class Sha256 {
public:
    Sha256() { reset(); }
    void update(const uint8_t* p, size_t n) {
        total_ += n;
        while (n) {
            const size_t take = std::min(n, 64 - fill_);
            std::memcpy(buf_ + fill_, p, take);
            fill_ += take;
            p += take;
            n -= take;
            if (fill_ == 64) {
                block(buf_);
                fill_ = 0;
            }
        }
    }
    void finish(uint8_t out[32]) {
        const uint64_t bits = total_ * 8;
        const uint8_t one = 0x80, zero = 0;
        update(&one, 1);
        while (fill_ != 56) update(&zero, 1);
        uint8_t len[8];
        for (int i = 0; i < 8; ++i) len[i] = (uint8_t)(bits >> (56 - 8 * i));
        update(len, 8);
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 4; ++j) out[4 * i + j] = (uint8_t)(h_[i] >> (24 - 8 * j));
    }

private:
    static uint32_t rotr(uint32_t x, int r) { return (x >> r) | (x << (32 - r)); }
    void reset() {
        static const uint32_t init[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                         0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
        std::memcpy(h_, init, sizeof h_);
        fill_ = 0;
        total_ = 0;
    }
    void block(const uint8_t* b) {
        static const uint32_t k[64] = {
            0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
            0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
            0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
            0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
            0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
            0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
            0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
            0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
        uint32_t w[64];
        for (int i = 0; i < 16; ++i)
            w[i] = (uint32_t)b[4 * i] << 24 | (uint32_t)b[4 * i + 1] << 16 | (uint32_t)b[4 * i + 2] << 8 | b[4 * i + 3];
        for (int i = 16; i < 64; ++i) {
            const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
            const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        uint32_t a = h_[0], bb = h_[1], c = h_[2], d = h_[3], e = h_[4], f = h_[5], g = h_[6], h = h_[7];
        for (int i = 0; i < 64; ++i) {
            const uint32_t t1 = h + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + k[i] + w[i];
            const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & bb) ^ (a & c) ^ (bb & c));
            h = g;
            g = f;
            f = e;
            e = d + t1;
            d = c;
            c = bb;
            bb = a;
            a = t1 + t2;
        }
        h_[0] += a;
        h_[1] += bb;
        h_[2] += c;
        h_[3] += d;
        h_[4] += e;
        h_[5] += f;
        h_[6] += g;
        h_[7] += h;
    }
    uint32_t h_[8];
    uint8_t buf_[64];
    size_t fill_;
    uint64_t total_;
};

constexpr char kMagic[8] = {'T', 'P', 'K', 'E', 'Y', 'v', '1', 0};
constexpr uint32_t kHeaderBytes = 128;
constexpr uint32_t kLayoutReference = 1;

template <class T>
void put(uint8_t* h, size_t off, T v) {
    for (size_t i = 0; i < sizeof(T); ++i) h[off + i] = (uint8_t)((uint64_t)v >> (8 * i));
}
template <class T>
T get(const uint8_t* h, size_t off) {
    uint64_t v = 0;
    for (size_t i = 0; i < sizeof(T); ++i) v |= (uint64_t)h[off + i] << (8 * i);
    return (T)v;
}

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

void payload_sha(const uint64_t* words, uint64_t count, uint8_t out[32]) {
    Sha256 s;
    std::vector<uint8_t> buf;
    const uint64_t chunk = 1 << 16;
    buf.resize(chunk * 8);
    for (uint64_t i = 0; i < count; i += chunk) {
        const uint64_t n = std::min(chunk, count - i);
        for (uint64_t j = 0; j < n; ++j) put<uint64_t>(buf.data(), 8 * j, words[i + j]);
        s.update(buf.data(), n * 8);
    }
    s.finish(out);
}

tp_status read_header(FILE* f, const char* path, tp_key_info* info, uint8_t sha[32]) {
    uint8_t h[kHeaderBytes];
    if (std::fread(h, 1, kHeaderBytes, f) != kHeaderBytes)
        return tp::set_error(TP_ERR_LAYOUT, "%s: shorter than a key-file header", path);
    if (std::memcmp(h, kMagic, 8) != 0) return tp::set_error(TP_ERR_LAYOUT, "%s: not a key file (bad magic)", path);
    if (get<uint32_t>(h, 8) != kHeaderBytes) return tp::set_error(TP_ERR_LAYOUT, "%s: unsupported header size", path);
    if (get<uint32_t>(h, 52) != kLayoutReference) return tp::set_error(TP_ERR_LAYOUT, "%s: unknown layout tag", path);
    info->kind = get<uint32_t>(h, 12);
    info->variant = get<uint32_t>(h, 16);
    info->ring_dim = get<uint32_t>(h, 20);
    info->lwe_dim = get<uint32_t>(h, 24);
    info->digits = get<uint32_t>(h, 28);
    info->modulus = get<uint64_t>(h, 32);
    info->basis = get<uint64_t>(h, 40);
    info->index = get<uint32_t>(h, 48);
    info->words = get<uint64_t>(h, 56);
    std::memcpy(sha, h + 64, 32);
    return TP_OK;
}

}  // namespace

extern "C" {

tp_status tp_key_file_write(const char* path, const tp_key_info* info, const uint64_t* words) {
    if (!path || !info || (!words && info->words)) return tp::set_error(TP_ERR_PARAM, "null argument");
    if (info->kind == TP_CT_LWE || info->kind == TP_CT_RLWE) {
        const uint64_t row = info->kind == TP_CT_LWE ? info->lwe_dim + 1ull : 2ull * info->ring_dim;
        if (info->kind == TP_CT_RLWE && info->variant > 1)
            return tp::set_error(TP_ERR_PARAM, "RLWE batch domain must be 0 (coefficients) or 1 (NTT)");
        if ((uint64_t)info->index * row != info->words)
            return tp::set_error(TP_ERR_PARAM, "ciphertext batch: %llu words are not %u rows of %llu words",
                                 (unsigned long long)info->words, info->index, (unsigned long long)row);
    }
    uint8_t h[kHeaderBytes] = {};
    std::memcpy(h, kMagic, 8);
    put<uint32_t>(h, 8, kHeaderBytes);
    put<uint32_t>(h, 12, info->kind);
    put<uint32_t>(h, 16, info->variant);
    put<uint32_t>(h, 20, info->ring_dim);
    put<uint32_t>(h, 24, info->lwe_dim);
    put<uint32_t>(h, 28, info->digits);
    put<uint64_t>(h, 32, info->modulus);
    put<uint64_t>(h, 40, info->basis);
    put<uint32_t>(h, 48, info->index);
    put<uint32_t>(h, 52, kLayoutReference);
    put<uint64_t>(h, 56, info->words);
    payload_sha(words, info->words, h + 64);
    File f;
    f.f = std::fopen(path, "wb");
    if (!f.f) return tp::set_error(TP_ERR_PARAM, "%s: cannot open for writing", path);
    bool ok = std::fwrite(h, 1, kHeaderBytes, f.f) == kHeaderBytes;
    std::vector<uint8_t> buf(1 << 19);
    for (uint64_t i = 0; ok && i < info->words; i += buf.size() / 8) {
        const uint64_t n = std::min<uint64_t>(buf.size() / 8, info->words - i);
        for (uint64_t j = 0; j < n; ++j) put<uint64_t>(buf.data(), 8 * j, words[i + j]);
        ok = std::fwrite(buf.data(), 8, n, f.f) == n;
    }
    if (!ok || std::fflush(f.f) != 0) return tp::set_error(TP_ERR_PARAM, "%s: write failed", path);
    return TP_OK;
}

tp_status tp_key_file_info(const char* path, tp_key_info* info) {
    if (!path || !info) return tp::set_error(TP_ERR_PARAM, "null argument");
    File f;
    f.f = std::fopen(path, "rb");
    if (!f.f) return tp::set_error(TP_ERR_PARAM, "%s: cannot open", path);
    uint8_t sha[32];
    return read_header(f.f, path, info, sha);
}

tp_status tp_key_file_read(const char* path, tp_key_info* info, uint64_t* words, uint64_t capacity) {
    if (!path || !info || !words) return tp::set_error(TP_ERR_PARAM, "null argument");
    File f;
    f.f = std::fopen(path, "rb");
    if (!f.f) return tp::set_error(TP_ERR_PARAM, "%s: cannot open", path);
    uint8_t sha[32], got[32];
    tp_status s = read_header(f.f, path, info, sha);
    if (s != TP_OK) return s;
    if (info->words > capacity)
        return tp::set_error(TP_ERR_PARAM, "%s: %llu words do not fit the %llu-word buffer", path,
                            (unsigned long long)info->words, (unsigned long long)capacity);
    std::vector<uint8_t> buf(1 << 19);
    for (uint64_t i = 0; i < info->words; i += buf.size() / 8) {
        const uint64_t n = std::min<uint64_t>(buf.size() / 8, info->words - i);
        if (std::fread(buf.data(), 8, n, f.f) != n) return tp::set_error(TP_ERR_LAYOUT, "%s: truncated payload", path);
        for (uint64_t j = 0; j < n; ++j) words[i + j] = get<uint64_t>(buf.data(), 8 * j);
    }
    payload_sha(words, info->words, got);
    if (std::memcmp(sha, got, 32) != 0) return tp::set_error(TP_ERR_LAYOUT, "%s: payload SHA-256 does not match", path);
    return TP_OK;
}

}  // extern "C"
