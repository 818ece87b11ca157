// CRC32 (zlib's polynomial, reflected) arithmetic shared by the inflater and the compressor.
//
// Spans are checksummed in parallel: each part gets a raw column (the CRC register run over its
// bytes from zero, no pre- or post-inversion), and columns are joined with
// raw(A || B) = raw(A) * x^(8 |B|) + raw(B) in GF(2)[x] modulo the polynomial, the combination
// zlib's crc32_combine is built on.  The zlib CRC of n bytes is then
// raw ^ (0xFFFFFFFF * x^(8 n)) ^ 0xFFFFFFFF.
#pragma once

#include <cstdint>

namespace cb {

// Reflected representation of GF(2)[x] modulo the CRC-32 polynomial: bit 31 is x^0.
constexpr uint32_t POLY = 0xEDB88320u;

__host__ __device__ constexpr uint32_t gf_mul(uint32_t a, uint32_t b) {
    uint32_t p = 0;
    for (int i = 0; i < 32; i++) {
        if (a & 0x80000000u) p ^= b;
        a <<= 1;
        b = (b & 1u) ? (b >> 1) ^ POLY : (b >> 1);
    }
    return p;
}

struct CrcConst {
    uint32_t x2n[32];   // x^(2^k)
    uint32_t seg[5];    // x^(8 * 32 * 2^k): shifts that combine the lane columns
    uint32_t k992;      // x^(8 * 992): one window minus one column
};

__host__ __device__ constexpr uint32_t xpow_from(const uint32_t* x2n, unsigned long long n) {
    uint32_t r = 0x80000000u;  // x^0
    for (int k = 0; n; n >>= 1, k++)
        if (n & 1) r = gf_mul(r, x2n[k]);
    return r;
}

constexpr CrcConst make_crc_const() {
    CrcConst c{};
    uint32_t p = 0x40000000u;  // x^1
    for (int k = 0; k < 32; k++) {
        c.x2n[k] = p;
        p = gf_mul(p, p);
    }
    for (int k = 0; k < 5; k++) c.seg[k] = xpow_from(c.x2n, 8ull * 32ull * (1ull << k));
    c.k992 = xpow_from(c.x2n, 8ull * 992ull);
    return c;
}

// One copy per translation unit (static: the host-side shadows of two units do not collide).
static __constant__ CrcConst kCrc = make_crc_const();

// zlib's CRC of n bytes from their raw column.
__device__ __forceinline__ uint32_t crc_finish(uint32_t raw, unsigned long long n) {
    return raw ^ gf_mul(0xFFFFFFFFu, xpow_from(kCrc.x2n, 8ull * n)) ^ 0xFFFFFFFFu;
}

// Slice-by-8 CRC tables (table t: the CRC of a byte followed by t zero bytes).
__device__ inline void init_crc8(uint32_t (*crc8)[256]) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        uint32_t c = (uint32_t)i;
        for (int k = 0; k < 8; k++) c = (c & 1u) ? (c >> 1) ^ POLY : c >> 1;
        crc8[0][i] = c;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        uint32_t c = crc8[0][i];
        for (int t = 1; t < 8; t++) {
            c = (c >> 8) ^ crc8[0][c & 255];
            crc8[t][i] = c;
        }
    }
}

// The raw column after 8 more bytes (w0 = bytes 0-3, w1 = bytes 4-7, little-endian).
__device__ __forceinline__ uint32_t crc_step8(const uint32_t (*T)[256], uint32_t c, uint32_t w0, uint32_t w1) {
    c ^= w0;
    return T[7][c & 255] ^ T[6][(c >> 8) & 255] ^ T[5][(c >> 16) & 255] ^ T[4][c >> 24] ^ T[3][w1 & 255] ^
           T[2][(w1 >> 8) & 255] ^ T[1][(w1 >> 16) & 255] ^ T[0][w1 >> 24];
}

}  // namespace cb
