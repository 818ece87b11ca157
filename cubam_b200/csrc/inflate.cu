// Raw-DEFLATE inflater for BGZF members on B200 (sm_100a), with the CRC32 and ISIZE checks.
//
// Replaces cubam's call of nvcompBatchedDeflateDecompressAsync and its status/size check
// (src/cubam/bgzf.py:587-611); the CRC32 check is new (cubam's reader does not check it,
// docs/reading.md:48-51).  DEFLATE itself is RFC 1951.
//
// Design (one warp per member, persistent grid, work queue):
//  * The warp decodes in lock step: every lane holds the same 64-bit bit buffer.  Lane l keeps
//    word l of the current 128-byte group of input in a register (loaded coalesced); refills take
//    the next word with __shfl_sync, and the next group is prefetched while this one is consumed.
//  * Huffman tables live in shared memory, one set per warp: a 2^LB-entry literal/length table
//    and a 2^DB-entry distance table.  Codes longer than the root bits take a canonical slow path
//    (count/symbol arrays).  Tables are built by the 32 lanes together (__match_any_sync ranks).
//  * Output goes to a per-warp 4 KB ring in shared memory; back-references up to RING-258 bytes
//    read the ring, farther ones read the already written output.  The ring is flushed to HBM one
//    1 KB window at a time with 16-byte stores.  Windows are aligned to the END of the member, so
//    the CRC32 is computed window by window with slice-by-8 tables: lane l folds bytes
//    [32l, 32l+32) of every window into its own column register, and the 32 columns are combined
//    once per member (GF(2) arithmetic modulo the CRC polynomial).
//  * Every loop is bounded by the member's sizes: output beyond ISIZE, a distance before the start,
//    bits read beyond the payload, bad code lengths and invalid symbols are per-member errors.

#include "common.cuh"

namespace cb {
namespace infl {

constexpr int LB = 10;                  // literal/length root bits
constexpr int DB = 8;                   // distance root bits
constexpr int CLB = 7;                  // code-length code bits
constexpr int RING = 4096;              // output ring per warp
constexpr int RMASK = RING - 1;
constexpr int WIN = 1024;               // flush / CRC window
constexpr int DMAX_RING = RING - 258;   // longest distance served from the ring
constexpr int WARPS = 4;                // warps per CTA

static_assert(RING > WIN + 2 * 258, "ring too small for the flush window");
static_assert(WIN == 32 * 32, "one 32-byte CRC column per lane");

enum : uint32_t { K_LIT = 0, K_LEN = 1, K_EOB = 2, K_SLOW = 3, K_BAD = 4 };

__device__ __forceinline__ uint32_t entry(uint32_t nbits, uint32_t kind, uint32_t extra, uint32_t value) {
    return nbits | (kind << 5) | (extra << 8) | (value << 16);
}
__device__ __forceinline__ uint32_t e_bits(uint32_t e) { return e & 31; }
__device__ __forceinline__ uint32_t e_kind(uint32_t e) { return (e >> 5) & 7; }
__device__ __forceinline__ uint32_t e_extra(uint32_t e) { return (e >> 8) & 15; }
__device__ __forceinline__ uint32_t e_value(uint32_t e) { return e >> 16; }

// RFC 1951 3.2.5: length and distance bases and extra bits.
__constant__ uint16_t kLenBase[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                      31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
__constant__ uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
__constant__ uint16_t kDistBase[30] = {1,   2,   3,   4,   5,   7,    9,    13,   17,   25,   33,   49,   65,    97,    129,
                                       193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
__constant__ uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
// RFC 1951 3.2.7: order of the code length code lengths.
__constant__ uint8_t kClOrder[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

// ---------------------------------------------------------------- CRC32 arithmetic
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

__constant__ CrcConst kCrc = make_crc_const();

// ---------------------------------------------------------------- shared memory

struct WarpSmem {
    uint32_t lit[1 << LB];
    uint32_t dist[1 << DB];      // also the code-length table while a dynamic header is read
    uint32_t scratch[48];        // table build: running index, first code, first index per length
    uint16_t lsorted[288];
    uint16_t dsorted[32];
    uint16_t lcount[16];
    uint16_t dcount[16];
    uint8_t lens[352];           // 19 code length code lengths, then up to 286 + 30 code lengths at +32
    alignas(16) uint8_t ring[RING];
};

struct CtaSmem {
    uint32_t crc8[8][256];       // slice-by-8 tables
    uint32_t mulk[4][256];       // multiplication by x^(8*992), one table per byte of the operand
    WarpSmem w[WARPS];
};

// ---------------------------------------------------------------- bit reader

struct Reader {
    const uint32_t* wbase;  // 4-byte aligned start at or before the payload
    uint32_t nvalid;        // words fully inside payload + trailer
    uint32_t g;             // current group of 32 words
    uint32_t widx;          // next word of the group
    uint32_t gw, gn;        // this lane's word of the current / next group
    uint64_t bb;            // bit buffer (LSB first)
    int bc;                 // valid bits in bb
    uint32_t s0;            // bits of wbase before the payload
};

__device__ __forceinline__ uint32_t load_word(const Reader& r, uint32_t group, int lane) {
    uint32_t w = group * 32u + (uint32_t)lane;
    return w < r.nvalid ? __ldg(r.wbase + w) : 0u;
}

__device__ __forceinline__ void refill(Reader& r) {
    uint32_t w = __shfl_sync(FULL, r.gw, r.widx);
    r.bb |= (uint64_t)w << r.bc;
    r.bc += 32;
    if (++r.widx == 32) {
        r.gw = r.gn;
        r.g++;
        r.gn = load_word(r, r.g + 1, threadIdx.x & 31);
        r.widx = 0;
    }
}

__device__ __forceinline__ void consume(Reader& r, int n) {
    r.bb >>= n;
    r.bc -= n;
}

// Bits consumed since the start of the payload.
__device__ __forceinline__ long long consumed(const Reader& r) {
    return ((long long)r.g * 32 + r.widx) * 32 - r.bc - r.s0;
}

__device__ __forceinline__ void seek(Reader& r, long long bitpos) {
    long long abs = bitpos + r.s0;
    uint32_t word = (uint32_t)(abs >> 5);
    int lane = threadIdx.x & 31;
    r.g = word >> 5;
    r.widx = word & 31;
    r.gw = load_word(r, r.g, lane);
    r.gn = load_word(r, r.g + 1, lane);
    r.bb = 0;
    r.bc = 0;
    refill(r);
    consume(r, (int)(abs & 31));
}

// ---------------------------------------------------------------- table build (whole warp)

enum : int { T_CLEN = 0, T_LIT = 1, T_DIST = 2 };

__device__ __forceinline__ uint32_t sym_entry(int kind, uint32_t s, uint32_t L) {
    if (kind == T_CLEN) return entry(L, K_LIT, 0, s);
    if (kind == T_LIT) {
        if (s < 256) return entry(L, K_LIT, 0, s);
        if (s == 256) return entry(L, K_EOB, 0, 0);
        if (s < 286) return entry(L, K_LEN, kLenExtra[s - 257], kLenBase[s - 257]);
        return entry(L, K_BAD, 0, 0);
    }
    if (s < 30) return entry(L, K_LEN, kDistExtra[s], kDistBase[s]);
    return entry(L, K_BAD, 0, 0);
}

// Canonical Huffman table of lens[0:nsym): tab[2^lb] indexed by the next lb bits, count[16] and
// sorted[] for the slow path.  Returns false for an over-subscribed code, or an incomplete one
// except a single code of length 1 (literal/length and distance codes), as zlib's inflate accepts.
__device__ __noinline__ bool build_table(const uint8_t* lens, int nsym, int lb, int kind, uint32_t* tab, uint16_t* count,
                            uint16_t* sorted, uint32_t* scratch) {
    const int lane = threadIdx.x & 31;
    if (lane < 16) scratch[lane] = 0;
    __syncwarp();
    for (int s = lane; s < nsym; s += 32) {
        uint32_t L = lens[s];
        if (L) atomicAdd(&scratch[L], 1u);
    }
    __syncwarp();
    uint32_t cnt = (lane >= 1 && lane < 16) ? scratch[lane] : 0u;
    // Kraft sum and the canonical first codes / first indices, the same in every lane.
    int left = 1, maxlen = 0;
    uint32_t code = 0, index = 0, my_first = 0, my_index = 0;
    for (int L = 1; L < 16; L++) {
        uint32_t c = __shfl_sync(FULL, cnt, L);
        left = (left << 1) - (int)c;
        if (c) maxlen = L;
        if (lane == L) {
            my_first = code;
            my_index = index;
        }
        index += c;
        code = (code + c) << 1;
        if (left < 0) break;
    }
    __syncwarp();
    if (left < 0) return false;
    bool incomplete = left > 0;
    if (kind == T_CLEN && (incomplete || maxlen == 0)) return false;
    if (incomplete && maxlen > 1) return false;
    if (lane >= 1 && lane < 16) {
        scratch[lane] = my_index;       // running insertion index
        scratch[16 + lane] = my_first;  // first code of the length
        scratch[32 + lane] = my_index;  // first index of the length
    }
    if (lane < 16 && count) count[lane] = (uint16_t)cnt;
    if (incomplete || maxlen == 0) {
        const uint32_t bad = entry(1, K_BAD, 0, 0);
        for (int i = lane; i < (1 << lb); i += 32) tab[i] = bad;
    }
    __syncwarp();
    for (int base = 0; base < nsym; base += 32) {
        int s = base + lane;
        uint32_t L = s < nsym ? lens[s] : 0u;
        uint32_t peers = __match_any_sync(FULL, L);
        uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        uint32_t pos = L ? scratch[L] : 0u;
        __syncwarp();
        if (L && lane == __ffs(peers) - 1) scratch[L] = pos + __popc(peers);
        __syncwarp();
        if (L) {
            uint32_t idx = pos + rank;
            if (sorted) sorted[idx] = (uint16_t)s;
            uint32_t c = scratch[16 + L] + (idx - scratch[32 + L]);
            if ((int)L <= lb) {
                uint32_t e = sym_entry(kind, (uint32_t)s, L);
                uint32_t r = __brev(c) >> (32 - L);
                for (uint32_t x = r; x < (1u << lb); x += (1u << L)) tab[x] = e;
            } else {
                uint32_t r = __brev(c >> (L - lb)) >> (32 - lb);
                tab[r] = entry(lb, K_SLOW, 0, 0);
            }
        }
        __syncwarp();
    }
    return true;
}

// Canonical decode of a code longer than the root bits (the same in every lane).  Returns the
// table entry of the symbol, with its full code length.
__device__ __forceinline__ uint32_t slow_decode(uint64_t bb, const uint16_t* count, const uint16_t* sorted, int kind) {
    int code = 0, first = 0, index = 0;
    for (int L = 1; L < 16; L++) {
        code |= (int)((bb >> (L - 1)) & 1u);
        int c = count[L];
        if (code - c < first) return sym_entry(kind, sorted[index + (code - first)], (uint32_t)L);
        index += c;
        first += c;
        first <<= 1;
        code <<= 1;
    }
    return entry(1, K_BAD, 0, 0);
}

// ---------------------------------------------------------------- output window

struct Out {
    uint8_t* out;          // member output in HBM
    uint32_t a;            // out & 15: ring slot of output byte p is (p + a) & RMASK
    uint32_t isize;
    uint32_t pad;          // (-isize) mod WIN: windows are aligned to the end of the member
    uint32_t p;            // bytes written
    uint32_t ws, we;       // current window [ws, we)
    uint32_t kwin;         // current window index
    uint32_t col;          // this lane's CRC column (raw, zero initial value)
};

__device__ __forceinline__ uint32_t mulk(const CtaSmem& S, uint32_t x) {
    return S.mulk[0][x & 255] ^ S.mulk[1][(x >> 8) & 255] ^ S.mulk[2][(x >> 16) & 255] ^ S.mulk[3][x >> 24];
}

// Store the window [ws, we) of the member's output to HBM and fold it into this lane's CRC column
// (returned).  Called once per 1 KB of output, out of line to keep the decode loop's registers free.
__device__ __noinline__ uint32_t flush_window(uint8_t* out, uint32_t a, uint32_t ws, uint32_t we, uint32_t kwin,
                                              uint32_t pad, uint32_t col, const uint8_t* ring, const CtaSmem& S,
                                              bool crc) {
    const int lane = threadIdx.x & 31;
    uintptr_t o16 = (uintptr_t)out & ~(uintptr_t)15;
    uintptr_t lo = (uintptr_t)out + ws, hi = (uintptr_t)out + we;
    uintptr_t A0 = lo & ~(uintptr_t)15;
    uint32_t nunits = (uint32_t)(((hi + 15) & ~(uintptr_t)15) - A0) >> 4;
    for (uint32_t u = lane; u < nunits; u += 32) {
        uintptr_t ga = A0 + 16 * (uintptr_t)u;
        uint32_t slot = (uint32_t)(ga - o16) & RMASK;
        if (ga >= lo && ga + 16 <= hi) {
            *reinterpret_cast<uint4*>(ga) = *reinterpret_cast<const uint4*>(ring + slot);
        } else {
            for (uint32_t k = 0; k < 16; k++)
                if (ga + k >= lo && ga + k < hi) *reinterpret_cast<uint8_t*>(ga + k) = ring[(slot + k) & RMASK];
        }
    }
    if (crc) {
        uint32_t c = mulk(S, col);
        long long v0 = (long long)kwin * WIN + 32 * lane - (long long)pad;  // real position of the column
#pragma unroll
        for (int q = 0; q < 32; q += 8) {
            uint32_t w0 = 0, w1 = 0;
#pragma unroll
            for (int t = 0; t < 4; t++) {
                long long r0 = v0 + q + t, r1 = v0 + q + 4 + t;
                uint32_t b0 = r0 >= 0 ? ring[(uint32_t)(r0 + a) & RMASK] : 0u;
                uint32_t b1 = r1 >= 0 ? ring[(uint32_t)(r1 + a) & RMASK] : 0u;
                w0 |= b0 << (8 * t);
                w1 |= b1 << (8 * t);
            }
            c ^= w0;
            c = S.crc8[7][c & 255] ^ S.crc8[6][(c >> 8) & 255] ^ S.crc8[5][(c >> 16) & 255] ^ S.crc8[4][c >> 24] ^
                S.crc8[3][w1 & 255] ^ S.crc8[2][(w1 >> 8) & 255] ^ S.crc8[1][(w1 >> 16) & 255] ^ S.crc8[0][w1 >> 24];
        }
        col = c;
    }
    __syncwarp();
    return col;
}

__device__ __forceinline__ void next_window(Out& o, const WarpSmem& W, const CtaSmem& S, bool crc) {
    o.col = flush_window(o.out, o.a, o.ws, o.we, o.kwin, o.pad, o.col, W.ring, S, crc);
    o.ws = o.we;
    o.we = min(o.we + WIN, o.isize);
    o.kwin++;
}

__device__ __forceinline__ void put_literal(Out& o, WarpSmem& W, const CtaSmem& S, uint32_t byte, bool crc) {
    if ((threadIdx.x & 31) == 0) W.ring[(o.p + o.a) & RMASK] = (uint8_t)byte;
    o.p++;
    if (o.p >= o.we) {
        __syncwarp();
        next_window(o, W, S, crc);
    }
}

// The zlib CRC32 of the member from the lane columns.
__device__ __noinline__ uint32_t finish_crc(uint32_t col, uint32_t isize) {
    const int lane = threadIdx.x & 31;
    uint32_t v = col;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        int d = 1 << k;
        uint32_t other = __shfl_down_sync(FULL, v, d);
        if ((lane & (2 * d - 1)) == 0) v = gf_mul(v, kCrc.seg[k]) ^ other;
    }
    v = __shfl_sync(FULL, v, 0);
    uint32_t cond = gf_mul(0xFFFFFFFFu, xpow_from(kCrc.x2n, 8ull * isize));
    return v ^ cond ^ 0xFFFFFFFFu;
}

// ---------------------------------------------------------------- one member

__device__ uint32_t inflate_member(const cb_member_job& job, uint8_t* out_base, bool crc, WarpSmem& W,
                                   const CtaSmem& S) {
    const int lane = threadIdx.x & 31;
    Reader r;
    uintptr_t in = (uintptr_t)job.in;
    r.wbase = reinterpret_cast<const uint32_t*>(in & ~(uintptr_t)3);
    r.s0 = (uint32_t)(in & 3) * 8;
    r.nvalid = (uint32_t)((in + job.in_len + 8 - (uintptr_t)r.wbase) >> 2);
    r.g = 0;
    r.widx = 0;
    r.gw = load_word(r, 0, lane);
    r.gn = load_word(r, 1, lane);
    r.bb = 0;
    r.bc = 0;
    refill(r);
    consume(r, (int)r.s0);

    Out o;
    o.out = out_base + job.out_off;
    o.a = (uint32_t)((uintptr_t)o.out & 15);
    o.isize = job.isize;
    o.pad = (uint32_t)(-(int32_t)job.isize) & (WIN - 1);
    o.p = 0;
    o.ws = 0;
    o.we = min((uint32_t)WIN - o.pad, o.isize);
    o.kwin = 0;
    o.col = 0;
    const long long in_bits = (long long)job.in_len * 8;
    const uint32_t isize = job.isize;

    bool final_block = false;
    while (!final_block) {
        if (consumed(r) > in_bits) return CB_ERR_INFLATE;
        if (r.bc < 32) refill(r);
        uint32_t hdr = (uint32_t)r.bb & 7u;
        consume(r, 3);
        final_block = hdr & 1u;
        uint32_t btype = hdr >> 1;
        if (btype == 0) {
            // stored block: byte aligned LEN, NLEN, then LEN bytes
            long long pos = consumed(r);
            pos = (pos + 7) & ~7ll;
            seek(r, pos);
            if (r.bc < 32) refill(r);
            uint32_t len = (uint32_t)r.bb & 0xFFFFu, nlen = ((uint32_t)r.bb >> 16) & 0xFFFFu;
            if (len != (~nlen & 0xFFFFu)) return CB_ERR_INFLATE;
            long long byte = pos / 8 + 4;
            if (byte + len > (long long)job.in_len || o.p + len > isize) return CB_ERR_INFLATE;
            const uint8_t* src = job.in + byte;
            for (uint32_t k = 0; k < len; k += 32) {
                uint32_t n = min(32u, len - k);
                __syncwarp();
                if ((uint32_t)lane < n) W.ring[(o.p + lane + o.a) & RMASK] = src[k + lane];
                o.p += n;
                __syncwarp();
                if (o.p >= o.we) next_window(o, W, S, crc);
            }
            seek(r, (byte + len) * 8);
            continue;
        }
        if (btype == 3) return CB_ERR_INFLATE;
        if (btype == 1) {
            for (int s = lane; s < 288; s += 32) W.lens[s] = s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : 8;
            for (int s = lane; s < 32; s += 32) W.lens[288 + s] = 5;
            __syncwarp();
            if (!build_table(W.lens, 288, LB, T_LIT, W.lit, W.lcount, W.lsorted, W.scratch)) return CB_ERR_INFLATE;
            if (!build_table(W.lens + 288, 32, DB, T_DIST, W.dist, W.dcount, W.dsorted, W.scratch))
                return CB_ERR_INFLATE;
        } else {
            // dynamic block header
            if (r.bc < 32) refill(r);
            uint32_t hlit = ((uint32_t)r.bb & 31u) + 257, hdist = (((uint32_t)r.bb >> 5) & 31u) + 1;
            uint32_t hclen = (((uint32_t)r.bb >> 10) & 15u) + 4;
            consume(r, 14);
            if (hlit > 286 || hdist > 30) return CB_ERR_INFLATE;
            if (lane < 19) W.lens[lane] = 0;
            __syncwarp();
            // code length code lengths: 3 bits each, the first 10 then the rest
            for (uint32_t base = 0; base < hclen; base += 10) {
                if (r.bc < 32) refill(r);
                uint32_t cnt = min(10u, hclen - base);
                if ((uint32_t)lane < cnt) W.lens[kClOrder[base + lane]] = (uint8_t)((r.bb >> (3 * lane)) & 7u);
                consume(r, 3 * cnt);
            }
            __syncwarp();
            uint32_t* cltab = W.dist;  // 128 entries, reused before the distance table is built
            if (!build_table(W.lens, 19, CLB, T_CLEN, cltab, nullptr, nullptr, W.scratch)) return CB_ERR_INFLATE;
            const uint32_t total = hlit + hdist;
            uint32_t i = 0;
            uint8_t* L = W.lens + 32;  // lengths go after the 19 code length code lengths
            while (i < total) {
                if (r.bc < 32) refill(r);
                uint32_t e = cltab[(uint32_t)r.bb & ((1u << CLB) - 1)];
                if (e_kind(e) != K_LIT) return CB_ERR_INFLATE;
                consume(r, (int)e_bits(e));
                uint32_t sym = e_value(e);
                if (sym < 16) {
                    if (lane == 0) L[i] = (uint8_t)sym;
                    i++;
                    continue;
                }
                uint32_t rep, val = 0;
                if (sym == 16) {
                    if (i == 0) return CB_ERR_INFLATE;
                    __syncwarp();
                    val = L[i - 1];
                    rep = 3 + ((uint32_t)r.bb & 3u);
                    consume(r, 2);
                } else if (sym == 17) {
                    rep = 3 + ((uint32_t)r.bb & 7u);
                    consume(r, 3);
                } else {
                    rep = 11 + ((uint32_t)r.bb & 127u);
                    consume(r, 7);
                }
                if (i + rep > total) return CB_ERR_INFLATE;
                for (uint32_t j = lane; j < rep; j += 32) L[i + j] = (uint8_t)val;
                i += rep;
            }
            __syncwarp();
            if (L[256] == 0) return CB_ERR_INFLATE;  // no end-of-block code
            if (!build_table(L, (int)hlit, LB, T_LIT, W.lit, W.lcount, W.lsorted, W.scratch)) return CB_ERR_INFLATE;
            if (!build_table(L + hlit, (int)hdist, DB, T_DIST, W.dist, W.dcount, W.dsorted, W.scratch))
                return CB_ERR_INFLATE;
        }
        // ------------------------------------------------ Huffman-coded data
        for (;;) {
            if (r.bc < 32) refill(r);
            uint32_t e = W.lit[(uint32_t)r.bb & ((1u << LB) - 1)];
            uint32_t kind = e_kind(e);
            if (kind == K_LIT) {
                consume(r, (int)e_bits(e));
                if (o.p >= isize) return CB_ERR_INFLATE;
                put_literal(o, W, S, e_value(e), crc);
                continue;
            }
            if (kind == K_SLOW) {
                e = slow_decode(r.bb, W.lcount, W.lsorted, T_LIT);
                kind = e_kind(e);
                if (kind == K_LIT) {
                    consume(r, (int)e_bits(e));
                    if (o.p >= isize) return CB_ERR_INFLATE;
                    put_literal(o, W, S, e_value(e), crc);
                    continue;
                }
            }
            if (kind == K_EOB) {
                consume(r, (int)e_bits(e));
                break;
            }
            if (kind != K_LEN) return CB_ERR_INFLATE;
            consume(r, (int)e_bits(e));
            uint32_t ext = e_extra(e);
            uint32_t len = e_value(e) + ((uint32_t)r.bb & ((1u << ext) - 1u));
            consume(r, (int)ext);
            if (r.bc < 32) refill(r);
            uint32_t d = W.dist[(uint32_t)r.bb & ((1u << DB) - 1)];
            if (e_kind(d) == K_SLOW) d = slow_decode(r.bb, W.dcount, W.dsorted, T_DIST);
            if (e_kind(d) != K_LEN) return CB_ERR_INFLATE;
            consume(r, (int)e_bits(d));
            uint32_t dext = e_extra(d);
            uint32_t dist = e_value(d) + ((uint32_t)r.bb & ((1u << dext) - 1u));
            consume(r, (int)dext);
            if (dist > o.p || o.p + len > isize) return CB_ERR_INFLATE;
            __syncwarp();
            const uint32_t src = o.p - dist;
            if (dist <= (uint32_t)DMAX_RING) {
                if (dist >= len) {
                    for (uint32_t j = lane; j < len; j += 32)
                        W.ring[(o.p + j + o.a) & RMASK] = W.ring[(src + j + o.a) & RMASK];
                } else {
                    for (uint32_t j = lane; j < len; j += 32)
                        W.ring[(o.p + j + o.a) & RMASK] = W.ring[(src + j % dist + o.a) & RMASK];
                }
            } else {
                for (uint32_t j = lane; j < len; j += 32) W.ring[(o.p + j + o.a) & RMASK] = o.out[src + j];
            }
            o.p += len;
            __syncwarp();
            if (o.p >= o.we) next_window(o, W, S, crc);
        }
    }
    if (consumed(r) > in_bits || o.p != isize) return CB_ERR_INFLATE;
    if (crc && finish_crc(o.col, isize) != job.crc) return CB_ERR_CRC;
    return CB_OK;
}

// ---------------------------------------------------------------- kernels

__global__ void k_inflate_init(cb_inflate_summary* summary, unsigned long long* queue) {
    summary->status = CB_OK;
    summary->reserved = 0;
    summary->n_bad = 0;
    summary->first_bad = INT64_MAX;
    *queue = 0;
}

__global__ void k_inflate_finish(cb_inflate_summary* summary) {
    if (summary->first_bad == INT64_MAX) summary->first_bad = -1;
}

__global__ void __launch_bounds__(WARPS * 32, 4) k_inflate(const cb_member_job* __restrict__ jobs, int64_t n_jobs,
                                                        const int64_t* __restrict__ d_n_jobs, uint8_t* out_base,
                                                        int check_crc, uint32_t* job_status,
                                                        cb_inflate_summary* summary, unsigned long long* queue) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    CtaSmem& S = *reinterpret_cast<CtaSmem*>(smem_raw);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        uint32_t c = (uint32_t)i;
        for (int k = 0; k < 8; k++) c = (c & 1u) ? (c >> 1) ^ POLY : c >> 1;
        S.crc8[0][i] = c;
#pragma unroll
        for (int b = 0; b < 4; b++) S.mulk[b][i] = gf_mul((uint32_t)i << (8 * b), kCrc.k992);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        uint32_t c = S.crc8[0][i];
        for (int t = 1; t < 8; t++) {
            c = (c >> 8) ^ S.crc8[0][c & 255];
            S.crc8[t][i] = c;
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpSmem& W = S.w[warp];
    int64_t n = n_jobs;
    if (d_n_jobs) n = min(n, *d_n_jobs);
    const bool crc = check_crc != 0;
    for (;;) {
        unsigned long long j = 0;
        if (lane == 0) j = atomicAdd(queue, 1ull);
        j = __shfl_sync(FULL, j, 0);
        if ((int64_t)j >= n) break;
        cb_member_job job = jobs[j];
        uint32_t st = inflate_member(job, out_base, crc, W, S);
        __syncwarp();
        if (lane == 0) {
            if (job_status) job_status[j] = st;
            if (st != CB_OK) {
                atomicAdd(reinterpret_cast<unsigned long long*>(&summary->n_bad), 1ull);
                atomicMin(reinterpret_cast<long long*>(&summary->first_bad), (long long)j);
                atomicMax(&summary->status, (int)st);
            }
        }
    }
}

}  // namespace infl
}  // namespace cb

using namespace cb;

static int g_inflate_blocks_per_sm = -1;

extern "C" size_t cb_inflate_workspace_bytes(void) { return 256; }

int cb_set_error(cudaError_t e);  // abi.cu

extern "C" int cb_inflate(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint8_t* out_base,
                          int check_crc, uint32_t* job_status, cb_inflate_summary* summary, void* workspace,
                          size_t workspace_bytes, void* stream) {
    if (!summary || !workspace || workspace_bytes < cb_inflate_workspace_bytes() || n_jobs < 0) return CB_ERR_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    auto* queue = reinterpret_cast<unsigned long long*>(workspace);
    const size_t smem = sizeof(infl::CtaSmem);
    if (g_inflate_blocks_per_sm < 0) {
        cudaError_t e = cudaFuncSetAttribute(infl::k_inflate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cb_set_error(e);
        int b = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, infl::k_inflate, infl::WARPS * 32, smem);
        if (e != cudaSuccess) return cb_set_error(e);
        g_inflate_blocks_per_sm = b > 0 ? b : 1;
    }
    infl::k_inflate_init<<<1, 1, 0, s>>>(summary, queue);
    if (n_jobs > 0) {
        long long warps_needed = n_jobs;
        long long grid = (long long)cb_device_sm_count() * g_inflate_blocks_per_sm;
        long long by_work = (warps_needed + infl::WARPS - 1) / infl::WARPS;
        if (!d_n_jobs && by_work < grid) grid = by_work;
        if (grid < 1) grid = 1;
        infl::k_inflate<<<(unsigned)grid, infl::WARPS * 32, smem, s>>>(jobs, n_jobs, d_n_jobs, out_base, check_crc,
                                                                        job_status, summary, queue);
    }
    infl::k_inflate_finish<<<1, 1, 0, s>>>(summary);
    return cb_set_error(cudaGetLastError());
}
