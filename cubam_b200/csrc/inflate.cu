// Raw-DEFLATE inflater for BGZF members on B200 (sm_100a), with the CRC32 and ISIZE checks.
//
// Replaces cubam's call of nvcompBatchedDeflateDecompressAsync and its status/size check
// (src/cubam/bgzf.py:587-611); the CRC32 check is new (cubam's reader does not check it,
// docs/reading.md:48-51).  DEFLATE itself is RFC 1951.
//
// One warp per member, persistent grid, members taken from a work queue.  Huffman decoding is
// serial in principle; the 32 lanes of the warp decode one block in parallel by speculation, as
// Huffman codes resynchronise after a few symbols when decoding starts at a wrong bit:
//
//  D  lane i decodes the block from bit S + 768 i to S + 768 (i + 1) (S: a known symbol start),
//     writing tokens (literal, or length/distance) to its row of shared memory and marking the bit
//     where each symbol starts in its own bitmap.  Lane 0 starts at a true symbol start.
//  S  lane i re-decodes from the end of lane i-1 (the true start of its stream, once lane i-1 is
//     right) until it reaches a bit its own speculative pass marked: from there on its tokens are
//     right.  The few symbols before ("fixups") are re-decoded again in pass W and written in front
//     of the kept tokens.  Passes repeat while a lane's start changes (rarely more than one).
//     A lane that does not resynchronise within a bound ends the round; the next round starts
//     where the last good lane ended.  The first lane whose true stream has the end-of-block code
//     ends the block.
//  M  tokens are written in stream order, 32 at a time (one per lane): literals at once, then the
//     matches in waves -- a match is ready when its source lies before the first unfinished one.
//
// Output goes to a 36 KB ring per warp in shared memory (the whole 32 KB DEFLATE window plus a
// group), flushed to HBM in 1 KB windows aligned to the END of the member with 16-byte stores.
// Each flushed window is folded into the CRC32: slice-by-8 tables in shared memory, lane l keeps a
// column of bytes [32l, 32l+32) of every window, combined once per member by GF(2) arithmetic
// modulo the CRC polynomial (constants computed at compile time).  Stored blocks are copied by the
// whole warp; block headers and code-length tables are read by the warp in lock step, with the
// 32 lanes building the lookup tables together (__match_any_sync ranks).
//
// Every loop is bounded by the member's sizes or a fixed count: output beyond ISIZE, a distance
// before the member's start, bits read beyond the payload, bad code lengths, invalid symbols in the
// true stream are per-member errors.

#include <cstdlib>

#include "common.cuh"

namespace cb {
namespace infl {

constexpr int LB = 10;                    // literal/length root bits
constexpr int DB = 8;                     // distance root bits
constexpr int CLB = 7;                    // code-length code bits
constexpr int WARPS = 3;                  // warps per CTA (one CTA per SM: shared memory)
constexpr int SEG = 768;                  // input bits per lane per round
constexpr int BMPW = SEG / 32;            // bitmap words per lane
constexpr int BSTRIDE = BMPW + 1;         // odd row strides: conflict-free shared memory rows
constexpr int RESERVE = 12;               // token slots in front of a lane's speculative tokens (fixups)
constexpr int CAP = 120;                  // speculative tokens per lane per round
constexpr int TSTRIDE = RESERVE + CAP + 1;
constexpr int MAXFIX = 24;                // symbols a lane may re-decode looking for its resync point
constexpr int GROUP_BYTES = 1024;         // a group of tokens starts within this many output bytes
constexpr int WIN = 1024;                 // flush / CRC window
constexpr int RING = 36864;               // 32 KB window + room for one group; multiple of 16 and WIN
constexpr uint32_t LMASK = (1u << LB) - 1, DMASK = (1u << DB) - 1;

static_assert(RING >= 32768 + GROUP_BYTES + 258 + WIN, "ring must hold the window, a group and a flush window");
static_assert(RING % WIN == 0 && RING % 16 == 0, "ring of whole windows");
static_assert(WIN == 32 * 32, "one 32-byte CRC column per lane");
static_assert(TSTRIDE % 2 == 1 && BSTRIDE % 2 == 1, "odd strides");

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
    uint32_t tok[32 * TSTRIDE];  // lane rows of tokens: RESERVE fixup slots, then speculative tokens
    uint32_t bmp[32 * BSTRIDE];  // lane rows: bit r set when a speculative symbol starts at bit S_lane + r
    alignas(16) uint8_t ring[RING];
};

struct CtaSmem {
    uint32_t crc8[8][256];       // slice-by-8 tables
    uint32_t mulk[4][256];       // multiplication by x^(8*992), one table per byte of the operand
    WarpSmem w[WARPS];
};

__device__ __forceinline__ uint32_t slot(uint32_t x) { return x < (uint32_t)RING ? x : x - (uint32_t)RING; }

// Slot of x in a ring of RN bytes (x below 2 RN when RN is not a power of two).
template <uint32_t RN> __device__ __forceinline__ uint32_t slot_of(uint32_t x) {
    if constexpr ((RN & (RN - 1)) == 0) return x & (RN - 1);
    else return x < RN ? x : x - RN;
}

// ---------------------------------------------------------------- lock-step reader (whole warp)
// Every lane holds the same bit buffer.  Lane l keeps word l of the current 128-byte group of input;
// refills take the next word with __shfl_sync and the next group is prefetched a group ahead.

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

__device__ __forceinline__ uint32_t load_word(const uint32_t* wbase, uint32_t nvalid, uint32_t w) {
    return w < nvalid ? __ldg(wbase + w) : 0u;
}

__device__ __forceinline__ void refill(Reader& r) {
    uint32_t w = __shfl_sync(FULL, r.gw, r.widx);
    r.bb |= (uint64_t)w << r.bc;
    r.bc += 32;
    if (++r.widx == 32) {
        r.gw = r.gn;
        r.g++;
        r.gn = load_word(r.wbase, r.nvalid, (r.g + 1) * 32u + (threadIdx.x & 31));
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
    r.gw = load_word(r.wbase, r.nvalid, r.g * 32u + lane);
    r.gn = load_word(r.wbase, r.nvalid, (r.g + 1) * 32u + lane);
    r.bb = 0;
    r.bc = 0;
    refill(r);
    consume(r, (int)(abs & 31));
}

// ---------------------------------------------------------------- per-lane reader (speculative)

struct LaneReader {
    uint64_t bb;
    int bc;
    uint32_t nextw;
    long long pos;  // bit of the payload the next unconsumed bit is
};

__device__ __forceinline__ void lr_init(LaneReader& r, const uint32_t* wbase, uint32_t nvalid, uint32_t s0,
                                        long long pos) {
    long long a = pos + s0;
    uint32_t w = (uint32_t)(a >> 5);
    int sh = (int)(a & 31);
    uint64_t x = (uint64_t)load_word(wbase, nvalid, w) | ((uint64_t)load_word(wbase, nvalid, w + 1) << 32);
    r.bb = x >> sh;
    r.bc = 64 - sh;
    r.nextw = w + 2;
    r.pos = pos;
}

__device__ __forceinline__ void lr_refill(LaneReader& r, const uint32_t* wbase, uint32_t nvalid) {
    if (r.bc <= 32) {
        r.bb |= (uint64_t)load_word(wbase, nvalid, r.nextw++) << r.bc;
        r.bc += 32;
    }
}

__device__ __forceinline__ void lr_consume(LaneReader& r, int n) {
    r.bb >>= n;
    r.bc -= n;
    r.pos += n;
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

// ---------------------------------------------------------------- symbols

enum : int { S_LIT = 0, S_MATCH = 1, S_EOB = 2, S_BAD = 3 };

// One symbol (a literal, a length/distance pair or the end-of-block code) at the lane's position.
// Tokens: literal = the byte; match = 0x80000000 | length << 16 | (distance - 1).
__device__ __forceinline__ int lane_symbol(LaneReader& r, const WarpSmem& W, const uint32_t* wbase, uint32_t nvalid,
                                           uint32_t& tok) {
    lr_refill(r, wbase, nvalid);
    uint32_t e = W.lit[(uint32_t)r.bb & LMASK];
    if (e_kind(e) == K_SLOW) e = slow_decode(r.bb, W.lcount, W.lsorted, T_LIT);
    const uint32_t k = e_kind(e);
    if (k == K_LIT) {
        lr_consume(r, (int)e_bits(e));
        tok = e_value(e);
        return S_LIT;
    }
    if (k == K_EOB) {
        lr_consume(r, (int)e_bits(e));
        return S_EOB;
    }
    if (k != K_LEN) return S_BAD;
    lr_consume(r, (int)e_bits(e));
    const uint32_t ext = e_extra(e);
    const uint32_t len = e_value(e) + ((uint32_t)r.bb & ((1u << ext) - 1u));
    lr_consume(r, (int)ext);
    lr_refill(r, wbase, nvalid);
    uint32_t d = W.dist[(uint32_t)r.bb & DMASK];
    if (e_kind(d) == K_SLOW) d = slow_decode(r.bb, W.dcount, W.dsorted, T_DIST);
    if (e_kind(d) != K_LEN) return S_BAD;
    lr_consume(r, (int)e_bits(d));
    const uint32_t dext = e_extra(d);
    const uint32_t dist = e_value(d) + ((uint32_t)r.bb & ((1u << dext) - 1u));
    lr_consume(r, (int)dext);
    tok = 0x80000000u | (len << 16) | (dist - 1);
    return S_MATCH;
}

__device__ __forceinline__ bool tok_match(uint32_t t) { return (t & 0x80000000u) != 0; }
__device__ __forceinline__ uint32_t tok_len(uint32_t t) { return tok_match(t) ? (t >> 16) & 0x1FFu : 1u; }
__device__ __forceinline__ uint32_t tok_dist(uint32_t t) { return (t & 0xFFFFu) + 1u; }

// ---------------------------------------------------------------- output window

struct Out {
    uint8_t* out;          // member output in HBM
    uint32_t a;            // out & 15: ring slot of output byte p is slot(p + a)
    uint32_t isize;
    uint32_t pad;          // (-isize) mod WIN: windows are aligned to the end of the member
    uint32_t p;            // bytes written
    uint32_t ws, we;       // current window [ws, we)
    uint32_t kwin;         // current window index
    uint32_t col;          // this lane's CRC column (raw, zero initial value)
};

template <class CS> __device__ __forceinline__ uint32_t mulk(const CS& S, uint32_t x) {
    return S.mulk[0][x & 255] ^ S.mulk[1][(x >> 8) & 255] ^ S.mulk[2][(x >> 16) & 255] ^ S.mulk[3][x >> 24];
}

// Store the window [ws, we) of the member's output to HBM and fold it into this lane's CRC column
// (returned).  Called once per 1 KB of output, out of line.  The window's bytes are in `ring` (RN bytes,
// output byte p at slot p + a).
template <uint32_t RN, class CS>
__device__ __noinline__ uint32_t flush_window_t(uint8_t* out, uint32_t a, uint32_t ws, uint32_t we, uint32_t kwin,
                                                uint32_t pad, uint32_t col, const uint8_t* ring, const CS& S,
                                                bool crc) {
    const int lane = threadIdx.x & 31;
    uintptr_t o16 = (uintptr_t)out & ~(uintptr_t)15;
    uintptr_t lo = (uintptr_t)out + ws, hi = (uintptr_t)out + we;
    uintptr_t A0 = lo & ~(uintptr_t)15;
    uint32_t nunits = (uint32_t)(((hi + 15) & ~(uintptr_t)15) - A0) >> 4;
    for (uint32_t u = lane; u < nunits; u += 32) {
        uintptr_t ga = A0 + 16 * (uintptr_t)u;
        uint32_t s = slot_of<RN>((uint32_t)(ga - o16));
        if (ga >= lo && ga + 16 <= hi) {
            *reinterpret_cast<uint4*>(ga) = *reinterpret_cast<const uint4*>(ring + s);
        } else {
            for (uint32_t k = 0; k < 16; k++)
                if (ga + k >= lo && ga + k < hi) *reinterpret_cast<uint8_t*>(ga + k) = ring[s + k];
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
                uint32_t b0 = r0 >= 0 ? ring[slot_of<RN>((uint32_t)(r0 + a))] : 0u;
                uint32_t b1 = r1 >= 0 ? ring[slot_of<RN>((uint32_t)(r1 + a))] : 0u;
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

// Flush every complete window (all lanes).
template <uint32_t RN, class WS, class CS>
__device__ __forceinline__ void flush_ready(Out& o, const WS& W, const CS& S, bool crc) {
    while (o.we > o.ws && o.p >= o.we) {
        o.col = flush_window_t<RN>(o.out, o.a, o.ws, o.we, o.kwin, o.pad, o.col, W.ring, S, crc);
        o.ws = o.we;
        o.we = min(o.we + WIN, o.isize);
        o.kwin++;
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

__device__ __forceinline__ long long shfl_up_ll(long long v, int d) {
    int lo = __shfl_up_sync(FULL, (int)(v & 0xffffffff), d), hi = __shfl_up_sync(FULL, (int)(v >> 32), d);
    return ((long long)hi << 32) | (unsigned)lo;
}
__device__ __forceinline__ long long shfl_ll(long long v, int src) {
    int lo = __shfl_sync(FULL, (int)(v & 0xffffffff), src), hi = __shfl_sync(FULL, (int)(v >> 32), src);
    return ((long long)hi << 32) | (unsigned)lo;
}

// ---------------------------------------------------------------- one Huffman block, speculatively

enum : int { L_SYNC = 0, L_AUTH = 1, L_FAIL = 2, L_BAD = 3, L_EOBFIX = 4 };

// Decode the Huffman-coded data of one block from bit `pos` (a symbol start) to its end-of-block
// code.  Returns CB_OK with *pos after the end-of-block code, or CB_ERR_INFLATE.
__device__ uint32_t spec_block(long long& pos, const uint32_t* wbase, uint32_t nvalid, uint32_t s0, long long in_bits,
                               Out& o, WarpSmem& W, const CtaSmem& S, bool crc) {
    const int lane = threadIdx.x & 31;
    uint32_t* T = W.tok + lane * TSTRIDE;
    uint32_t* B = W.bmp + lane * BSTRIDE;
    for (int round = 0;; round++) {
        if (pos > in_bits) return CB_ERR_INFLATE;  // the block runs past the payload
        // ---------------- D: speculative decode of this lane's segment
        const long long seg0 = pos + (long long)lane * SEG, seg1 = seg0 + SEG;
        for (int i = 0; i < BMPW; i++) B[i] = 0;
        LaneReader r;
        lr_init(r, wbase, nvalid, s0, seg0);
        int n = 0, flag = S_LIT;
        uint32_t curw = 0;
        int curwi = 0;
        long long spec_end = seg0, eob_end = -1;
        // one symbol per lane per iteration; the vote keeps the lanes converged (independent thread
        // scheduling would otherwise run the lanes' loops one after another)
        bool act = true;
        for (int it = 0; it < CAP; it++) {
            act = act && r.pos < seg1;
            if (!__any_sync(FULL, act)) break;
            if (act) {
                const int rel = (int)(r.pos - seg0);
                if ((rel >> 5) != curwi) {
                    B[curwi] = curw;
                    curwi = rel >> 5;
                    curw = 0;
                }
                curw |= 1u << (rel & 31);
                const long long at = r.pos;
                uint32_t t = 0;
                const int k = lane_symbol(r, W, wbase, nvalid, t);
                if (k == S_BAD) {
                    flag = S_BAD;
                    r.pos = at;
                    act = false;
                } else if (k == S_EOB) {
                    flag = S_EOB;
                    eob_end = r.pos;
                    act = false;
                } else {
                    T[RESERVE + n++] = t;
                }
            }
        }
        B[curwi] = curw;
        spec_end = r.pos;
        __syncwarp();
        // ---------------- S: find where each lane's true stream joins its speculative one
        long long t_start = lane == 0 ? pos : -1;   // true start of this lane's stream
        long long true_end = flag == S_EOB ? eob_end : spec_end;
        int st = L_SYNC, k_sync = 0, nf = 0;
        long long fix_eob_end = -1;
        for (int pass = 0; pass < 32; pass++) {
            const long long prev_end = shfl_up_ll(true_end, 1);
            // lanes after a failure or after the end of the block are not needed
            const unsigned stop = __ballot_sync(FULL, st == L_FAIL || st == L_BAD || st == L_EOBFIX ||
                                                          (st == L_SYNC && flag == S_EOB));
            const int first_stop = stop ? __ffs(stop) - 1 : 32;
            const bool need = lane > 0 && lane <= first_stop && prev_end != t_start;
            if (!__any_sync(FULL, need)) break;
            LaneReader rr;
            bool go = need;
            if (need) {
                t_start = prev_end;
                lr_init(rr, wbase, nvalid, s0, t_start);
                nf = 0;
                st = L_FAIL;
            }
            for (int it = 0; it <= MAXFIX; it++) {
                if (!__any_sync(FULL, go)) break;
                if (go) {
                    const long long p = rr.pos;
                    const long long rel = p - seg0;
                    if (rel >= 0 && rel < SEG && p < spec_end + (flag == S_EOB ? 1 : 0) &&
                        ((B[rel >> 5] >> (rel & 31)) & 1u)) {
                        // resynchronised: count the speculative symbols before this bit
                        int kk = __popc(B[rel >> 5] & ((1u << (rel & 31)) - 1u));
                        for (int w = 0; w < BMPW; w++) kk += w < (int)(rel >> 5) ? __popc(B[w]) : 0;
                        k_sync = kk;
                        st = nf <= RESERVE + kk ? L_SYNC : L_FAIL;
                        true_end = flag == S_EOB ? eob_end : spec_end;
                        go = false;
                    } else if (p >= spec_end && flag != S_EOB) {
                        // the true stream covered this lane's segment without meeting it
                        k_sync = n;
                        st = nf <= RESERVE + n ? L_AUTH : L_FAIL;
                        true_end = p;
                        go = false;
                    } else if (nf >= MAXFIX) {
                        go = false;
                    } else {
                        uint32_t t = 0;
                        const int k = lane_symbol(rr, W, wbase, nvalid, t);
                        if (k == S_BAD) {
                            st = L_BAD;
                            go = false;
                        } else if (k == S_EOB) {
                            k_sync = n;
                            st = nf <= RESERVE + n ? L_EOBFIX : L_FAIL;
                            fix_eob_end = rr.pos;
                            true_end = rr.pos;
                            go = false;
                        } else {
                            nf++;
                        }
                    }
                }
            }
            if (need && (st == L_FAIL || st == L_BAD)) true_end = -2;
        }
        // ---------------- the lanes of this round: up to the first failure, or the end of the block
        const unsigned failm = __ballot_sync(FULL, st == L_FAIL || st == L_BAD);
        const unsigned eobm = __ballot_sync(FULL, st == L_EOBFIX || (st == L_SYNC && flag == S_EOB));
        const unsigned badm = __ballot_sync(FULL, st == L_SYNC && flag == S_BAD && spec_end < seg1);
        const int first_fail = failm ? __ffs(failm) - 1 : 32;
        const int first_eob = eobm ? __ffs(eobm) - 1 : 32;
        const int first_bad = badm ? __ffs(badm) - 1 : 32;
        // a bad symbol in the true stream (before any end-of-block): corrupt data
        if (first_bad < first_fail && first_bad <= first_eob) return CB_ERR_INFLATE;
        if (first_fail < first_eob && first_fail < 32 &&
            __shfl_sync(FULL, st, first_fail) == L_BAD)
            return CB_ERR_INFLATE;
        const int last = first_eob < first_fail ? first_eob : first_fail - 1;  // last lane whose tokens count
        const bool ends_block = first_eob < first_fail;
        // ---------------- W: write the fixups of the lanes that count
        {
            const int nw = (lane > 0 && lane <= last) ? nf : 0;
            LaneReader rr;
            if (nw) lr_init(rr, wbase, nvalid, s0, t_start);
            const int at = RESERVE + k_sync - nf;
            for (int j = 0; j < MAXFIX; j++) {
                if (!__any_sync(FULL, j < nw)) break;
                if (j < nw) {
                    uint32_t t = 0;
                    lane_symbol(rr, W, wbase, nvalid, t);
                    T[at + j] = t;
                }
            }
        }
        __syncwarp();
        // token range of this lane in its row
        int first = RESERVE + k_sync - nf, count = 0;
        if (lane <= last) {
            int end_idx = n;                            // after the last speculative token
            if (st == L_SYNC && flag == S_EOB) end_idx = n;  // the end-of-block code follows token n-1
            if (st == L_AUTH || st == L_EOBFIX) end_idx = k_sync;
            count = RESERVE + end_idx - first;
            if (lane == 0) {
                first = RESERVE;
                count = n;
            }
        }
        long long new_pos = shfl_ll(ends_block ? (st == L_EOBFIX ? fix_eob_end : eob_end) : true_end,
                                    last < 0 ? 0 : last);
        // ---------------- M: materialise the tokens in stream order, 32 at a time
        uint32_t total;
        const uint32_t base = warp_exclusive_scan((uint32_t)count, total);
        for (uint32_t g0 = 0; g0 < total;) {
            const uint32_t t = g0 + lane;
            const bool have = t < total;
            int own = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const int cand = own + step;
                const uint32_t b = __shfl_sync(FULL, base, cand & 31);
                if (cand < 32 && b <= t) own = cand;
            }
            const uint32_t ob = __shfl_sync(FULL, base, own);
            const int of = __shfl_sync(FULL, first, own);
            const uint32_t tk = have ? W.tok[own * TSTRIDE + of + (int)(t - ob)] : 0u;
            const uint32_t len = have ? tok_len(tk) : 0u;
            uint32_t gsum;
            const uint32_t ex = warp_exclusive_scan(len, gsum);
            const unsigned takem = __ballot_sync(FULL, have && ex < (uint32_t)GROUP_BYTES);
            const int gcount = __popc(takem);
            const bool valid = lane < gcount;
            const uint32_t glen = __shfl_sync(FULL, ex + len, gcount - 1);
            const uint32_t q = o.p + ex;
            const bool is_m = valid && tok_match(tk);
            const uint32_t dist = is_m ? tok_dist(tk) : 0u;
            if (__any_sync(FULL, valid && (q + len > o.isize || dist > q))) return CB_ERR_INFLATE;
            if (valid && !is_m) W.ring[slot(q + o.a)] = (uint8_t)tk;
            __syncwarp();
            bool pend = is_m;
            for (int it = 0; it < 33; it++) {
                if (!__any_sync(FULL, pend)) break;
                const uint32_t P = __reduce_min_sync(FULL, pend ? q : 0xFFFFFFFFu);
                const bool ready = pend && (q - dist + min(len, dist) <= P);
                {
                    const uint32_t cl = ready ? len : 0u;
                    uint32_t sd = slot(q + o.a), ss = slot(q - dist + o.a);
                    for (uint32_t j = 0; j < 258; j++) {
                        if (!__any_sync(FULL, j < cl)) break;
                        if (j < cl) {
                            W.ring[sd] = W.ring[ss];
                            sd = sd + 1 == (uint32_t)RING ? 0u : sd + 1;
                            ss = ss + 1 == (uint32_t)RING ? 0u : ss + 1;
                        }
                    }
                }
                __syncwarp();
                pend = pend && !ready;
            }
            o.p += glen;
            flush_ready<RING>(o, W, S, crc);
            g0 += (uint32_t)gcount;
        }
        pos = new_pos;
        if (ends_block) return CB_OK;
        (void)round;
    }
}

// The Huffman tables of a fixed (btype 1) or dynamic (btype 2) block, the dynamic header read by the
// whole warp in lock step.  CB_OK or CB_ERR_INFLATE.
template <class WS> __device__ uint32_t read_tables(Reader& r, WS& W, uint32_t btype) {
    const int lane = threadIdx.x & 31;
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
    return CB_OK;
}

// ================================================================ lock-step decode, batched writes
// The other form of the inflater: 8 warps per CTA, 2 CTAs per SM.  The warp decodes symbols in lock
// step into a token buffer only (no output writes, no copies in the serial loop), then writes the
// batch of tokens warp-parallel: 32 tokens per group, literals at once, matches in waves (ready when
// the source lies before the first unfinished match).  Back-references within the 4 KB ring read
// shared memory, older ones read the flushed output in HBM.

namespace lk {

constexpr int WARPS = 8;
constexpr int NTOK = 512;                 // tokens decoded before a batch is written
constexpr uint32_t RING = 4096;
constexpr uint32_t GROUP = 512;           // a group of tokens starts within this many output bytes
static_assert(RING >= GROUP + 258 + WIN + 16, "ring must hold a group and an unflushed window");

struct WarpSmem {
    uint32_t lit[1 << LB];
    uint32_t dist[1 << DB];
    uint32_t scratch[48];
    uint16_t lsorted[288];
    uint16_t dsorted[32];
    uint16_t lcount[16];
    uint16_t dcount[16];
    uint8_t lens[352];
    uint32_t tok[NTOK];
    alignas(16) uint8_t ring[RING];
};

struct CtaSmem {
    uint32_t crc8[8][256];
    uint32_t mulk[4][256];
    WarpSmem w[WARPS];
};

}  // namespace lk

// Write tokens [0, nt) of the warp's buffer at the member's output position.
__device__ uint32_t materialize(int nt, Out& o, lk::WarpSmem& W, const lk::CtaSmem& S, bool crc) {
    const int lane = threadIdx.x & 31;
    for (int g0 = 0; g0 < nt;) {
        const int t = g0 + lane;
        const bool have = t < nt;
        const uint32_t tk = have ? W.tok[t] : 0u;
        const uint32_t len = have ? tok_len(tk) : 0u;
        uint32_t gsum;
        const uint32_t ex = warp_exclusive_scan(len, gsum);
        const unsigned takem = __ballot_sync(FULL, have && ex < lk::GROUP);
        const int gcount = __popc(takem);
        const bool valid = lane < gcount;
        const uint32_t glen = __shfl_sync(FULL, ex + len, gcount - 1);
        const uint32_t q = o.p + ex;
        const bool is_m = valid && tok_match(tk);
        const uint32_t dist = is_m ? tok_dist(tk) : 0u;
        if (__any_sync(FULL, valid && (q + len > o.isize || dist > q))) return CB_ERR_INFLATE;
        if (valid && !is_m) W.ring[slot_of<lk::RING>(q + o.a)] = (uint8_t)tk;
        __syncwarp();
        const uint32_t q1 = o.p + glen;
        const long long lim = (long long)q1 - (long long)lk::RING;  // sources below it: flushed, in HBM
        bool pend = is_m;
        for (int it = 0; it < 33; it++) {
            if (!__any_sync(FULL, pend)) break;
            const uint32_t P = __reduce_min_sync(FULL, pend ? q : 0xFFFFFFFFu);
            const bool ready = pend && (q - dist + min(len, dist) <= P);
            if (ready) {
                const uint32_t src = q - dist;
                // an overlapping copy (dist < len) reads bytes this loop wrote before
                for (uint32_t j = 0; j < len; j++) {
                    const uint32_t x = src + j;
                    const uint8_t v = (long long)x >= lim ? W.ring[slot_of<lk::RING>(x + o.a)] : o.out[x];
                    W.ring[slot_of<lk::RING>(q + j + o.a)] = v;
                }
            }
            __syncwarp();
            pend = pend && !ready;
        }
        o.p = q1;
        flush_ready<lk::RING>(o, W, S, crc);
        g0 += gcount;
    }
    return CB_OK;
}

// The Huffman-coded data of one block, from the reader's position to its end-of-block code; the
// reader is left after the end-of-block code.
//
// The hot loop keeps the two current input words (lo, hi) and a bit offset, the same in every lane:
// one funnel shift gives the next 32 bits, a symbol's code and extra bits are taken from that window
// and consumed with one add; a word is pulled from the lane registers of the current 128-byte group
// (__shfl_sync) only when the offset passes 32.
__device__ uint32_t lock_block(Reader& r, long long in_bits, Out& o, lk::WarpSmem& W, const lk::CtaSmem& S,
                               bool crc) {
    const int lane = threadIdx.x & 31;
    const long long A = consumed(r) + r.s0;
    const uint32_t w0 = (uint32_t)(A >> 5);
    uint32_t off = (uint32_t)(A & 31);
    uint32_t lo = load_word(r.wbase, r.nvalid, w0), hi = load_word(r.wbase, r.nvalid, w0 + 1);
    uint32_t g = (w0 + 2) >> 5, widx = (w0 + 2) & 31;  // the next word to pull into hi
    uint32_t gw = load_word(r.wbase, r.nvalid, g * 32u + lane);
    uint32_t gn = load_word(r.wbase, r.nvalid, (g + 1) * 32u + lane);
    auto advance = [&](uint32_t n) {
        off += n;
        if (off >= 32) {
            off -= 32;
            lo = hi;
            hi = __shfl_sync(FULL, gw, widx);
            if (++widx == 32) {
                widx = 0;
                g++;
                gw = gn;
                gn = load_word(r.wbase, r.nvalid, (g + 1) * 32u + lane);
            }
        }
    };
    for (;;) {
        int nt = 0;
        bool eob = false;
        while (nt < lk::NTOK) {
            const uint32_t x = __funnelshift_r(lo, hi, off);
            uint32_t e = W.lit[x & LMASK];
            uint32_t kind = e_kind(e);
            if (kind == K_LIT) {
                advance(e_bits(e));
                if (lane == 0) W.tok[nt] = e_value(e);
                nt++;
                continue;
            }
            if (kind == K_SLOW) {
                e = slow_decode((uint64_t)x, W.lcount, W.lsorted, T_LIT);
                kind = e_kind(e);
                if (kind == K_LIT) {
                    advance(e_bits(e));
                    if (lane == 0) W.tok[nt] = e_value(e);
                    nt++;
                    continue;
                }
            }
            if (kind == K_EOB) {
                advance(e_bits(e));
                eob = true;
                break;
            }
            if (kind != K_LEN) return CB_ERR_INFLATE;
            const uint32_t cb = e_bits(e), ext = e_extra(e);
            const uint32_t len = e_value(e) + ((x >> cb) & ((1u << ext) - 1u));
            advance(cb + ext);
            const uint32_t y = __funnelshift_r(lo, hi, off);
            uint32_t d = W.dist[y & DMASK];
            if (e_kind(d) == K_SLOW) d = slow_decode((uint64_t)y, W.dcount, W.dsorted, T_DIST);
            if (e_kind(d) != K_LEN) return CB_ERR_INFLATE;
            const uint32_t db = e_bits(d), dext = e_extra(d);
            const uint32_t dist = e_value(d) + ((y >> db) & ((1u << dext) - 1u));
            advance(db + dext);
            if (lane == 0) W.tok[nt] = 0x80000000u | (len << 16) | (dist - 1);
            nt++;
        }
        const long long pos = ((long long)g * 32 + widx - 2) * 32 + off - r.s0;  // bits consumed
        if (pos > in_bits) return CB_ERR_INFLATE;
        __syncwarp();
        const uint32_t st = materialize(nt, o, W, S, crc);
        if (st != CB_OK) return st;
        if (eob) {
            seek(r, pos);
            return CB_OK;
        }
    }
}

// ---------------------------------------------------------------- one member

template <bool SPEC, uint32_t RN, class WS, class CS>
__device__ uint32_t inflate_member(const cb_member_job& job, uint8_t* out_base, bool crc, WS& W, const CS& S) {
    const int lane = threadIdx.x & 31;
    Reader r;
    uintptr_t in = (uintptr_t)job.in;
    r.wbase = reinterpret_cast<const uint32_t*>(in & ~(uintptr_t)3);
    r.s0 = (uint32_t)(in & 3) * 8;
    r.nvalid = (uint32_t)((in + job.in_len + 8 - (uintptr_t)r.wbase) >> 2);
    seek(r, 0);

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
                uint32_t cnt = min(32u, len - k);
                if ((uint32_t)lane < cnt) W.ring[slot_of<RN>(o.p + lane + o.a)] = src[k + lane];
                o.p += cnt;
                __syncwarp();
                flush_ready<RN>(o, W, S, crc);
            }
            seek(r, (byte + len) * 8);
            continue;
        }
        if (btype == 3) return CB_ERR_INFLATE;
        const uint32_t tst = read_tables(r, W, btype);
        if (tst != CB_OK) return tst;
        // ------------------------------------------------ Huffman-coded data
        if constexpr (SPEC) {
            long long pos = consumed(r);
            uint32_t st = spec_block(pos, r.wbase, r.nvalid, r.s0, in_bits, o, W, S, crc);
            if (st != CB_OK) return st;
            seek(r, pos);
        } else {
            uint32_t st = lock_block(r, in_bits, o, W, S, crc);
            if (st != CB_OK) return st;
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

__global__ void __launch_bounds__(WARPS * 32, 1) k_inflate(const cb_member_job* __restrict__ jobs, int64_t n_jobs,
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
        uint32_t st = inflate_member<true, RING>(job, out_base, crc, W, S);
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

__global__ void __launch_bounds__(lk::WARPS * 32, 2) k_inflate_lk(const cb_member_job* __restrict__ jobs, int64_t n_jobs,
                                                           const int64_t* __restrict__ d_n_jobs, uint8_t* out_base,
                                                           int check_crc, uint32_t* job_status,
                                                           cb_inflate_summary* summary, unsigned long long* queue) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    lk::CtaSmem& S = *reinterpret_cast<lk::CtaSmem*>(smem_raw);
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
    lk::WarpSmem& W = S.w[warp];
    int64_t n = n_jobs;
    if (d_n_jobs) n = min(n, *d_n_jobs);
    const bool crc = check_crc != 0;
    for (;;) {
        unsigned long long j = 0;
        if (lane == 0) j = atomicAdd(queue, 1ull);
        j = __shfl_sync(FULL, j, 0);
        if ((int64_t)j >= n) break;
        cb_member_job job = jobs[j];
        uint32_t st = inflate_member<false, lk::RING>(job, out_base, crc, W, S);
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
static int g_lk_blocks_per_sm = -1;
static int g_variant = -1;  // 0 speculative, 1 lock-step

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
    if (g_variant < 0) {
        const char* v = getenv("CUBAM_B200_INFLATE");
        g_variant = (v && v[0] == 's') ? 0 : 1;
    }
    const size_t smem_lk = sizeof(infl::lk::CtaSmem);
    if (g_lk_blocks_per_sm < 0) {
        cudaError_t e = cudaFuncSetAttribute(infl::k_inflate_lk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem_lk);
        if (e != cudaSuccess) return cb_set_error(e);
        int b = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, infl::k_inflate_lk, infl::lk::WARPS * 32, smem_lk);
        if (e != cudaSuccess) return cb_set_error(e);
        g_lk_blocks_per_sm = b > 0 ? b : 1;
    }
    infl::k_inflate_init<<<1, 1, 0, s>>>(summary, queue);
    if (n_jobs > 0 && g_variant == 0) {
        long long grid = (long long)cb_device_sm_count() * g_inflate_blocks_per_sm;
        long long by_work = (n_jobs + infl::WARPS - 1) / infl::WARPS;
        if (!d_n_jobs && by_work < grid) grid = by_work;
        if (grid < 1) grid = 1;
        infl::k_inflate<<<(unsigned)grid, infl::WARPS * 32, smem, s>>>(jobs, n_jobs, d_n_jobs, out_base, check_crc,
                                                                        job_status, summary, queue);
    } else if (n_jobs > 0) {
        long long grid = (long long)cb_device_sm_count() * g_lk_blocks_per_sm;
        long long by_work = (n_jobs + infl::lk::WARPS - 1) / infl::lk::WARPS;
        if (!d_n_jobs && by_work < grid) grid = by_work;
        if (grid < 1) grid = 1;
        infl::k_inflate_lk<<<(unsigned)grid, infl::lk::WARPS * 32, smem_lk, s>>>(
            jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, queue);
    }
    infl::k_inflate_finish<<<1, 1, 0, s>>>(summary);
    return cb_set_error(cudaGetLastError());
}
