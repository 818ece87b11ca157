// Raw-DEFLATE inflater for BGZF members on B200 (sm_100a), with the CRC32 and ISIZE checks.
//
// Replaces cubam's call of nvcompBatchedDeflateDecompressAsync and its status/size check
// (src/cubam/bgzf.py:587-611); the CRC32 check is new (cubam's reader does not check it,
// docs/reading.md:48-51).  DEFLATE itself is RFC 1951.
//
// Huffman decoding is serial within a member; the parallelism is across members.  Two forms, both
// persistent grids that take members from a work queue, with the same per-member results:
//
//  1. one member per warp (k_inflate_warp, 32 warps per SM): the warp reads the bit stream in lock
//     step, decodes a batch of symbols into tokens and writes them warp-parallel.
//  2. one member per lane (k_inflate_lanes): 8 lanes of each of 16 warps per SM each inflate a
//     member of their own, 128 members per SM in flight.
//
// cb_inflate runs form 1 (the faster at every batch size measured); cb_inflate_form takes the form
// from the caller.
//
// Every loop is bounded by the member's sizes or a fixed count: output beyond ISIZE, a distance
// before the member's start, bits read beyond the payload, bad code lengths and invalid symbols are
// per-member errors.

#include "common.cuh"
#include "crc.cuh"

namespace cb {
namespace infl {

constexpr int LB = 8;                     // literal/length root bits (form 1)
constexpr int DB = 7;                     // distance root bits (form 1)
constexpr int CLB = 7;                    // code-length code bits
constexpr int WIN = 1024;                 // form 1 flush / CRC window
constexpr uint32_t LMASK = (1u << LB) - 1, DMASK = (1u << DB) - 1;
static_assert(WIN == 32 * 32, "one 32-byte CRC column per lane");
static_assert(15 - LB <= 8 && 15 - DB <= 8 && LB >= DB, "limits of the longer codes fit their arrays");

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

// Canonical Huffman table of lens[0:nsym): tab[2^lb] indexed by the next lb bits; for the codes
// longer than lb bits, sorted[] (the symbols in canonical order) and, for code length lb + 1 + i,
// lim[i] = (end of the length's codes, left-justified to 15 bits) | (index of its first code in
// sorted[] minus its first code) << 16.  Returns false for an over-subscribed code, or an
// incomplete one except a single code of length 1 (literal/length and distance codes), as zlib's
// inflate accepts.
__device__ __noinline__ bool build_table(const uint8_t* lens, int nsym, int lb, int kind, uint32_t* tab, uint32_t* lim,
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
    if (lim && lane > lb && lane < 16) {
        const uint32_t limit = (my_first + cnt) << (15 - lane);
        const int base = (int)my_index - (int)my_first;
        lim[lane - lb - 1] = (limit & 0xFFFFu) | ((uint32_t)(uint16_t)(int16_t)base << 16);
    }
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

// The table entry, with its full code length, of a code longer than the root bits (N = 15 - root
// bits): x holds at least the next 15 bits.  The same in every lane.
template <int N>
__device__ __forceinline__ uint32_t slow_decode(uint32_t x, const uint32_t* lim, const uint16_t* sorted, int nsym,
                                                int kind) {
    const uint32_t c = __brev(x) >> 17;  // the next 15 bits, first bit highest
    int idx = -1;
    uint32_t L = 0;
#pragma unroll
    for (int i = N - 1; i >= 0; i--) {
        const uint32_t e = lim[i];
        if (c < (e & 0xFFFFu)) {
            idx = (int)(int16_t)(e >> 16) + (int)(c >> (N - 1 - i));
            L = (uint32_t)(16 - N + i);
        }
    }
    return (idx >= 0 && idx < nsym) ? sym_entry(kind, sorted[idx], L) : entry(1, K_BAD, 0, 0);
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

__device__ __forceinline__ long long shfl_ll(long long v, int src) {
    int lo = __shfl_sync(FULL, (int)(v & 0xffffffff), src), hi = __shfl_sync(FULL, (int)(v >> 32), src);
    return ((long long)hi << 32) | (unsigned)lo;
}

// The Huffman tables of a fixed (btype 1) or dynamic (btype 2) block, the dynamic header read by the
// whole warp in lock step.  CB_OK or CB_ERR_INFLATE.
template <class WS> __device__ uint32_t read_tables(Reader& r, WS& W, uint32_t btype) {
    const int lane = threadIdx.x & 31;
    if (btype == 1) {
        for (int s = lane; s < 288; s += 32) W.lens[s] = s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : 8;
        for (int s = lane; s < 32; s += 32) W.lens[288 + s] = 5;
        __syncwarp();
        if (!build_table(W.lens, 288, LB, T_LIT, W.lit, W.llim, W.lsorted, W.scratch)) return CB_ERR_INFLATE;
        if (!build_table(W.lens + 288, 32, DB, T_DIST, W.dist, W.dlim, W.dsorted, W.scratch))
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
        if (!build_table(L, (int)hlit, LB, T_LIT, W.lit, W.llim, W.lsorted, W.scratch)) return CB_ERR_INFLATE;
        if (!build_table(L + hlit, (int)hdist, DB, T_DIST, W.dist, W.dlim, W.dsorted, W.scratch))
            return CB_ERR_INFLATE;
    }
    return CB_OK;
}

// ================================================================ form 1: one member per warp
// 8 warps per CTA, 2 CTAs per SM.  The warp decodes symbols in lock step into a token buffer only
// (no output writes, no copies in the serial loop), then writes the batch of tokens warp-parallel:
// 32 tokens per group, literals at once, matches in waves (ready when the source lies before the
// first unfinished match).  Back-references within the 4 KB ring read shared memory, older ones
// read the flushed output in HBM.

namespace wm {

constexpr int WARPS = 8;
constexpr int NTOK = 128;                 // tokens decoded before a batch is written
constexpr uint32_t RING = 2048;
constexpr uint32_t GROUP = 512;           // a group of tokens starts within this many output bytes
static_assert(RING >= GROUP + 258 + WIN + 16, "ring must hold a group and an unflushed window");

struct WarpSmem {
    uint32_t lit[1 << LB];
    uint32_t dist[1 << DB];
    uint32_t scratch[48];
    uint16_t lsorted[288];
    uint16_t dsorted[32];
    uint32_t llim[8];            // limits of the literal/length codes longer than LB bits
    uint32_t dlim[8];            // limits of the distance codes longer than DB bits
    uint8_t lens[352];
    uint32_t tok[NTOK];
    alignas(16) uint8_t ring[RING];
};

struct CtaSmem {
    uint32_t crc8[8][256];
    uint32_t mulk[4][256];
    WarpSmem w[WARPS];
};

}  // namespace wm

// Write tokens [0, nt) of the warp's buffer at the member's output position.
__device__ uint32_t materialize(int nt, Out& o, wm::WarpSmem& W, const wm::CtaSmem& S, bool crc) {
    const int lane = threadIdx.x & 31;
    for (int g0 = 0; g0 < nt;) {
        const int t = g0 + lane;
        const bool have = t < nt;
        const uint32_t tk = have ? W.tok[t] : 0u;
        const uint32_t len = have ? tok_len(tk) : 0u;
        uint32_t gsum;
        const uint32_t ex = warp_exclusive_scan(len, gsum);
        const unsigned takem = __ballot_sync(FULL, have && ex < wm::GROUP);
        const int gcount = __popc(takem);
        const bool valid = lane < gcount;
        const uint32_t glen = __shfl_sync(FULL, ex + len, gcount - 1);
        const uint32_t q = o.p + ex;
        const bool is_m = valid && tok_match(tk);
        const uint32_t dist = is_m ? tok_dist(tk) : 0u;
        if (__any_sync(FULL, valid && (q + len > o.isize || dist > q))) return CB_ERR_INFLATE;
        const uint32_t q1 = o.p + glen;
        const long long lim = (long long)q1 - (long long)wm::RING;  // sources below it: flushed, in HBM
        // the group's bytes, 32 at a time: lane j writes byte r0 + j.  Its symbol is found by a binary
        // search over the symbols' offsets; a literal gives the byte, a match byte is the byte dist
        // before it -- in the ring or HBM when that lies before this round, else the byte another lane
        // computes in this round (pointer jumping: at most 5 exchanges for a chain of 31)
        for (uint32_t r0 = 0; r0 < glen; r0 += 32) {
            const uint32_t rel = r0 + lane;
            const bool act = rel < glen;
            int k = 0;
#pragma unroll
            for (int step = 16; step; step >>= 1) {
                const int c = k + step;
                const uint32_t exc = __shfl_sync(FULL, ex, c & 31);
                if (c < gcount && exc <= rel) k = c;
            }
            const uint32_t tkk = __shfl_sync(FULL, tk, k);
            const uint32_t b = o.p + rel;
            const uint32_t base = o.p + r0;
            uint32_t val = tkk & 0xFFu;
            int src = lane;  // lane of this round that holds the byte's source (itself: resolved)
            if (act && tok_match(tkk)) {
                const uint32_t x = b - tok_dist(tkk);
                if (x >= base) src = (int)(x - base);
                else val = (long long)x >= lim ? W.ring[slot_of<wm::RING>(x + o.a)] : o.out[x];
            }
            bool need = src != lane;
            for (int it = 0; it < 6 && __any_sync(FULL, need); it++) {
                const uint32_t v2 = __shfl_sync(FULL, val, src);
                const int s2 = __shfl_sync(FULL, src, src);
                const bool n2 = __shfl_sync(FULL, (int)need, src) != 0;
                if (need) {
                    if (!n2) {
                        val = v2;
                        need = false;
                    } else {
                        src = s2;
                    }
                }
            }
            if (act) W.ring[slot_of<wm::RING>(b + o.a)] = (uint8_t)val;
            __syncwarp();
        }
        o.p = q1;
        flush_ready<wm::RING>(o, W, S, crc);
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
__device__ uint32_t lock_block(Reader& r, long long in_bits, Out& o, wm::WarpSmem& W, const wm::CtaSmem& S,
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
        while (nt < wm::NTOK) {
            uint32_t x = __funnelshift_r(lo, hi, off);
            uint32_t e = W.lit[x & LMASK];
            while (e_kind(e) == K_LIT) {  // a run of literals: the tight loop of the common case
                advance(e_bits(e));
                if (lane == 0) W.tok[nt] = e_value(e);
                if (++nt == wm::NTOK) break;
                x = __funnelshift_r(lo, hi, off);
                e = W.lit[x & LMASK];
            }
            if (nt == wm::NTOK) break;
            uint32_t kind = e_kind(e);
            if (kind == K_SLOW) {
                e = slow_decode<15 - LB>(x, W.llim, W.lsorted, 288, T_LIT);
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
            if (e_kind(d) == K_SLOW) d = slow_decode<15 - DB>(y, W.dlim, W.dsorted, 32, T_DIST);
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

// ---------------------------------------------------------------- form 1: one member

__device__ uint32_t inflate_member(const cb_member_job& job, uint8_t* out_base, bool crc, wm::WarpSmem& W,
                                   const wm::CtaSmem& S) {
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
                if ((uint32_t)lane < cnt) W.ring[slot_of<wm::RING>(o.p + lane + o.a)] = src[k + lane];
                o.p += cnt;
                __syncwarp();
                flush_ready<wm::RING>(o, W, S, crc);
            }
            seek(r, (byte + len) * 8);
            continue;
        }
        if (btype == 3) return CB_ERR_INFLATE;
        const uint32_t tst = read_tables(r, W, btype);
        if (tst != CB_OK) return tst;
        const uint32_t st = lock_block(r, in_bits, o, W, S, crc);
        if (st != CB_OK) return st;
    }
    if (consumed(r) > in_bits || o.p != isize) return CB_ERR_INFLATE;
    if (crc && finish_crc(o.col, isize) != job.crc) return CB_ERR_CRC;
    return CB_OK;
}

// ================================================================ form 2: one member per lane
// MLANES lanes of each warp inflate a member of their own (the warp's other lanes only help with
// block headers).  Everything a lane decodes with is in shared memory or registers: a 2^LNB-entry
// literal/length table and a 2^LDB-entry distance table of 16-bit entries, the entries of the
// longer codes in canonical order, and, in registers, the limits of the longer code lengths; plus a
// 256-byte output ring and the running CRC32 of the bytes stored so far (in order, slice-by-8
// tables shared by the CTA).
//
// A lane's step makes its next copy (a literal, or up to 16 bytes of a match or stored block) and
// carries out the copy made by its previous step, so the load of a back-reference beyond the ring
// (issued when the copy is made; those bytes are already in HBM) overlaps a decode.  Every copy is
// one 16-byte store into the ring; a match of distance d < 16 copies d, 2d, 4d, ... bytes at a time
// (from one period before its start the bytes repeat with period d).  Every STEPS steps each lane
// stores the complete 16-byte units of its ring to HBM (16-byte aligned) and folds them into its
// CRC.  Block headers, stored-block headers and code tables are read by the whole warp for one lane
// at a time (the lock-step reader and a warp table builder).

// Entries of the 16-bit tables: code length << 12 | kind << 10 | value, with kind 0 literal (value:
// the byte), 1 length or distance (value: symbol index), 2 end of block, 3 special (value 0: a
// longer code; value 1: no such code).
__device__ __forceinline__ uint16_t e16(uint32_t L, uint32_t kind, uint32_t v) {
    return (uint16_t)((L << 12) | (kind << 10) | v);
}
constexpr uint16_t E16_SLOW = (uint16_t)(3u << 10);
constexpr uint16_t E16_BAD = (uint16_t)((3u << 10) | 1u);

__device__ __forceinline__ uint16_t sym_entry16(int kind, uint32_t s, uint32_t L) {
    if (kind == T_LIT) {
        if (s < 256) return e16(L, 0, s);
        if (s == 256) return e16(L, 2, 0);
        if (s < 286) return e16(L, 1, s - 257);
        return E16_BAD;
    }
    if (s < 30) return e16(L, 1, s);
    return E16_BAD;
}

namespace ln {

template <int LNB_, int LDB_, int WARPS_, int STEPS_, int MLANES_>
struct Cfg {
    static constexpr int LNB = LNB_, LDB = LDB_, WARPS = WARPS_, STEPS = STEPS_, MLANES = MLANES_;
    static constexpr int NLL = 15 - LNB_, NLD = 15 - LDB_;  // longer code lengths per table
    static constexpr uint32_t LRING = 256, RSTRIDE = LRING + 16;
    static constexpr uint32_t RV = 224;     // back-references up to this distance read the ring
    static constexpr uint32_t PAUSE = 192;  // a lane with more unstored bytes waits for the next store
    static constexpr int LSTRIDE = (1 << LNB_) + 2, DSTRIDE = (1 << LDB_) + 2;  // odd word strides
    static constexpr int LSYM = 290, DSYM = 34;
    // A 16-byte copy into the ring writes up to 4 bytes past its end, so at output position x the
    // ring holds [x + 19 - LRING, x) intact.  A copy is made at most 16 bytes above the output
    // position, which is at most PAUSE bytes above the stored units; a step adds at most 16.
    static_assert(RV + 19 <= LRING, "back-references up to RV read intact ring bytes");
    static_assert(PAUSE + 31 <= RV, "longer back-references read bytes already stored in HBM");
    static_assert(PAUSE + 16 + 19 <= LRING, "the unstored bytes stay intact in the ring");
    static_assert(16 + 16 * STEPS_ <= (int)PAUSE, "no lane waits between two stores in the steady state");
    static_assert(NLL <= 8 && NLD <= 9 && MLANES_ <= 32, "register limits, lanes");

    struct WarpSmem {
        uint16_t lit[MLANES_ * LSTRIDE];
        uint16_t lsym[MLANES_ * LSYM];
        uint16_t dist[MLANES_ * DSTRIDE];
        uint16_t dsym[MLANES_ * DSYM];
        uint32_t lim[20];  // limits of the lane whose tables were just built
        uint32_t cltab[1 << CLB];
        uint32_t scratch[48];
        uint8_t lens[352];
        alignas(16) uint8_t ring[MLANES_ * RSTRIDE];
    };
    struct CtaSmem {
        uint32_t crc8[8][256];
        uint32_t li[32];  // length symbol: base | extra bits << 16
        uint32_t di[32];  // distance symbol: base | extra bits << 16
        WarpSmem w[WARPS_];
    };
};

// The configuration in use: 7 + 6 root bits, 16 warps of 8 member lanes, a store every 8 steps.
using Form2 = Cfg<7, 6, 16, 8, 8>;

enum : int { IDLE = 0, HEADER = 1, RUN = 2, FIN = 3, DONE = 4 };

}  // namespace ln

// Canonical table of lens[0:nsym) for one lane: tab[2^lb] (16-bit entries) indexed by the next lb
// bits; the codes longer than lb bits have their entries in sym[] in canonical order and, for code
// length lb + 1 + i, lim[i] = (end of the length's codes, left-justified to 15 bits) | (index of
// its first code in sym[] minus its first code) << 16.  The acceptance rules are build_table's.
__device__ __noinline__ bool build_lane_table(const uint8_t* lens, int nsym, int lb, int kind, uint16_t* tab,
                                              uint32_t* lim, uint16_t* sym, uint32_t* scratch) {
    const int lane = threadIdx.x & 31;
    if (lane < 16) scratch[lane] = 0;
    __syncwarp();
    for (int s = lane; s < nsym; s += 32) {
        const uint32_t L = lens[s];
        if (L) atomicAdd(&scratch[L], 1u);
    }
    __syncwarp();
    const uint32_t cnt = (lane >= 1 && lane < 16) ? scratch[lane] : 0u;
    int left = 1, maxlen = 0;
    uint32_t code = 0, index = 0, my_first = 0, my_index = 0;
    for (int L = 1; L < 16; L++) {
        const uint32_t c = __shfl_sync(FULL, cnt, L);
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
    const bool incomplete = left > 0;
    if (incomplete && maxlen > 1) return false;
    const uint32_t nshort = __shfl_sync(FULL, my_index, lb + 1);
    if (lane > lb && lane < 16) {
        const uint32_t limit = (my_first + cnt) << (15 - lane);
        const int base = (int)(my_index - nshort) - (int)my_first;
        lim[lane - lb - 1] = (limit & 0xFFFFu) | ((uint32_t)(uint16_t)(int16_t)base << 16);
    }
    if (lane >= 1 && lane < 16) {
        scratch[lane] = my_index;
        scratch[16 + lane] = my_first;
        scratch[32 + lane] = my_index;
    }
    if (incomplete || maxlen == 0)
        for (int i = lane; i < (1 << lb); i += 32) tab[i] = E16_BAD;
    __syncwarp();
    for (int base = 0; base < nsym; base += 32) {
        const int s = base + lane;
        const uint32_t L = s < nsym ? lens[s] : 0u;
        const uint32_t peers = __match_any_sync(FULL, L);
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        const uint32_t pos = L ? scratch[L] : 0u;
        __syncwarp();
        if (L && lane == __ffs(peers) - 1) scratch[L] = pos + __popc(peers);
        __syncwarp();
        if (L) {
            const uint32_t idx = pos + rank;
            const uint32_t c = scratch[16 + L] + (idx - scratch[32 + L]);
            const uint16_t e = sym_entry16(kind, (uint32_t)s, L);
            if ((int)L <= lb) {
                const uint32_t r = __brev(c) >> (32 - L);
                for (uint32_t x = r; x < (1u << lb); x += (1u << L)) tab[x] = e;
            } else {
                sym[idx - nshort] = e;
                tab[__brev(c >> (L - lb)) >> (32 - lb)] = E16_SLOW;
            }
        }
        __syncwarp();
    }
    return true;
}

// Lane t's tables for a fixed (btype 1) or dynamic (btype 2) block, the header read by the whole
// warp in lock step from r; the limits go to W.lim[0:NLL) and W.lim[NLL:NLL+NLD).
// CB_OK or CB_ERR_INFLATE.
template <class C>
__device__ uint32_t read_lane_tables(Reader& r, typename C::WarpSmem& W, uint32_t btype, int t) {
    const int lane = threadIdx.x & 31;
    const uint8_t* L;
    uint32_t hlit, hdist;
    if (btype == 1) {
        for (int s = lane; s < 288; s += 32) W.lens[s] = s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : 8;
        W.lens[288 + lane] = 5;
        __syncwarp();
        L = W.lens;
        hlit = 288;
        hdist = 32;
    } else {
        if (r.bc < 32) refill(r);
        hlit = ((uint32_t)r.bb & 31u) + 257;
        hdist = (((uint32_t)r.bb >> 5) & 31u) + 1;
        const uint32_t hclen = (((uint32_t)r.bb >> 10) & 15u) + 4;
        consume(r, 14);
        if (hlit > 286 || hdist > 30) return CB_ERR_INFLATE;
        if (lane < 19) W.lens[lane] = 0;
        __syncwarp();
        for (uint32_t base = 0; base < hclen; base += 10) {
            if (r.bc < 32) refill(r);
            const uint32_t cnt = min(10u, hclen - base);
            if ((uint32_t)lane < cnt) W.lens[kClOrder[base + lane]] = (uint8_t)((r.bb >> (3 * lane)) & 7u);
            consume(r, 3 * cnt);
        }
        __syncwarp();
        if (!build_table(W.lens, 19, CLB, T_CLEN, W.cltab, nullptr, nullptr, W.scratch)) return CB_ERR_INFLATE;
        const uint32_t total = hlit + hdist;
        uint32_t i = 0;
        uint8_t* D = W.lens + 32;
        while (i < total) {
            if (r.bc < 32) refill(r);
            const uint32_t e = W.cltab[(uint32_t)r.bb & ((1u << CLB) - 1)];
            if (e_kind(e) != K_LIT) return CB_ERR_INFLATE;
            consume(r, (int)e_bits(e));
            const uint32_t sym = e_value(e);
            if (sym < 16) {
                if (lane == 0) D[i] = (uint8_t)sym;
                i++;
                continue;
            }
            uint32_t rep, val = 0;
            if (sym == 16) {
                if (i == 0) return CB_ERR_INFLATE;
                __syncwarp();
                val = D[i - 1];
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
            for (uint32_t j = lane; j < rep; j += 32) D[i + j] = (uint8_t)val;
            i += rep;
        }
        __syncwarp();
        if (D[256] == 0) return CB_ERR_INFLATE;  // no end-of-block code
        L = D;
    }
    if (!build_lane_table(L, (int)hlit, C::LNB, T_LIT, W.lit + t * C::LSTRIDE, W.lim, W.lsym + t * C::LSYM,
                          W.scratch))
        return CB_ERR_INFLATE;
    if (!build_lane_table(L + hlit, (int)hdist, C::LDB, T_DIST, W.dist + t * C::DSTRIDE, W.lim + C::NLL,
                          W.dsym + t * C::DSYM, W.scratch))
        return CB_ERR_INFLATE;
    return CB_OK;
}

// The entry of a code longer than the table's root bits, from the lane's limits (registers): bits
// holds at least the next 15 bits.
template <int N>
__device__ __forceinline__ uint32_t long_code(uint32_t bits, const uint32_t (&lim)[N], const uint16_t* sym, int nsym) {
    const uint32_t c = __brev(bits) >> 17;  // the next 15 bits, first bit highest
    int idx = -1;
#pragma unroll
    for (int i = N - 1; i >= 0; i--) {
        if (c < (lim[i] & 0xFFFFu)) idx = (int)(int16_t)(lim[i] >> 16) + (int)(c >> (N - 1 - i));
    }
    return (idx >= 0 && idx < nsym) ? (uint32_t)sym[idx] : (uint32_t)E16_BAD;
}

// 16 bytes from ptr (any alignment) with aligned 16-byte loads; the second unit only when it holds
// a byte below limit (ptr < limit).  RO: the bytes are read-only for the kernel's lifetime (the
// payload); otherwise this thread stored them earlier in the kernel and they are read from L2.
template <bool RO>
__device__ __forceinline__ void gather16(const uint8_t* ptr, const uint8_t* limit, uint32_t (&v)[4]) {
    const uintptr_t A = (uintptr_t)ptr & ~(uintptr_t)15;
    const uint4* P = reinterpret_cast<const uint4*>(A);
    const uint4 u0 = RO ? __ldg(P) : __ldcg(P);
    uint4 u1 = make_uint4(0, 0, 0, 0);
    if ((uintptr_t)ptr != A && A + 16 < (uintptr_t)limit) u1 = RO ? __ldg(P + 1) : __ldcg(P + 1);
    const uint32_t s = (uint32_t)((uintptr_t)ptr & 15), q = s >> 2, sh = (s & 3) * 8;
    uint32_t w0 = u0.x, w1 = u0.y, w2 = u0.z, w3 = u0.w, w4 = u1.x, w5 = u1.y, w6 = u1.z, w7 = u1.w;
    if (q & 2) {
        w0 = w2; w1 = w3; w2 = w4; w3 = w5; w4 = w6; w5 = w7;
    }
    if (q & 1) {
        w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5;
    }
    v[0] = __funnelshift_r(w0, w1, sh);
    v[1] = __funnelshift_r(w1, w2, sh);
    v[2] = __funnelshift_r(w2, w3, sh);
    v[3] = __funnelshift_r(w3, w4, sh);
}

// 16 bytes of a lane ring of RW words from byte slot s.
template <uint32_t RW>
__device__ __forceinline__ void ring_load16(const uint32_t* ring, uint32_t s, uint32_t (&v)[4]) {
    const uint32_t w = s >> 2, sh = (s & 3) * 8;
    uint32_t r[5];
#pragma unroll
    for (int k = 0; k < 5; k++) r[k] = ring[(w + k) & (RW - 1)];
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = __funnelshift_r(r[k], r[k + 1], sh);
}

// Store 16 bytes at byte slot d of a lane ring; the bytes before d in its word are kept, the 4 bytes
// after the 16 get whatever comes (they are above the bytes written so far).
template <uint32_t RW>
__device__ __forceinline__ void ring_store16(uint32_t* ring, uint32_t d, const uint32_t (&v)[4]) {
    const uint32_t w = d >> 2, f = d & 3, sh = 8 * f;
    const uint32_t keep = f ? (0xFFFFFFFFu >> (32 - sh)) : 0u;
    ring[w] = (ring[w] & keep) | (v[0] << sh);
    ring[(w + 1) & (RW - 1)] = __funnelshift_l(v[0], v[1], sh);
    ring[(w + 2) & (RW - 1)] = __funnelshift_l(v[1], v[2], sh);
    ring[(w + 3) & (RW - 1)] = __funnelshift_l(v[2], v[3], sh);
    if (f) ring[(w + 4) & (RW - 1)] = v[3] >> (32 - sh);
}

// State of the member a lane inflates.
struct Lane {
    int st;
    uint32_t err;
    bool final_block, stored;
    long long j;                 // job index
    const uint8_t* in;           // payload
    const uint32_t* wbase;
    uint32_t nvalid, s0, in_len;
    uint64_t bb;                 // bit buffer, LSB first
    int bc;
    uint32_t nextw, pre;         // next word to load, prefetched word
    uint32_t bitpos;             // bits consumed, when the lane leaves its Huffman data
    uint8_t* out;
    uint32_t a, isize, want_crc;
    uint32_t p, flushed, crc;    // bytes in the ring, bytes stored in HBM, running CRC
    uint32_t rem, dist, spos;    // match or stored block in progress
};

__device__ __forceinline__ void ln_seek(Lane& L, uint32_t pos) {
    const uint32_t a = pos + L.s0, w = a >> 5, sh = a & 31;
    const uint64_t x = (uint64_t)load_word(L.wbase, L.nvalid, w) | ((uint64_t)load_word(L.wbase, L.nvalid, w + 1) << 32);
    L.bb = x >> sh;
    L.bc = 64 - (int)sh;
    L.pre = load_word(L.wbase, L.nvalid, w + 2);
    L.nextw = w + 3;
}

__device__ __forceinline__ void ln_refill(Lane& L) {
    if (L.bc < 32) {
        L.bb |= (uint64_t)L.pre << L.bc;
        L.bc += 32;
        L.pre = load_word(L.wbase, L.nvalid, L.nextw);
        L.nextw++;
    }
}

__device__ __forceinline__ uint32_t ln_bitpos(const Lane& L) { return (L.nextw - 1) * 32u - (uint32_t)L.bc - L.s0; }

// A copy made by a lane's step and carried out by its next step.
enum : uint32_t { OP_NONE = 0, OP_LIT = 1, OP_RING = 2, OP_LOADED = 3 };

struct Op {
    uint32_t kind, n, arg;  // LIT: arg = the byte; RING: arg = distance to read from; LOADED: v holds the bytes
    uint32_t v[4];
};

// The lane's next copy, at output position q = its ring position + pend_n (the pending copy).
template <class C>
__device__ __forceinline__ void ln_next(Lane& L, uint32_t q, uint32_t pend_n, const uint16_t* lit,
                                        const uint16_t* lsym, const uint16_t* dist, const uint16_t* dsym,
                                        const uint32_t (&llim)[C::NLL], const uint32_t (&dlim)[C::NLD],
                                        const uint32_t* ringw, const typename C::CtaSmem& S, Op& op) {
    op.kind = OP_NONE;
    op.n = 0;
    if (L.rem == 0) {
        if (L.stored) {
            L.stored = false;
            L.bitpos = L.spos * 8;
            L.st = L.final_block ? ln::FIN : ln::HEADER;
            return;
        }
        ln_refill(L);
        uint32_t e = lit[(uint32_t)L.bb & ((1u << C::LNB) - 1)];
        if (e == E16_SLOW) e = long_code(L.bb, llim, lsym, 288);
        const uint32_t cl = e >> 12, kind = (e >> 10) & 3u, v = e & 1023u;
        L.bb >>= cl;
        L.bc -= (int)cl;
        if (kind == 0u) {
            if (q >= L.isize) {
                L.err = CB_ERR_INFLATE;
                L.st = ln::FIN;
                return;
            }
            op.kind = OP_LIT;
            op.n = 1;
            op.arg = v;
            return;
        }
        if (kind != 1u) {
            if (kind == 2u) {
                L.bitpos = ln_bitpos(L);
                L.st = L.final_block ? ln::FIN : ln::HEADER;
            } else {
                L.err = CB_ERR_INFLATE;
                L.st = ln::FIN;
            }
            return;
        }
        const uint32_t li = S.li[v], ext = li >> 16;
        const uint32_t len = (li & 0xFFFFu) + ((uint32_t)L.bb & ((1u << ext) - 1u));
        L.bb >>= ext;
        L.bc -= (int)ext;
        ln_refill(L);
        uint32_t d = dist[(uint32_t)L.bb & ((1u << C::LDB) - 1)];
        if (d == E16_SLOW) d = long_code(L.bb, dlim, dsym, 32);
        const uint32_t dl = d >> 12;
        const uint32_t di = S.di[d & 31u], dext = di >> 16;
        const uint32_t dv = (di & 0xFFFFu) + ((uint32_t)(L.bb >> dl) & ((1u << dext) - 1u));
        L.bb >>= dl + dext;
        L.bc -= (int)(dl + dext);
        if ((d & 0x0C00u) != 0x0400u || dv > q || q + len > L.isize) {
            L.err = CB_ERR_INFLATE;
            L.st = ln::FIN;
            return;
        }
        L.rem = len;
        L.dist = dv;
    }
    const uint32_t n = min(min(L.rem, 16u), L.dist);
    op.n = n;
    if (L.stored) {
        op.kind = OP_LOADED;
        gather16<true>(L.in + L.spos, L.in + L.in_len + 8, op.v);
        L.spos += n;
    } else if (L.dist <= C::RV) {
        // bytes [q - dist, q - dist + n) lie below the pending copy's output (which starts at
        // q - pend_n) unless the distance is short: then they are read when the copy is carried out
        if (L.dist >= pend_n + n) {
            op.kind = OP_LOADED;
            ring_load16<C::LRING / 4>(ringw, (q - L.dist + L.a) & (C::LRING - 1), op.v);
        } else {
            op.kind = OP_RING;
            op.arg = L.dist;
        }
        if (L.dist < 16) L.dist <<= 1;
    } else {
        op.kind = OP_LOADED;
        gather16<false>(L.out + (q - L.dist), L.out + L.flushed, op.v);
    }
    L.rem -= n;
}

// Carry out a copy at the lane's ring position.
template <class C>
__device__ __forceinline__ void ln_exec(Lane& L, const Op& op, uint32_t* ringw) {
    constexpr uint32_t RW = C::LRING / 4, RM = C::LRING - 1;
    if (op.kind == OP_LIT) {
        reinterpret_cast<uint8_t*>(ringw)[(L.p + L.a) & RM] = (uint8_t)op.arg;
    } else if (op.kind == OP_RING) {
        uint32_t v[4];
        ring_load16<RW>(ringw, (L.p - op.arg + L.a) & RM, v);
        ring_store16<RW>(ringw, (L.p + L.a) & RM, v);
    } else if (op.kind == OP_LOADED) {
        ring_store16<RW>(ringw, (L.p + L.a) & RM, op.v);
    }
    L.p += op.n;
}

// Store the lane's complete 16-byte units (all its bytes when all) and fold them into its CRC.
template <class C>
__device__ __forceinline__ void ln_flush(Lane& L, const uint32_t* ringw, const typename C::CtaSmem& S, bool crc,
                                         bool all) {
    constexpr uint32_t RM = C::LRING - 1;
    const uint8_t* ring = reinterpret_cast<const uint8_t*>(ringw);
    if (L.flushed == 0 && L.a != 0 && L.p >= 16 - L.a) {
        for (uint32_t x = 0; x < 16 - L.a; x++) {
            const uint32_t b = ring[(x + L.a) & RM];
            L.out[x] = (uint8_t)b;
            if (crc) L.crc = S.crc8[0][(L.crc ^ b) & 255] ^ (L.crc >> 8);
        }
        L.flushed = 16 - L.a;
    }
    const uint32_t lim = (L.p + L.a >= 16) ? ((L.p + L.a) & ~15u) - L.a : 0u;
    while (L.flushed + 16 <= lim) {
        const uint4 u = *reinterpret_cast<const uint4*>(ring + ((L.flushed + L.a) & RM));
        *reinterpret_cast<uint4*>(L.out + L.flushed) = u;
        if (crc) {
            L.crc = crc_step8(S.crc8, L.crc, u.x, u.y);
            L.crc = crc_step8(S.crc8, L.crc, u.z, u.w);
        }
        L.flushed += 16;
    }
    if (all) {
        for (uint32_t x = L.flushed; x < L.p; x++) {
            const uint32_t b = ring[(x + L.a) & RM];
            L.out[x] = (uint8_t)b;
            if (crc) L.crc = S.crc8[0][(L.crc ^ b) & 255] ^ (L.crc >> 8);
        }
        L.flushed = L.p;
    }
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

__device__ __forceinline__ void report(cb_inflate_summary* summary, uint32_t* job_status, long long j, uint32_t st) {
    if (job_status) job_status[j] = st;
    if (st != CB_OK) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&summary->n_bad), 1ull);
        atomicMin(reinterpret_cast<long long*>(&summary->first_bad), j);
        atomicMax(&summary->status, (int)st);
    }
}


__global__ void __launch_bounds__(wm::WARPS * 32, 4)
    k_inflate_warp(const cb_member_job* __restrict__ jobs, int64_t n_jobs, const int64_t* __restrict__ d_n_jobs,
                   uint8_t* out_base, int check_crc, uint32_t* job_status, cb_inflate_summary* summary,
                   unsigned long long* queue) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    wm::CtaSmem& S = *reinterpret_cast<wm::CtaSmem*>(smem_raw);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
#pragma unroll
        for (int b = 0; b < 4; b++) S.mulk[b][i] = gf_mul((uint32_t)i << (8 * b), kCrc.k992);
    }
    init_crc8(S.crc8);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    wm::WarpSmem& W = S.w[warp];
    int64_t n = n_jobs;
    if (d_n_jobs) n = min(n, *d_n_jobs);
    const bool crc = check_crc != 0;
    for (;;) {
        unsigned long long j = 0;
        if (lane == 0) j = atomicAdd(queue, 1ull);
        j = __shfl_sync(FULL, j, 0);
        if ((int64_t)j >= n) break;
        const cb_member_job job = jobs[j];
        const uint32_t st = inflate_member(job, out_base, crc, W, S);
        __syncwarp();
        if (lane == 0) report(summary, job_status, (long long)j, st);
    }
}

template <class C>
__global__ void __launch_bounds__(C::WARPS * 32, 1)
    k_inflate_lanes(const cb_member_job* __restrict__ jobs, int64_t n_jobs, const int64_t* __restrict__ d_n_jobs,
                    uint8_t* out_base, int check_crc, uint32_t* job_status, cb_inflate_summary* summary,
                    unsigned long long* queue) {
    using CtaSmem = typename C::CtaSmem;
    using WarpSmem = typename C::WarpSmem;
    extern __shared__ __align__(16) uint8_t smem_raw[];
    CtaSmem& S = *reinterpret_cast<CtaSmem*>(smem_raw);
    if (threadIdx.x < 32) {
        const int s = threadIdx.x;
        S.li[s] = s < 29 ? (uint32_t)kLenBase[s] | ((uint32_t)kLenExtra[s] << 16) : 0u;
        S.di[s] = s < 30 ? (uint32_t)kDistBase[s] | ((uint32_t)kDistExtra[s] << 16) : 0u;
    }
    init_crc8(S.crc8);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpSmem& W = S.w[warp];
    int64_t n = n_jobs;
    if (d_n_jobs) n = min(n, *d_n_jobs);
    const bool crc = check_crc != 0;
    const int ml = lane < C::MLANES ? lane : 0;  // lanes from MLANES on never take a member
    const uint16_t* my_lit = W.lit + ml * C::LSTRIDE;
    const uint16_t* my_lsym = W.lsym + ml * C::LSYM;
    const uint16_t* my_dist = W.dist + ml * C::DSTRIDE;
    const uint16_t* my_dsym = W.dsym + ml * C::DSYM;
    uint32_t* my_ring = reinterpret_cast<uint32_t*>(W.ring + ml * C::RSTRIDE);
    uint32_t llim[C::NLL], dlim[C::NLD];
#pragma unroll
    for (int i = 0; i < C::NLL; i++) llim[i] = 0;
#pragma unroll
    for (int i = 0; i < C::NLD; i++) dlim[i] = 0;

    Lane L;
    L.st = lane < C::MLANES ? ln::IDLE : ln::DONE;
    Op pend;
    pend.kind = OP_NONE;
    pend.n = 0;
    for (;;) {
        // members that ended: the rest of their output, the checks, the status
        if (L.st == ln::FIN) {
            uint32_t status = L.err;
            if (status == CB_OK && (L.p != L.isize || L.bitpos > L.in_len * 8u)) status = CB_ERR_INFLATE;
            if (status == CB_OK) {
                ln_flush<C>(L, my_ring, S, crc, true);
                if (crc && ~L.crc != L.want_crc) status = CB_ERR_CRC;
            }
            report(summary, job_status, L.j, status);
            L.st = ln::IDLE;
        }
        // idle lanes take the next members
        const unsigned idle = __ballot_sync(FULL, L.st == ln::IDLE);
        if (idle) {
            const int leader = __ffs(idle) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(queue, (unsigned long long)__popc(idle));
            base = __shfl_sync(FULL, base, leader);
            if (L.st == ln::IDLE) {
                const long long j = (long long)base + __popc(idle & ((1u << lane) - 1u));
                if (j >= n) {
                    L.st = ln::DONE;
                } else {
                    const cb_member_job job = jobs[j];
                    L.j = j;
                    L.in = job.in;
                    L.wbase = reinterpret_cast<const uint32_t*>((uintptr_t)job.in & ~(uintptr_t)3);
                    L.s0 = (uint32_t)((uintptr_t)job.in & 3) * 8;
                    L.nvalid = (uint32_t)(((uintptr_t)job.in + job.in_len + 8 - (uintptr_t)L.wbase) >> 2);
                    L.in_len = job.in_len;
                    L.out = out_base + job.out_off;
                    L.a = (uint32_t)((uintptr_t)L.out & 15);
                    L.isize = job.isize;
                    L.want_crc = job.crc;
                    L.p = 0;
                    L.flushed = 0;
                    L.crc = 0xFFFFFFFFu;
                    L.rem = 0;
                    L.dist = 16;
                    L.spos = 0;
                    L.stored = false;
                    L.final_block = false;
                    L.err = CB_OK;
                    L.bitpos = 0;
                    L.st = ln::HEADER;
                }
            }
        }
        if (__all_sync(FULL, L.st == ln::DONE)) break;
        // block headers, one lane at a time by the whole warp
        for (unsigned h = __ballot_sync(FULL, L.st == ln::HEADER); h; h = __ballot_sync(FULL, L.st == ln::HEADER)) {
            const int t = __ffs(h) - 1;
            Reader r;
            r.wbase = reinterpret_cast<const uint32_t*>(shfl_ll((long long)(uintptr_t)L.wbase, t));
            r.nvalid = __shfl_sync(FULL, L.nvalid, t);
            r.s0 = __shfl_sync(FULL, L.s0, t);
            const uint32_t pos = __shfl_sync(FULL, L.bitpos, t);
            const uint32_t in_len = __shfl_sync(FULL, L.in_len, t);
            const uint32_t room = __shfl_sync(FULL, L.isize - L.p, t);
            uint32_t st = CB_OK, final_block = 0, btype = 0, len = 0, spos = 0, next = 0;
            if (pos > in_len * 8u) {
                st = CB_ERR_INFLATE;
            } else {
                seek(r, pos);
                if (r.bc < 32) refill(r);
                const uint32_t hdr = (uint32_t)r.bb & 7u;
                consume(r, 3);
                final_block = hdr & 1u;
                btype = hdr >> 1;
                if (btype == 0) {
                    const uint32_t bp = ((uint32_t)consumed(r) + 7) & ~7u;
                    seek(r, bp);
                    if (r.bc < 32) refill(r);
                    len = (uint32_t)r.bb & 0xFFFFu;
                    const uint32_t nlen = ((uint32_t)r.bb >> 16) & 0xFFFFu;
                    spos = bp / 8 + 4;
                    if (len != (~nlen & 0xFFFFu) || spos + len > in_len || len > room) st = CB_ERR_INFLATE;
                    next = (spos + len) * 8;
                } else if (btype == 3) {
                    st = CB_ERR_INFLATE;
                } else {
                    st = read_lane_tables<C>(r, W, btype, t);
                    next = (uint32_t)consumed(r);
                }
            }
            __syncwarp();
            if (lane == t) {
                if (st != CB_OK) {
                    L.err = st;
                    L.st = ln::FIN;
                } else {
                    L.final_block = final_block != 0;
                    if (btype == 0) {
                        L.bitpos = next;
                        if (len == 0) {
                            L.st = L.final_block ? ln::FIN : ln::HEADER;
                        } else {
                            L.stored = true;
                            L.rem = len;
                            L.dist = 16;
                            L.spos = spos;
                            L.st = ln::RUN;
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < C::NLL; i++) llim[i] = W.lim[i];
#pragma unroll
                        for (int i = 0; i < C::NLD; i++) dlim[i] = W.lim[C::NLL + i];
                        ln_seek(L, next);
                        L.rem = 0;
                        L.st = ln::RUN;
                    }
                }
            }
            __syncwarp();
        }
        // decode steps: each makes the lane's next copy and carries out the one before
#pragma unroll 1
        for (int k = 0; k < C::STEPS; k++) {
            if (L.st == ln::RUN && L.p - L.flushed <= C::PAUSE) {
                Op cur;
                ln_next<C>(L, L.p + pend.n, pend.n, my_lit, my_lsym, my_dist, my_dsym, llim, dlim, my_ring, S, cur);
                ln_exec<C>(L, pend, my_ring);
                pend = cur;
            }
        }
        if (L.st == ln::RUN || L.st == ln::HEADER) ln_flush<C>(L, my_ring, S, crc, false);
    }
}

}  // namespace infl
}  // namespace cb

using namespace cb;

int cb_set_error(cudaError_t e);  // abi.cu

namespace {

using Form2 = infl::ln::Form2;
constexpr int MAX_DEVICES = 64;
int g_bps[2][MAX_DEVICES];  // CTAs per SM of each form, per device (0: not yet known)

int cur_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= MAX_DEVICES) return -1;
    return d;
}

// CTAs per SM of a form's kernel on the current device, setting its shared memory size once.
int blocks_per_sm(int form) {
    const int d = cur_device();
    if (d < 0) return -1;
    int& b = g_bps[form - 1][d];
    if (b > 0) return b;
    cudaError_t e;
    int occ = 0;
    if (form == 1) {
        const size_t smem = sizeof(infl::wm::CtaSmem);
        e = cudaFuncSetAttribute(infl::k_inflate_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, infl::k_inflate_warp, infl::wm::WARPS * 32, smem);
    } else {
        const size_t smem = sizeof(Form2::CtaSmem);
        e = cudaFuncSetAttribute(infl::k_inflate_lanes<Form2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, infl::k_inflate_lanes<Form2>, Form2::WARPS * 32,
                                                               smem);
    }
    if (e != cudaSuccess) return -(int)e;
    b = occ > 0 ? occ : 1;
    return b;
}

}  // namespace

extern "C" size_t cb_inflate_workspace_bytes(void) { return 256; }

extern "C" int64_t cb_inflate_lane_slots(void) {
    const int b = blocks_per_sm(2);
    if (b <= 0) {
        cb_set_error(b == -1 ? cudaErrorInvalidDevice : (cudaError_t)(-b));
        return 0;
    }
    return (int64_t)cb_device_sm_count() * b * Form2::WARPS * Form2::MLANES;
}

extern "C" int cb_inflate_form(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint8_t* out_base,
                               int check_crc, uint32_t* job_status, cb_inflate_summary* summary, void* workspace,
                               size_t workspace_bytes, int form, void* stream) {
    if (!summary || !workspace || workspace_bytes < cb_inflate_workspace_bytes() || n_jobs < 0) return CB_ERR_ARG;
    if (form == 0) {
        form = (int)cb_param(CB_PARAM_INFLATE_FORM);
        if (form == 3 && n_jobs < cb_param(CB_PARAM_SPLIT_MIN_JOBS)) form = 1;
    }
    if (form == 3) {
        // the split form needs its token arena: a workspace of the forms-1/2 size runs form 1 instead
        if (workspace_bytes > cb_inflate_workspace_bytes())
            return cb_inflate_split(jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, workspace,
                                    workspace_bytes, stream);
        form = 1;
    }
    if (form != 1 && form != 2) return CB_ERR_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    auto* queue = reinterpret_cast<unsigned long long*>(workspace);
    const int bps = blocks_per_sm(form);
    if (bps <= 0) return cb_set_error(bps == -1 ? cudaErrorInvalidDevice : (cudaError_t)(-bps));
    infl::k_inflate_init<<<1, 1, 0, s>>>(summary, queue);
    if (n_jobs > 0) {
        const int per_cta = form == 1 ? infl::wm::WARPS : Form2::WARPS * Form2::MLANES;
        long long grid = (long long)cb_device_sm_count() * bps;
        const long long by_work = (n_jobs + per_cta - 1) / per_cta;
        if (!d_n_jobs && by_work < grid) grid = by_work;
        if (grid < 1) grid = 1;
        if (form == 1)
            infl::k_inflate_warp<<<(unsigned)grid, infl::wm::WARPS * 32, sizeof(infl::wm::CtaSmem), s>>>(
                jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, queue);
        else
            infl::k_inflate_lanes<Form2><<<(unsigned)grid, Form2::WARPS * 32, sizeof(Form2::CtaSmem), s>>>(
                jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, queue);
    }
    infl::k_inflate_finish<<<1, 1, 0, s>>>(summary);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_inflate(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint8_t* out_base,
                          int check_crc, uint32_t* job_status, cb_inflate_summary* summary, void* workspace,
                          size_t workspace_bytes, void* stream) {
    return cb_inflate_form(jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, workspace,
                           workspace_bytes, 0, stream);
}
