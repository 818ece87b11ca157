// BGZF writer on B200 (sm_100a): raw-DEFLATE compression of spans, their CRC32, BGZF framing.
//
// Replaces cubam's nvCOMP Deflate compression call (src/cubam/bgzf.py:292-351), its CRC32 and
// Adler-32 span kernels (src/cubam/_kernels.py:93-158) and its framing kernel bgzf_frame
// (src/cubam/_kernels.py:161-191, called from src/cubam/bgzf.py:380-422).  DEFLATE is RFC 1951,
// the BGZF member layout SAMv1 section 4.1.
//
// k_deflate: a persistent grid, one CTA of 512 threads per span (at most 64 KiB) at a time, all of
// the span's work in shared memory:
//   1. the span is staged with 16-byte loads; its CRC32 is taken there (one column per thread in
//      8-byte steps, columns joined in a tree by shifts in GF(2)[x]);
//   2. match finding, 512 positions (one per thread) per tile: a hash of the 4 bytes at each
//      position; candidates are the nearest earlier position of the same hash in the warp
//      (__match_any_sync) and the latest one of earlier tiles (a table of hash heads kept with
//      atomicMax, so the result does not depend on thread timing); the longer match is kept;
//   3. the greedy parse of the tile without a serial walk: jmp[0][i] = i + the step at i (the
//      match length, or 1), jmp[k+1][i] = jmp[k][jmp[k][i]], and thread m finds token m of the tile
//      by advancing the entry position by the binary digits of m.  With level >= 2 a position
//      whose successor has a longer match is a literal (zlib's lazy evaluation, one position of
//      lookahead);
//   4. tokens go to a per-CTA buffer in HBM (it stays in L2), symbol counts to shared memory;
//   5. Huffman code lengths (ranking by counting, Moffat-Katajainen minimum-redundancy lengths,
//      limited to 15 and 7 bits), the code-length code, and the exact sizes of a dynamic, a fixed
//      and a stored block; the smallest is written;
//   6. bits go out at offsets from a block-wide prefix sum of token sizes (atomicOr into shared
//      memory words) and are copied to the span's slot.
// k_offsets (one CTA) sums the stream sizes into output offsets; k_pack copies each slot to its
// offset, with the BGZF header and trailer when framing.
//
// Every loop is bounded by the span's size or an alphabet; no thread waits on another CTA.

#include "common.cuh"
#include "crc.cuh"
#include "deflate_codes.cuh"

namespace cb {
namespace dfl {

constexpr int NT = 512;                        // threads per CTA = positions per tile
constexpr int MAXSPAN = 65536;                 // largest raw span
constexpr int BGZF_SPAN = 0xFF00;              // largest span framed as a BGZF member (BLOCK_DATA)
constexpr int INB = MAXSPAN + 32;              // staged bytes: the span at offset a < 16, then slack
constexpr int HB = 13, NH = 1 << HB;           // hash-head table
constexpr int LEVELS = 9;                      // jump levels: up to 2^9 tokens per tile
constexpr uint32_t MIN_MATCH = 4, MAX_MATCH = 258, WSIZE = 32768;
constexpr int64_t SLOT = MAXSPAN + 64;         // bytes per span slot (a stream is at most 65536 + 10)
constexpr int MAX_CTAS = 320;                  // token buffers in the workspace
constexpr int64_t TOKS = MAXSPAN;              // tokens per CTA buffer
constexpr int META = 4;                        // per span: stream bytes, CRC32, kind, input bytes
enum : uint32_t { K_STORED = 0, K_FIXED = 1, K_DYNAMIC = 2 };
static_assert((1 << LEVELS) == NT, "token m of a tile has LEVELS binary digits");

// Code-length construction of one alphabet (par_lengths).
struct LenScratch {
    uint16_t sorted[NLIT_ALL];   // used symbols by ascending (count, symbol)
    uint32_t A[NLIT_ALL];        // weights, then internal node weights and parent links
    uint16_t anc[2][NLIT_ALL];   // pointer jumping over internal nodes: ancestor, depth to it
    uint16_t dep[2][NLIT_ALL];
    uint32_t c[NLIT_ALL + 2];    // internal nodes per depth
    uint32_t cum[16];            // codes of length <= l
    int32_t maxd;
};

struct HuffScratch {
    LenScratch ls;
    uint8_t rsym[NRLE];
    uint8_t rext[NRLE];
    uint32_t roff[NRLE];  // bit offset of each code-length symbol within the run-length part
    uint32_t lcode[NLIT_ALL];
    uint32_t dcode[32];
    uint32_t clcode[20];
};

struct Smem {
    uint32_t in[INB / 4];       // the span's bytes; after tokenising, the output bit buffer
    uint32_t head[NH];          // position + 1 of the latest earlier-tile position of each hash (0 = none)
    union {
        uint16_t jmp[LEVELS][NT];  // jmp[k][i]: tile position after 2^k tokens from i (>= NT: beyond)
        uint32_t crc8[8][256];     // slice-by-8 tables, while the CRC is taken
        HuffScratch h;             // code construction, after the last tile
    } u;
    uint32_t mt[NT];            // match at each tile position: length << 16 | distance (0: none)
    uint32_t lfreq[NLIT_ALL], dfreq[32], clfreq[20];
    uint8_t llen[NLIT_ALL], dlen[32], cllen[20];
    uint32_t scan[33];
    uint32_t cnt[3][16], nxt[3][16];  // codes per length and first code per length: literal, distance, code-length
    uint32_t crcw[16], crck[LEVELS];
    int32_t ntok, exitp, nrle, hlit, hdist, hclen, kind, pad_;
    uint32_t hdr_bits, bits;
};

__device__ __forceinline__ uint32_t u32at(const uint32_t* w, uint32_t byte) {
    const uint32_t i = byte >> 2;
    return __funnelshift_r(w[i], w[i + 1], (byte & 3) * 8);
}

// 8 bytes at byte offset `byte` of the staged span (three aligned words).
__device__ __forceinline__ uint64_t u64at(const uint32_t* w, uint32_t byte) {
    const uint32_t i = byte >> 2, sh = (byte & 3) * 8;
    const uint32_t w0 = w[i], w1 = w[i + 1], w2 = w[i + 2];
    return (uint64_t)__funnelshift_r(w0, w1, sh) | ((uint64_t)__funnelshift_r(w1, w2, sh) << 32);
}

// Bytes in common at byte offsets q and c (c < q) of the staged span, at most maxl, 8 bytes per
// step.  Reads at most 11 bytes past q + maxl (inside the staging slack).
__device__ __forceinline__ uint32_t match_len(const uint32_t* w, uint32_t q, uint32_t c, uint32_t maxl) {
    uint32_t L = 0;
    while (L < maxl) {
        const uint64_t x = u64at(w, q + L) ^ u64at(w, c + L);
        if (x) {
            L += (uint32_t)(__ffsll((long long)x) - 1) >> 3;
            break;
        }
        L += 8;
    }
    return L < maxl ? L : maxl;
}

// OR the low nb (<= 32) bits of v into the bit stream at bit pos (a stream is shorter than the
// staging buffer by construction: a block longer than the stored one is never emitted; the bound
// keeps every write inside it regardless).
__device__ __forceinline__ void or_bits(uint32_t* buf, uint32_t pos, uint32_t v, uint32_t nb) {
    const uint32_t w = pos >> 5, s = pos & 31;
    if (nb == 0 || w + 1 >= (uint32_t)(INB / 4)) return;
    const uint64_t x = (uint64_t)v << s;
    atomicOr(&buf[w], (uint32_t)x);
    if (s + nb > 32) atomicOr(&buf[w + 1], (uint32_t)(x >> 32));
}

// Rank of symbol s among the symbols with nonzero counts, by (count, symbol): sorted[rank] = s.
__device__ __forceinline__ void rank_symbol(const uint32_t* freq, int nsym, int s, uint16_t* sorted) {
    const uint32_t f = freq[s];
    if (!f) return;
    int r = 0;
    for (int j = 0; j < nsym; j++) {
        const uint32_t g = freq[j];
        r += (g != 0) & ((g < f) | ((g == f) & (j < s)));
    }
    sorted[r] = (uint16_t)s;
}

// Per-size constants of span_crc, kept by thread 0 from one span to the next (spans mostly have
// the same size).
struct CrcCache {
    uint32_t seg = 0xFFFFFFFFu, n = 0xFFFFFFFFu, fin = 0;
};

// The zlib CRC32 of the staged span (bytes a .. a + n of S.in), every thread taking part; the
// result is valid in thread 0.
__device__ uint32_t span_crc(Smem& S, uint32_t a, uint32_t n, CrcCache& cc) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint8_t* in8 = reinterpret_cast<const uint8_t*>(S.in);
    init_crc8(S.u.crc8);
    // thread t: bytes [t*seg - pad, (t+1)*seg - pad) of the span behind pad zero bytes (zeros in
    // front leave a raw column unchanged), so all columns are seg bytes long
    const uint32_t seg = ((n + NT - 1) / NT + 7) & ~7u;
    const int32_t pad = (int32_t)(NT * seg) - (int32_t)n;
    if (t == 0 && seg != cc.seg) {
        cc.seg = seg;
        uint32_t c = xpow_from(kCrc.x2n, 8ull * seg);
        for (int k = 0; k < LEVELS; k++) {
            S.crck[k] = c;
            c = gf_mul(c, c);
        }
    }
    __syncthreads();
    uint32_t col = 0;
    const int32_t r1 = (int32_t)(t * seg) + (int32_t)seg - pad;
    if (r1 > 0) {
        int32_t r = (int32_t)(t * seg) - pad;
        if (r < 0) r = 0;
        for (; (r1 - r) & 7; r++) col = S.u.crc8[0][(col ^ in8[a + r]) & 255] ^ (col >> 8);
        for (; r < r1; r += 8) col = crc_step8(S.u.crc8, col, u32at(S.in, a + r), u32at(S.in, a + r + 4));
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const uint32_t other = __shfl_down_sync(FULL, col, 1 << k);
        if ((lane & ((2 << k) - 1)) == 0) col = gf_mul(col, S.crck[k]) ^ other;
    }
    if (lane == 0) S.crcw[warp] = col;
    __syncthreads();
    uint32_t crc = 0;
    if (warp == 0) {
        uint32_t v = lane < NT / 32 ? S.crcw[lane] : 0u;
#pragma unroll
        for (int k = 5; k < LEVELS; k++) {
            const uint32_t other = __shfl_down_sync(FULL, v, 1 << (k - 5));
            if ((lane & ((2 << (k - 5)) - 1)) == 0) v = gf_mul(v, S.crck[k]) ^ other;
        }
        if (t == 0) {
            if (n != cc.n) {
                cc.n = n;
                cc.fin = gf_mul(0xFFFFFFFFu, xpow_from(kCrc.x2n, 8ull * n));
            }
            crc = v ^ cc.fin ^ 0xFFFFFFFFu;  // crc_finish(v, n)
        }
    }
    return crc;
}

// Tokens of the span into tok[0..), symbol counts into S.lfreq / S.dfreq.  Returns the token count.
__device__ uint32_t tokenize(Smem& S, uint32_t a, uint32_t n, int level, uint32_t* __restrict__ tok) {
    const int t = threadIdx.x, lane = t & 31;
    const uint8_t* in8 = reinterpret_cast<const uint8_t*>(S.in);
    uint32_t entry = 0, tbase = 0;
    for (uint32_t T0 = 0; T0 < n; T0 += NT) {
        const uint32_t tend = min((uint32_t)NT, n - T0);
        const uint32_t p = T0 + t;
        const bool v4 = level > 0 && p + 4 <= n;
        const uint32_t cur = v4 ? u32at(S.in, a + p) : 0u;
        const uint32_t h = (cur * 0x9E3779B1u) >> (32 - HB);
        const unsigned grp = __match_any_sync(FULL, v4 ? h : (0x80000000u | (uint32_t)t));
        const uint32_t hv = v4 ? S.head[h] : 0u;
        __syncthreads();  // every read of the heads before this tile's updates
        if (t == 0) S.ntok = 0;
        if (v4 && (grp >> lane) == 1u) atomicMax(&S.head[h], p + 1);
        uint32_t best = 0;
        if (v4) {
            const uint32_t maxl = min(MAX_MATCH, n - p);
            const unsigned below = grp & ((1u << lane) - 1u);
            if (below) {
                const uint32_t c = p - (uint32_t)lane + (31u - (uint32_t)__clz(below));
                const uint32_t L = match_len(S.in, a + p, a + c, maxl);
                if (L >= MIN_MATCH) best = (L << 16) | (p - c);
            }
            if (hv && (best >> 16) < maxl) {  // a match of maxl cannot be beaten
                const uint32_t c = hv - 1;
                if (p - c <= WSIZE) {
                    const uint32_t L = match_len(S.in, a + p, a + c, maxl);
                    if (L >= MIN_MATCH && L > (best >> 16)) best = (L << 16) | (p - c);
                }
            }
        }
        S.mt[t] = best;
        __syncthreads();
        uint32_t step = 1;
        if ((uint32_t)t < tend) {
            const uint32_t m0 = S.mt[t];
            if (m0) {
                step = m0 >> 16;
                if (level >= 2 && (uint32_t)t + 1 < tend && (S.mt[t + 1] >> 16) > step) step = 1;
            }
        }
        S.u.jmp[0][t] = (uint16_t)((uint32_t)t < tend ? t + step : NT);
        __syncthreads();
#pragma unroll 1
        for (int k = 0; k + 1 < LEVELS; k++) {
            const uint32_t x = S.u.jmp[k][t];
            S.u.jmp[k + 1][t] = x < (uint32_t)NT ? S.u.jmp[k][x] : (uint16_t)x;
            __syncthreads();
        }
        uint32_t pos = entry;
#pragma unroll
        for (int k = 0; k < LEVELS; k++)
            if (((t >> k) & 1) && pos < (uint32_t)NT) pos = S.u.jmp[k][pos];
        if (pos < tend) {
            const uint32_t nx = S.u.jmp[0][pos], st = nx - pos;
            uint32_t tk;
            if (st >= MIN_MATCH) {
                const uint32_t d = S.mt[pos] & 0xFFFFu;
                tk = 0x80000000u | (st << 16) | (d - 1);
                atomicAdd(&S.lfreq[len_sym(st)], 1u);
                atomicAdd(&S.dfreq[dist_sym(d)], 1u);
            } else {
                tk = in8[a + T0 + pos];
                atomicAdd(&S.lfreq[tk], 1u);
            }
            tok[tbase + t] = tk;
            if (nx >= tend) {
                S.ntok = t + 1;
                S.exitp = (int32_t)nx - NT;
            }
        }
        __syncthreads();
        tbase += (uint32_t)S.ntok;
        entry = S.exitp > 0 ? (uint32_t)S.exitp : 0u;
    }
    return tbase;
}

// Code lengths (at most L bits) of the symbols 0..nrank-1 with counts freq, into len[0..nlen), as
// build_lengths gives them; every thread takes part.  Thread 0 runs the first, sequential pass of
// the Moffat-Katajainen method (the merge of leaves and internal nodes); the depths of internal
// nodes come from pointer jumping over its parent links, the leaves per depth from a histogram of
// those depths, and each symbol's length from its rank (lengths_from_depths, length_of_rank).
__device__ void par_lengths(Smem& S, const uint32_t* freq, int nrank, int nlen, uint32_t L, uint8_t* len) {
    const int t = threadIdx.x;
    LenScratch& P = S.u.h.ls;
    if (t < nrank) rank_symbol(freq, nrank, t, P.sorted);
    const int m = __syncthreads_count(t < nrank && freq[t] != 0);
    if (t < nlen) len[t] = 0;
    if (t < m) P.A[t] = freq[P.sorted[t]];
    for (int i = t; i < m + 2; i += NT) P.c[i] = 0u;
    if (t == 0) P.maxd = 0;
    __syncthreads();
    if (m < 2) {  // a complete two-code all the same, as decoders want
        if (t == 0) {
            if (m == 0) {
                len[0] = len[1] = 1;
            } else {
                len[P.sorted[0]] = 1;
                len[P.sorted[0] == 0 ? 1 : 0] = 1;
            }
        }
        __syncthreads();
        return;
    }
    if (t == 0) mk_pass1(P.A, m);
    __syncthreads();
    const int ni = m - 1, root = m - 2;  // internal nodes; the last one is the root
    if (t < ni) {
        P.anc[0][t] = (uint16_t)(t == root ? t : P.A[t]);
        P.dep[0][t] = (uint16_t)(t == root ? 0 : 1);
    }
    __syncthreads();
    int cur = 0;
    for (int r = 0; r < LEVELS; r++) {  // depths below 2^LEVELS = 512 > NLIT_ALL
        bool more = false;
        if (t < ni) {
            const uint32_t a = P.anc[cur][t];
            P.dep[cur ^ 1][t] = (uint16_t)(P.dep[cur][t] + P.dep[cur][a]);
            const uint32_t aa = P.anc[cur][a];
            P.anc[cur ^ 1][t] = (uint16_t)aa;
            more = aa != (uint32_t)root;
        }
        cur ^= 1;
        if (!__syncthreads_or(more)) break;
    }
    if (t < ni) {
        atomicAdd(&P.c[P.dep[cur][t]], 1u);
        atomicMax(&P.maxd, (int)P.dep[cur][t]);
    }
    __syncthreads();
    if (t == 0) lengths_from_depths(P.c, P.maxd, L, P.cum);
    __syncthreads();
    if (t < m) len[P.sorted[t]] = (uint8_t)length_of_rank((uint32_t)(m - 1 - t), P.cum);
    __syncthreads();
}

// First code of each length (RFC 1951 3.2.2) from the number of codes of each length.
__device__ __forceinline__ void first_codes(const uint32_t* cnt, uint32_t* nxt) {
    uint32_t c = 0;
    nxt[0] = 0;
    for (int l = 1; l <= 15; l++) {
        c = (c + (l > 1 ? cnt[l - 1] : 0u)) << 1;
        nxt[l] = c;
    }
}

// The canonical code of symbol s (as canonical_codes): the first code of its length plus the
// number of earlier symbols of that length; length << 16 | the code's bits reversed.
__device__ __forceinline__ uint32_t canonical_of(const uint8_t* len, int s, const uint32_t* nxt) {
    const uint32_t l = len[s];
    if (!l) return 0u;
    uint32_t r = 0;
    for (int j = 0; j < s; j++) r += len[j] == l;
    return (l << 16) | reverse_bits(nxt[l] + r, l);
}

// Code lengths, the block kind and its size, and the codes the emitter uses, every thread taking
// part (the same results as the serial build_lengths, rle_lengths and canonical_codes).
__device__ void build_codes(Smem& S, uint32_t n) {
    const int t = threadIdx.x;
    HuffScratch& H = S.u.h;
    par_lengths(S, S.lfreq, NLIT, NLIT_ALL, MAXBITS, S.llen);
    par_lengths(S, S.dfreq, NDIST, NDIST, MAXBITS, S.dlen);
    if (t == 0) {
        S.hlit = 257;
        S.hdist = 1;
    }
    if (t < 20) S.clfreq[t] = 0u;
    __syncthreads();
    if (t < NLIT && S.llen[t]) atomicMax(&S.hlit, t + 1);
    if (t < NDIST && S.dlen[t]) atomicMax(&S.hdist, t + 1);
    __syncthreads();
    // run-length coding of the code lengths: each run of equal lengths writes its symbols at the
    // prefix sum of the symbol counts of the runs before it
    const int hlit = S.hlit, T = hlit + S.hdist;
    int cnt = 0, run = 0;
    uint8_t v = 0;
    if (t < T) {
        v = t < hlit ? S.llen[t] : S.dlen[t - hlit];
        const uint8_t prev = t == 0 ? 0xFF : (t - 1 < hlit ? S.llen[t - 1] : S.dlen[t - 1 - hlit]);
        if (v != prev) {
            run = 1;
            while (t + run < T && (t + run < hlit ? S.llen[t + run] : S.dlen[t + run - hlit]) == v) run++;
            cnt = rle_run(v, run, nullptr, nullptr);
        }
    }
    uint32_t nrle;
    const uint32_t ro = block_exclusive_scan<NT>((uint32_t)cnt, nrle, S.scan);
    if (cnt) {
        rle_run(v, run, H.rsym + ro, H.rext + ro);
        for (int k = 0; k < cnt; k++) atomicAdd(&S.clfreq[H.rsym[ro + k]], 1u);
    }
    __syncthreads();
    par_lengths(S, S.clfreq, NCL, NCL, CLBITS, S.cllen);
    if (t == 0) {
        int hclen = NCL;
        while (hclen > 4 && S.cllen[cl_order(hclen - 1)] == 0) hclen--;
        S.hclen = hclen;
        S.nrle = (int32_t)nrle;
    }
    if (t < 48) S.cnt[t >> 4][t & 15] = 0u;
    __syncthreads();
    // bits of the dynamic payload, the fixed payload and the run-length part of the header
    uint32_t dyn = 0, fix = 0, hdr = 0;
    if (t < NLIT) {
        const uint32_t f = S.lfreq[t], e = t > 256 ? len_extra_bits(t) : 0;
        dyn = f * (S.llen[t] + e);
        fix = f * (fixed_lit_len(t) + e);
    } else if (t >= 320 && t < 320 + NDIST) {
        const uint32_t d = t - 320, f = S.dfreq[d], e = dist_extra_bits(d);
        dyn = f * (S.dlen[d] + e);
        fix = f * (FIXED_DIST_LEN + e);
    }
    if ((uint32_t)t < nrle) hdr = S.cllen[H.rsym[t]] + cl_extra_bits(H.rsym[t]);
    uint32_t dyn_t, fix_t, hdr_t;
    const uint32_t hoff = block_exclusive_scan<NT>(hdr, hdr_t, S.scan);
    block_exclusive_scan<NT>(dyn, dyn_t, S.scan);
    block_exclusive_scan<NT>(fix, fix_t, S.scan);
    if ((uint32_t)t < nrle) H.roff[t] = hoff;
    if (t == 0) {
        const uint64_t hdr_bits = 17 + 3 * (uint64_t)S.hclen + hdr_t;
        const uint64_t dbits = hdr_bits + dyn_t, fbits = 3 + (uint64_t)fix_t;
        const uint64_t nblk = n ? (n + 65534) / 65535 : 1;
        const uint64_t stored = n + 5 * nblk;
        uint32_t kind = (fbits + 7) / 8 <= (dbits + 7) / 8 ? K_FIXED : K_DYNAMIC;
        const uint64_t bits = kind == K_FIXED ? fbits : dbits;
        if (stored < (bits + 7) / 8) kind = K_STORED;
        S.kind = (int32_t)kind;
        S.bits = (uint32_t)(kind == K_STORED ? stored * 8 : bits);
        S.hdr_bits = kind == K_DYNAMIC ? (uint32_t)hdr_bits : 3u;
    }
    __syncthreads();
    const int kind = S.kind;
    if (kind == (int32_t)K_STORED) return;
    if (kind == (int32_t)K_FIXED) {
        if (t < NLIT_ALL) S.llen[t] = (uint8_t)fixed_lit_len(t);
        if (t < NDIST) S.dlen[t] = (uint8_t)FIXED_DIST_LEN;
        __syncthreads();
    }
    if (t < NLIT_ALL && S.llen[t]) atomicAdd(&S.cnt[0][S.llen[t]], 1u);
    if (t >= 320 && t < 320 + NDIST && S.dlen[t - 320]) atomicAdd(&S.cnt[1][S.dlen[t - 320]], 1u);
    if (t >= 384 && t < 384 + NCL && S.cllen[t - 384]) atomicAdd(&S.cnt[2][S.cllen[t - 384]], 1u);
    __syncthreads();
    if (t < 3) first_codes(S.cnt[t], S.nxt[t]);
    __syncthreads();
    if (t < NLIT_ALL) H.lcode[t] = canonical_of(S.llen, t, S.nxt[0]);
    else if (t >= 320 && t < 320 + NDIST) H.dcode[t - 320] = canonical_of(S.dlen, t - 320, S.nxt[1]);
    else if (t >= 384 && t < 384 + NCL) H.clcode[t - 384] = canonical_of(S.cllen, t - 384, S.nxt[2]);
    __syncthreads();
}

// The chosen block into S.in as a bit stream (not for stored blocks).
__device__ void emit(Smem& S, uint32_t ntok, const uint32_t* __restrict__ tok) {
    const int t = threadIdx.x;
    const HuffScratch& H = S.u.h;
    const uint32_t words = (S.bits + 31) / 32 + 1;
    for (uint32_t w = t; w < words && w < (uint32_t)(INB / 4); w += NT) S.in[w] = 0u;
    __syncthreads();
    if (S.kind == (int32_t)K_FIXED) {
        if (t == 0) or_bits(S.in, 0, 1u | (1u << 1), 3);
    } else {
        if (t == 0) {
            or_bits(S.in, 0, 1u | (2u << 1), 3);
            or_bits(S.in, 3, (uint32_t)(S.hlit - 257), 5);
            or_bits(S.in, 8, (uint32_t)(S.hdist - 1), 5);
            or_bits(S.in, 13, (uint32_t)(S.hclen - 4), 4);
        }
        if (t < S.hclen) or_bits(S.in, 17 + 3 * t, S.cllen[cl_order(t)], 3);
        if (t < S.nrle) {
            const uint32_t s = H.rsym[t], c = H.clcode[s], pos = 17 + 3 * S.hclen + H.roff[t];
            or_bits(S.in, pos, c & 0xFFFFu, c >> 16);
            or_bits(S.in, pos + (c >> 16), H.rext[t], cl_extra_bits(s));
        }
    }
    uint32_t base = S.hdr_bits;
    uint32_t next = (uint32_t)t < ntok ? tok[t] : 0u;  // each chunk's tokens are loaded a chunk ahead
    for (uint32_t c0 = 0; c0 < ntok; c0 += NT) {
        const uint32_t i = c0 + t;
        const uint32_t tk = next;
        next = i + NT < ntok ? tok[i + NT] : 0u;
        uint32_t v1 = 0, n1 = 0, v2 = 0, n2 = 0;
        if (i < ntok) {
            if (tk & 0x80000000u) {
                const uint32_t L = (tk >> 16) & 0x1FFu, d = (tk & 0xFFFFu) + 1;
                const uint32_t ls = len_sym(L), lc = H.lcode[ls], lb = lc >> 16;
                v1 = (lc & 0xFFFFu) | (len_extra_val(L) << lb);
                n1 = lb + len_extra_bits(ls);
                const uint32_t ds = dist_sym(d), dc = H.dcode[ds], db = dc >> 16;
                v2 = (dc & 0xFFFFu) | (dist_extra_val(d) << db);
                n2 = db + dist_extra_bits(ds);
            } else {
                const uint32_t lc = H.lcode[tk & 255u];
                v1 = lc & 0xFFFFu;
                n1 = lc >> 16;
            }
        }
        uint32_t total;
        const uint32_t off = base + block_exclusive_scan<NT>(n1 + n2, total, S.scan);
        if (i < ntok) {
            or_bits(S.in, off, v1, n1);
            or_bits(S.in, off + n1, v2, n2);
        }
        base += total;
    }
    if (t == 0) {
        const uint32_t e = H.lcode[256];
        or_bits(S.in, base, e & 0xFFFFu, e >> 16);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(NT, 2)
    k_deflate(const uint8_t* __restrict__ data, const int64_t* __restrict__ off, const int64_t* __restrict__ size,
              int64_t n_spans, int level, int max_span, uint32_t* __restrict__ tokens, uint8_t* __restrict__ slots,
              uint32_t* __restrict__ meta, cb_deflate_summary* __restrict__ summary) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    const int t = threadIdx.x;
    uint8_t* in8 = reinterpret_cast<uint8_t*>(S.in);
    uint32_t* tok = tokens + (int64_t)blockIdx.x * TOKS;
    CrcCache cc;
    for (int64_t sp = blockIdx.x; sp < n_spans; sp += gridDim.x) {
        const int64_t len = size[sp];
        if (len < 0 || len > max_span) {
            if (t == 0) {
                atomicMax(&summary->status, (int)CB_ERR_ARG);
                meta[META * sp] = 0;
                meta[META * sp + 1] = 0;
                meta[META * sp + 2] = K_STORED;
                meta[META * sp + 3] = 0;
            }
            continue;
        }
        const uint32_t n = (uint32_t)len;
        const uint8_t* src = data + off[sp];
        const uint32_t a = (uint32_t)(reinterpret_cast<uintptr_t>(src) & 15u);
        const uint4* g = reinterpret_cast<const uint4*>(src - a);
        const uint32_t nch = n ? (a + n + 15) / 16 : 0;  // 16-byte chunks holding the span (within its allocation)
        for (uint32_t c = t; c < nch; c += NT) reinterpret_cast<uint4*>(S.in)[c] = __ldg(g + c);
        __syncthreads();
        if (t < 8 && a + n + t < (uint32_t)INB) in8[a + n + t] = 0;
        const uint32_t crc = span_crc(S, a, n, cc);
        for (int i = t; i < NH; i += NT) S.head[i] = 0u;
        for (int i = t; i < NLIT_ALL; i += NT) S.lfreq[i] = 0u;
        if (t < 32) S.dfreq[t] = 0u;
        __syncthreads();
        const uint32_t ntok = tokenize(S, a, n, level, tok);
        if (t == 0) S.lfreq[256] = 1u;  // the end-of-block symbol
        __syncthreads();
        build_codes(S, n);
        uint8_t* slot = slots + sp * SLOT;
        uint32_t bytes;
        if (S.kind == (int32_t)K_STORED) {
            const uint32_t nblk = n ? (n + 65534) / 65535 : 1;
            if ((uint32_t)t < nblk) {
                const uint32_t b = t, l = min(65535u, n - b * 65535u);
                uint8_t* h = slot + b * 65540u;
                h[0] = b + 1 == nblk ? 1 : 0;
                h[1] = l & 255;
                h[2] = l >> 8;
                h[3] = ~l & 255;
                h[4] = (~l >> 8) & 255;
            }
            for (uint32_t i = t; i < n; i += NT) {
                const uint32_t b = i / 65535u;
                slot[b * 65540u + 5 + (i - b * 65535u)] = in8[a + i];
            }
            bytes = n + 5 * nblk;
        } else {
            emit(S, ntok, tok);
            bytes = (S.bits + 7) / 8;
            const uint32_t words = (bytes + 3) / 4;
            uint32_t* sw = reinterpret_cast<uint32_t*>(slot);
            for (uint32_t w = t; w < words; w += NT) sw[w] = S.in[w];
        }
        if (t == 0) {
            meta[META * sp] = bytes;
            meta[META * sp + 1] = crc;
            meta[META * sp + 2] = (uint32_t)S.kind;
            meta[META * sp + 3] = n;
        }
        __syncthreads();  // the next span overwrites shared memory
    }
}

// Output offsets: exclusive sum of the stream sizes (+ 26 bytes of BGZF header and trailer).
__global__ void __launch_bounds__(1024) k_offsets(const uint32_t* __restrict__ meta, int64_t n, int frame,
                                                  int64_t out_cap, int64_t* __restrict__ out_off,
                                                  int64_t* __restrict__ out_size, uint32_t* __restrict__ crc,
                                                  cb_deflate_summary* __restrict__ summary) {
    __shared__ long long sc[33];
    const int t = threadIdx.x;
    long long base = 0, stored = 0;
    for (int64_t c0 = 0; c0 < n; c0 += 1024) {
        const int64_t i = c0 + t;
        long long sz = 0;
        if (i < n) {
            sz = (long long)meta[META * i] + (frame ? 26 : 0);
            stored += meta[META * i + 2] == K_STORED;
        }
        long long total;
        const long long o = base + block_exclusive_scan<1024>(sz, total, sc);
        if (i < n) {
            out_off[i] = o;
            if (out_size) out_size[i] = sz;
            if (crc) crc[i] = meta[META * i + 1];
        }
        base += total;
    }
    if (stored) atomicAdd(reinterpret_cast<unsigned long long*>(&summary->n_stored), (unsigned long long)stored);
    if (t == 0) {
        summary->total = base;
        if (base > out_cap) atomicMax(&summary->status, (int)CB_ERR_CAPACITY);
    }
}

// Streams from their slots to their offsets, framed as BGZF members when frame != 0.
__global__ void __launch_bounds__(256) k_pack(const uint8_t* __restrict__ slots, const uint32_t* __restrict__ meta,
                                              int64_t n, int frame, const int64_t* __restrict__ out_off,
                                              uint8_t* __restrict__ out,
                                              const cb_deflate_summary* __restrict__ summary) {
    if (summary->status != CB_OK) return;  // a bad span or too small an output: nothing is written
    const int t = threadIdx.x;
    for (int64_t sp = blockIdx.x; sp < n; sp += gridDim.x) {
        const uint32_t cs = meta[META * sp], crc = meta[META * sp + 1], isize = meta[META * sp + 3];
        uint8_t* d = out + out_off[sp];
        const uint8_t* s = slots + sp * SLOT;
        const uint32_t h = frame ? 18 : 0;
        if (frame && t < 18) {
            // gzip header with the BGZF extra field BC (SAMv1 4.1): BSIZE = member bytes - 1
            const uint32_t bsize = cs + 25;
            const uint8_t hb[16] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67, 2, 0};
            d[t] = t < 16 ? hb[t] : (uint8_t)(t == 16 ? bsize & 255 : bsize >> 8);
        }
        for (uint32_t i = t; i < cs; i += blockDim.x) d[h + i] = s[i];
        if (frame && t < 8) d[h + cs + t] = (uint8_t)(t < 4 ? crc >> (8 * t) : isize >> (8 * (t - 4)));
    }
}

// CRC32 of spans, one warp per span (lane columns joined as in span_crc).
__global__ void __launch_bounds__(256) k_crc32_spans(const uint8_t* __restrict__ data, const int64_t* __restrict__ off,
                                                     const int64_t* __restrict__ size, int64_t n,
                                                     uint32_t* __restrict__ out) {
    __shared__ uint32_t T[8][256];
    init_crc8(T);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n) return;
    const uint8_t* p = data + off[w];
    const int64_t len = size[w] > 0 ? size[w] : 0;
    const int64_t seg = (len + 31) / 32, pad = 32 * seg - len;
    const int64_t r1 = (int64_t)lane * seg + seg - pad;
    uint32_t col = 0;
    for (int64_t r = max((int64_t)0, (int64_t)lane * seg - pad); r < r1; r++) col = T[0][(col ^ p[r]) & 255] ^ (col >> 8);
    uint32_t ck = xpow_from(kCrc.x2n, 8ull * (unsigned long long)seg);
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const uint32_t other = __shfl_down_sync(FULL, col, 1 << k);
        if ((lane & ((2 << k) - 1)) == 0) col = gf_mul(col, ck) ^ other;
        ck = gf_mul(ck, ck);
    }
    if (lane == 0) out[w] = crc_finish(col, (unsigned long long)len);
}

// Adler-32 of spans, one warp per span: lane sums s1 = sum d, s2 = sum (L - j) d over its part,
// joined as B = n + sum (s2 + (bytes after the part) * s1).
__global__ void __launch_bounds__(256) k_adler32_spans(const uint8_t* __restrict__ data,
                                                       const int64_t* __restrict__ off,
                                                       const int64_t* __restrict__ size, int64_t n,
                                                       uint32_t* __restrict__ out) {
    constexpr uint32_t MOD = 65521u;
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n) return;
    const uint8_t* p = data + off[w];
    const int64_t len = size[w] > 0 ? size[w] : 0;
    const int64_t seg = (len + 31) / 32;
    const int64_t b0 = min(len, (int64_t)lane * seg), b1 = min(len, b0 + seg);
    uint32_t s1 = 0, s2 = 0;
    for (int64_t r = b0; r < b1;) {
        const int64_t e = min(b1, r + 1024);
        for (; r < e; r++) {
            s1 += p[r];
            s2 += s1;
        }
        s1 %= MOD;
        s2 %= MOD;
    }
    const uint64_t after = (uint64_t)(len - b1) % MOD;
    uint64_t A = s1, B = (s2 + after * s1) % MOD;
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) {
        A += __shfl_down_sync(FULL, A, k);
        B += __shfl_down_sync(FULL, B, k);
    }
    if (lane == 0) {
        A = (1 + A) % MOD;
        B = ((uint64_t)len % MOD + B) % MOD;
        out[w] = (uint32_t)((B << 16) | A);
    }
}

// CTAs of the persistent grid on the current device (resident at once), at most MAX_CTAS and n.
int grid_for(int64_t n_spans) {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (!cached[dev]) {
        int sms = 0, per = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        if (cudaFuncSetAttribute(k_deflate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem)) !=
            cudaSuccess)
            return 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_deflate, NT, sizeof(Smem)) != cudaSuccess || per < 1)
            return 0;
        cached[dev] = sms * per;
    }
    int64_t g = cached[dev] < MAX_CTAS ? cached[dev] : MAX_CTAS;
    if (n_spans < g) g = n_spans > 0 ? n_spans : 1;
    return (int)g;
}

}  // namespace dfl
}  // namespace cb

using namespace cb;

int cb_set_error(cudaError_t e);                    // abi.cu
int cb_set_error_text(int code, const char* text);  // abi.cu

extern "C" size_t cb_deflate_workspace_bytes(int64_t n_spans) {
    if (n_spans < 0) return 0;
    const int64_t ctas = n_spans < dfl::MAX_CTAS ? (n_spans > 0 ? n_spans : 1) : dfl::MAX_CTAS;
    return (size_t)(ctas * dfl::TOKS * 4 + n_spans * dfl::SLOT + n_spans * dfl::META * 4 + 256);
}

extern "C" int cb_deflate_spans(const uint8_t* data, const int64_t* off, const int64_t* size, int64_t n, int level,
                                int bgzf, uint8_t* out, int64_t out_cap, int64_t* out_off, int64_t* out_size,
                                uint32_t* crc, cb_deflate_summary* summary, void* workspace, size_t workspace_bytes,
                                void* stream) {
    if (n < 0 || level < 0 || level > 9 || !summary || (n > 0 && (!data || !off || !size || !out || !out_off)))
        return cb_set_error_text(CB_ERR_ARG, "cb_deflate_spans: bad arguments");
    if (!workspace || workspace_bytes < cb_deflate_workspace_bytes(n))
        return cb_set_error_text(CB_ERR_CAPACITY, "cb_deflate_spans: workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(summary, 0, sizeof(cb_deflate_summary), s) != cudaSuccess)
        return cb_set_error(cudaGetLastError());
    if (n == 0) return CB_OK;
    const int grid = dfl::grid_for(n);
    if (grid <= 0) return cb_set_error_text(CB_ERR_CUDA, "cb_deflate_spans: no device, or the kernel does not fit");
    const int64_t ctas = n < dfl::MAX_CTAS ? n : dfl::MAX_CTAS;
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    uint32_t* tokens = reinterpret_cast<uint32_t*>(ws);
    uint8_t* slots = ws + ctas * dfl::TOKS * 4;
    uint32_t* meta = reinterpret_cast<uint32_t*>(slots + n * dfl::SLOT);
    dfl::k_deflate<<<grid, dfl::NT, sizeof(dfl::Smem), s>>>(data, off, size, n, level,
                                                          bgzf ? dfl::BGZF_SPAN : dfl::MAXSPAN, tokens, slots, meta,
                                                          summary);
    dfl::k_offsets<<<1, 1024, 0, s>>>(meta, n, bgzf, out_cap, out_off, out_size, crc, summary);
    const int pack_grid = (int)(n < 148 * 8 ? n : 148 * 8);
    dfl::k_pack<<<pack_grid, 256, 0, s>>>(slots, meta, n, bgzf, out_off, out, summary);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_crc32_spans(const uint8_t* data, const int64_t* off, const int64_t* size, int64_t n, uint32_t* out,
                              void* stream) {
    if (n < 0 || (n > 0 && (!data || !off || !size || !out)))
        return cb_set_error_text(CB_ERR_ARG, "cb_crc32_spans: bad arguments");
    if (n == 0) return CB_OK;
    dfl::k_crc32_spans<<<(unsigned)((n + 7) / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(data, off, size, n, out);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_adler32_spans(const uint8_t* data, const int64_t* off, const int64_t* size, int64_t n, uint32_t* out,
                                void* stream) {
    if (n < 0 || (n > 0 && (!data || !off || !size || !out)))
        return cb_set_error_text(CB_ERR_ARG, "cb_adler32_spans: bad arguments");
    if (n == 0) return CB_OK;
    dfl::k_adler32_spans<<<(unsigned)((n + 7) / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(data, off, size, n, out);
    return cb_set_error(cudaGetLastError());
}
