// DEFLATE code construction (RFC 1951), shared by the compressor kernel and host-side checks:
// length/distance symbols, minimum-redundancy code lengths limited to a maximum, canonical codes
// and the run-length coding of code lengths.  Every function is serial and bounded by its
// alphabet (at most 288 symbols).
#pragma once

#include <cstdint>

namespace cb {
namespace dfl {

constexpr int NLIT = 286;     // literal/length symbols that may be used (0-255, 256 = end, 257-285)
constexpr int NLIT_ALL = 288; // the fixed code also gives 286 and 287 lengths
constexpr int NDIST = 30;
constexpr int NCL = 19;
constexpr int MAXBITS = 15;   // longest literal/length or distance code
constexpr int CLBITS = 7;     // longest code-length code
constexpr int NRLE = 320;     // code-length symbols of one header, at most NLIT + NDIST

// RFC 1951 3.2.7: order of the code length code lengths in a dynamic block header.
static __constant__ uint8_t kClOrd[NCL] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
static const uint8_t kClOrdHost[NCL] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

__host__ __device__ inline uint32_t cl_order(int i) {
#ifdef __CUDA_ARCH__
    return kClOrd[i];
#else
    return kClOrdHost[i];
#endif
}

__host__ __device__ inline uint32_t ilog2(uint32_t v) {  // v > 0
#ifdef __CUDA_ARCH__
    return 31u - (uint32_t)__clz(v);
#else
    return 31u - (uint32_t)__builtin_clz(v);
#endif
}

__host__ __device__ inline uint32_t reverse_bits(uint32_t v, uint32_t n) {  // the low n bits (1..15) reversed
#ifdef __CUDA_ARCH__
    return __brev(v) >> (32u - n);
#else
    uint32_t r = 0;
    for (uint32_t i = 0; i < n; i++) r |= ((v >> i) & 1u) << (n - 1 - i);
    return r;
#endif
}

// Length symbol (257-285) of a match length 3-258, the number of its extra bits and their value.
__host__ __device__ inline uint32_t len_sym(uint32_t len) {
    const uint32_t v = len - 3;
    if (v < 8) return 257 + v;
    if (v == 255) return 285;
    const uint32_t k = ilog2(v);
    return 257 + 4 * (k - 1) + ((v >> (k - 2)) & 3);
}
__host__ __device__ inline uint32_t len_extra_bits(uint32_t sym) { return (sym < 265 || sym == 285) ? 0 : (sym - 261) / 4; }
__host__ __device__ inline uint32_t len_extra_val(uint32_t len) {
    const uint32_t v = len - 3;
    if (v < 8 || v == 255) return 0;
    return v & ((1u << (ilog2(v) - 2)) - 1);
}

// Distance symbol (0-29) of a distance 1-32768, the number of its extra bits and their value.
__host__ __device__ inline uint32_t dist_sym(uint32_t d) {
    const uint32_t v = d - 1;
    if (v < 4) return v;
    const uint32_t k = ilog2(v);
    return 2 * k + ((v >> (k - 1)) & 1);
}
__host__ __device__ inline uint32_t dist_extra_bits(uint32_t sym) { return sym < 4 ? 0 : sym / 2 - 1; }
__host__ __device__ inline uint32_t dist_extra_val(uint32_t d) {
    const uint32_t v = d - 1;
    if (v < 4) return 0;
    return v & ((1u << (ilog2(v) - 1)) - 1);
}

// Lengths of the fixed code (RFC 1951 3.2.6).
__host__ __device__ inline uint32_t fixed_lit_len(uint32_t s) { return s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : 8; }
constexpr uint32_t FIXED_DIST_LEN = 5;

// Minimum-redundancy code lengths, in place: A[0..m) holds m >= 2 weights in ascending order and
// receives the length of each (A[0], the lightest, gets the longest).  The in-place method of
// Moffat and Katajainen ("In-place calculation of minimum-redundancy codes", 1995): a first pass
// forms the internal node weights with parent links, a second turns the links into depths, a
// third counts leaves per depth.  mk_pass1 is the first pass alone.
__host__ __device__ inline void mk_pass1(uint32_t* A, int m) {
    // A[next] becomes the weight of internal node next; consumed internal nodes hold their parent
    int leaf = 2, root = 0;
    A[0] += A[1];
    for (int next = 1; next < m - 1; next++) {
        if (leaf >= m || A[root] < A[leaf]) {
            A[next] = A[root];
            A[root++] = (uint32_t)next;
        } else {
            A[next] = A[leaf++];
        }
        if (leaf >= m || (root < next && A[root] < A[leaf])) {
            A[next] += A[root];
            A[root++] = (uint32_t)next;
        } else {
            A[next] += A[leaf++];
        }
    }
}

__host__ __device__ inline void mk_lengths(uint32_t* A, int m) {
    mk_pass1(A, m);
    // pass 2: depth of each internal node (the root is A[m-2])
    A[m - 2] = 0;
    for (int next = m - 3; next >= 0; next--) A[next] = A[A[next]] + 1;
    // pass 3: leaves per depth, written from the heaviest end
    int avail = 1, used = 0, depth = 0;
    int root = m - 2;
    int next = m - 1;
    while (avail > 0) {
        while (root >= 0 && (int)A[root] == depth) {
            used++;
            root--;
        }
        while (avail > used && next >= 0) {
            A[next--] = (uint32_t)depth;
            avail--;
        }
        avail = 2 * used;
        depth++;
        used = 0;
    }
}

// Lengths A[0..m) (non-increasing, a complete code) limited to at most L bits, still complete:
// lengths over L are cut to L, then while the Kraft sum is over 1 a leaf at depth L is removed and
// the deepest leaf above L is split into two, each step lowering the sum by one unit of 2^-L.
// Lengths are then handed out again, longest first, in the same symbol order.
__host__ __device__ inline void limit_lengths(uint32_t* A, int m, uint32_t L) {
    if (A[0] <= L) return;
    uint32_t bl[16] = {0};
    for (int i = 0; i < m; i++) bl[A[i] > L ? L : A[i]]++;
    uint32_t kraft = 0;
    for (uint32_t l = 1; l <= L; l++) kraft += bl[l] << (L - l);
    while (kraft > (1u << L) && bl[L] > 0) {
        bl[L]--;
        for (uint32_t l = L - 1; l > 0; l--) {
            if (bl[l]) {
                bl[l]--;
                bl[l + 1] += 2;
                break;
            }
        }
        kraft--;
    }
    int i = 0;
    for (uint32_t l = L; l >= 1; l--)
        for (uint32_t c = bl[l]; c > 0 && i < m; c--) A[i++] = l;
}

// The same lengths as mk_lengths + limit_lengths, as counts: cum[l] = codes of length <= l
// (l = 0..L) from c[d] = internal nodes at depth d (d = 0..maxd, the root at depth 0) of the
// minimum-redundancy tree.  The leaves at depth d are 2 c[d-1] - c[d]; depths over L are limited by
// the loop of limit_lengths.  The i-th lightest of m symbols then gets length_of_rank(m - 1 - i).
__host__ __device__ inline void lengths_from_depths(const uint32_t* c, int maxd, uint32_t L, uint32_t* cum) {
    uint32_t bl[16] = {0};
    int deepest = 0;
    for (int d = 1; d <= maxd + 1; d++) {
        const uint32_t leaves = 2 * c[d - 1] - (d <= maxd ? c[d] : 0u);
        if (leaves) {
            deepest = d;
            bl[d > (int)L ? L : (uint32_t)d] += leaves;
        }
    }
    if (deepest > (int)L) {
        uint32_t kraft = 0;
        for (uint32_t l = 1; l <= L; l++) kraft += bl[l] << (L - l);
        while (kraft > (1u << L) && bl[L] > 0) {
            bl[L]--;
            for (uint32_t l = L - 1; l > 0; l--) {
                if (bl[l]) {
                    bl[l]--;
                    bl[l + 1] += 2;
                    break;
                }
            }
            kraft--;
        }
    }
    cum[0] = 0;
    for (uint32_t l = 1; l <= L; l++) cum[l] = cum[l - 1] + bl[l];
    for (uint32_t l = L + 1; l < 16; l++) cum[l] = cum[L];
}

// The length of the symbol of heavy rank j (0 = the most frequent): the shortest length whose
// cumulative count passes j.
__host__ __device__ inline uint32_t length_of_rank(uint32_t j, const uint32_t* cum) {
    uint32_t l = 1;
    while (l < 15 && cum[l] <= j) l++;
    return l;
}

// The code-length symbols of one run of r >= 1 equal lengths v, as rle_lengths writes them (sym
// may be null: only counted).  Returns the number of symbols.
__host__ __device__ inline int rle_run(uint8_t v, int run, uint8_t* sym, uint8_t* ext) {
    int k = 0;
    if (v == 0) {
        while (run >= 11) {
            const int r = run < 138 ? run : 138;
            if (sym) { sym[k] = 18; ext[k] = (uint8_t)(r - 11); }
            k++;
            run -= r;
        }
        if (run >= 3) {
            if (sym) { sym[k] = 17; ext[k] = (uint8_t)(run - 3); }
            k++;
            run = 0;
        }
    } else {
        if (sym) { sym[k] = v; ext[k] = 0; }
        k++;
        run--;
        while (run >= 3) {
            const int r = run < 6 ? run : 6;
            if (sym) { sym[k] = 16; ext[k] = (uint8_t)(r - 3); }
            k++;
            run -= r;
        }
    }
    for (; run > 0; run--) {
        if (sym) { sym[k] = v; ext[k] = 0; }
        k++;
    }
    return k;
}

// Code lengths of an alphabet of nsym symbols from their counts.  sorted[0..m): the symbols with
// nonzero counts by ascending (count, symbol); A: m words of scratch.  Fewer than two used symbols
// still get a complete two-code (lengths 1 and 1), as decoders want.
__host__ __device__ inline void build_lengths(const uint32_t* freq, const uint16_t* sorted, int m, int nsym,
                                              uint32_t* A, uint8_t* len, uint32_t L) {
    for (int s = 0; s < nsym; s++) len[s] = 0;
    if (m == 0) {
        len[0] = len[1] = 1;
        return;
    }
    if (m == 1) {
        len[sorted[0]] = 1;
        len[sorted[0] == 0 ? 1 : 0] = 1;
        return;
    }
    for (int i = 0; i < m; i++) A[i] = freq[sorted[i]];
    mk_lengths(A, m);
    limit_lengths(A, m, L);
    for (int i = 0; i < m; i++) len[sorted[i]] = (uint8_t)A[i];
}

// Canonical codes (RFC 1951 3.2.2) of lengths len[0..nsym): code[s] = length << 16 | the code's
// bits reversed (DEFLATE sends Huffman codes most significant bit first into an LSB-first stream).
__host__ __device__ inline void canonical_codes(const uint8_t* len, int nsym, uint32_t* code) {
    uint32_t bl[16] = {0}, next[16] = {0};
    for (int s = 0; s < nsym; s++) bl[len[s] & 15]++;
    bl[0] = 0;
    uint32_t c = 0;
    for (int l = 1; l <= 15; l++) {
        c = (c + bl[l - 1]) << 1;
        next[l] = c;
    }
    for (int s = 0; s < nsym; s++) {
        const uint32_t l = len[s] & 15;
        code[s] = l ? (l << 16) | reverse_bits(next[l]++, l) : 0u;
    }
}

// Run-length coding of the code lengths lit[0..hlit) followed by dist[0..hdist) (RFC 1951 3.2.7):
// symbols 0-15 are lengths, 16 repeats the previous length 3-6 times (2 extra bits), 17 and 18 give
// 3-10 and 11-138 zeros (3 and 7 extra bits).  Returns the number of symbols written.
__host__ __device__ inline int rle_lengths(const uint8_t* lit, int hlit, const uint8_t* dist, int hdist, uint8_t* sym,
                                           uint8_t* ext) {
    const int total = hlit + hdist;
    int k = 0, i = 0;
    while (i < total) {
        const uint8_t v = i < hlit ? lit[i] : dist[i - hlit];
        int run = 1;
        while (i + run < total && (i + run < hlit ? lit[i + run] : dist[i + run - hlit]) == v) run++;
        i += run;
        if (v == 0) {
            while (run >= 11) {
                const int r = run < 138 ? run : 138;
                sym[k] = 18;
                ext[k++] = (uint8_t)(r - 11);
                run -= r;
            }
            if (run >= 3) {
                sym[k] = 17;
                ext[k++] = (uint8_t)(run - 3);
                run = 0;
            }
        } else {
            sym[k] = v;
            ext[k++] = 0;
            run--;
            while (run >= 3) {
                const int r = run < 6 ? run : 6;
                sym[k] = 16;
                ext[k++] = (uint8_t)(r - 3);
                run -= r;
            }
        }
        for (; run > 0; run--) {
            sym[k] = v;
            ext[k++] = 0;
        }
    }
    return k;
}

__host__ __device__ inline uint32_t cl_extra_bits(uint32_t s) { return s == 16 ? 2 : s == 17 ? 3 : s == 18 ? 7 : 0; }

}  // namespace dfl
}  // namespace cb
