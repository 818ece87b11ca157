// Raw-DEFLATE inflater for BGZF members, form 3: the Huffman decode and the copy in two kernels.
//
// Replaces cubam's nvcompBatchedDeflateDecompressAsync call and its status/size check
// (src/cubam/bgzf.py:587-611) with the CRC32 check added (cubam's reader does not check it,
// docs/reading.md:48-51).  DEFLATE is RFC 1951.
//
// Why two kernels.  Huffman decoding is serial within a member, and the copy of a back-reference
// needs the member's output up to 32 KiB back.  In BGZF files of BAM records most references reach
// far (on the GEX-shaped workload the median distance is about 3 KB and only 7% are within 224
// bytes), so a decoder that also copies either keeps 32 KiB per member on chip (few members in
// flight, idle issue slots) or reads HBM at every match (long waits).  Here:
//
//  1. k_decode: one member per LANE.  32 members per warp advance one symbol per step in lock step,
//     each lane with its own tables in shared memory (16-bit entries, 2^LB literal/length and 2^DB
//     distance root entries; longer codes by per-length limits kept in registers).  A step is one
//     straight path for literals and matches alike (the warp pays for every path a lane takes, so
//     they are merged and predicated), with a 64-bit bit buffer fed from two prefetched words, and
//     writes the
//     symbols as 16-bit units to a token arena in HBM: a literal is one unit, a match two (length and
//     the high distance bits, then the low distance bits).  Block headers, code lengths and stored
//     blocks are steps of the same lock-step loop; the code tables of one lane are built by the
//     whole warp.  The output size, distances and the end of the payload are checked here.
//  2. k_copy: one member per WARP.  The warp reads its member's units 32 at a time, places them by
//     a prefix sum of their lengths, and writes the bytes 32 at a time into a 16 KiB ring in shared
//     memory (sources up to about 16 KiB back; older ones, about one match in eight on the GEX-shaped
//     workload, read the output already written to HBM); a byte finds its token from a bit mask of the
//     tokens that start in its 32 bytes (one warp OR-reduction and a population count), and a byte
//     whose source lies in the same 32 bytes takes it from another lane.  Completed 1 KiB windows go to HBM with 16-byte stores and into
//     the CRC32 (32 lane columns joined in GF(2)).
//
// Units are at most one per output byte, so a member's units take at most 2 ISIZE bytes: the arena
// gives every member a slot of 2 ISIZE + 8 bytes at the prefix sum of the slots before it.
//
// Every loop is bounded: each decode step consumes input bits or produces output bytes, both
// bounded per member; every shared-memory index is masked or checked; arena and output writes
// stay within the member's slot and output range.

#include <mutex>

#include "common.cuh"
#include "crc.cuh"

namespace cb {
namespace split {

// ---------------------------------------------------------------- formats

// 16-bit table entries (k_decode).
//   bit 15 set: a length symbol: bits 12-14 extra bits, 8-11 code length, 0-7 base - 3.
//   bit 15 clear: bits 12-14 kind, 8-11 code length, 0-7 value:
//     0 literal (value: the byte), 1 end of block, 2 distance (value: symbol 0-29),
//     3 special (value 0: a code longer than the root bits; 1: no such code), 4 code-length symbol.
enum : uint32_t { E_LIT = 0, E_EOB = 1, E_DIST = 2, E_SPECIAL = 3, E_CL = 4 };
constexpr uint16_t E_LONG = (uint16_t)(E_SPECIAL << 12);
constexpr uint16_t E_BAD = (uint16_t)((E_SPECIAL << 12) | 1u);

__device__ __forceinline__ uint32_t e_len(uint32_t e) { return (e >> 8) & 15u; }
__device__ __forceinline__ uint32_t e_kind(uint32_t e) { return (e >> 12) & 7u; }

// RFC 1951 3.2.5 in closed form: length symbol i = sym - 257 (0-28), distance symbol i (0-29).
__device__ __forceinline__ void len_code(uint32_t i, uint32_t& base, uint32_t& ext) {
    if (i < 4) {
        base = 3 + i;
        ext = 0;
    } else if (i == 28) {
        base = 258;
        ext = 0;
    } else {
        ext = (i >> 2) - 1;
        base = 3 + ((4u | (i & 3u)) << ext);
    }
}
__device__ __forceinline__ void dist_code(uint32_t i, uint32_t& base, uint32_t& ext) {
    if (i < 4) {
        base = 1 + i;
        ext = 0;
    } else {
        ext = (i >> 1) - 1;
        base = 1 + ((2u | (i & 1u)) << ext);
    }
}

// RFC 1951 3.2.7: order of the code length code lengths.
__constant__ uint8_t kClOrder[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

enum : int { T_CL = 0, T_LIT = 1, T_DIST = 2 };

__device__ __forceinline__ uint16_t sym_entry(int kind, uint32_t s, uint32_t L) {
    if (kind == T_CL) return (uint16_t)((E_CL << 12) | (L << 8) | s);
    if (kind == T_LIT) {
        if (s < 256) return (uint16_t)((L << 8) | s);
        if (s == 256) return (uint16_t)((E_EOB << 12) | (L << 8));
        if (s < 286) {
            uint32_t base, ext;
            len_code(s - 257, base, ext);
            return (uint16_t)(0x8000u | (ext << 12) | (L << 8) | (base - 3));
        }
        return E_BAD;
    }
    if (s < 30) return (uint16_t)((E_DIST << 12) | (L << 8) | s);
    return E_BAD;
}

// 16-bit units (the token arena): a literal 0x00bb; a match head 0x8000 | (length - 3) << 6 |
// (distance - 1) >> 9, followed by its tail 0xC000 | ((distance - 1) & 0x1FF).
__device__ __forceinline__ uint32_t unit_match(uint32_t len, uint32_t dist) {
    const uint32_t d = dist - 1;
    return (0x8000u | ((len - 3) << 6) | (d >> 9)) | ((0xC000u | (d & 0x1FFu)) << 16);
}

// Workspace: [0, 256) queue counters; per job 16 bytes (units u32, status u32, arena slot u64); the
// arena after that, 256-byte aligned.  Job j's slot is the prefix sum of slot_bytes over the jobs
// before it (k_slots), so the arena holds 2 sum(ISIZE) + 16 n_jobs bytes at most, whatever the
// jobs' output offsets are.
constexpr size_t WS_HEAD = 256;
constexpr size_t PER_JOB = 16;
__host__ __device__ __forceinline__ size_t arena_offset(long long n_jobs) {
    return (WS_HEAD + PER_JOB * (size_t)n_jobs + 255) & ~(size_t)255;
}
// A slot's bytes: 2 ISIZE for the units and room for the last word, rounded to 8 so that every slot
// starts 8-byte aligned (k_decode stores the units as 4-byte words).
__host__ __device__ __forceinline__ unsigned long long slot_bytes(uint32_t isize) {
    return (2ull * isize + 8ull + 7ull) & ~7ull;
}

// The arena slot of every job: one CTA; thread t sums a contiguous run of jobs, a block scan joins
// the runs, and each thread writes its run's offsets.
constexpr int SLOT_NT = 1024;
__global__ void __launch_bounds__(SLOT_NT) k_slots(const cb_member_job* __restrict__ jobs, int64_t n_jobs,
                                                   const int64_t* __restrict__ d_n_jobs, uint8_t* ws) {
    // Each warp takes a contiguous segment of jobs, read coalesced with eight loads per lane in
    // flight: a first pass sums the segment's slots, the warps' sums are scanned, a second pass
    // writes the slot offsets.
    constexpr int NW = SLOT_NT / 32, U = 8;
    __shared__ unsigned long long wbase[NW + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long n = n_jobs;
    if (d_n_jobs) n = min((long long)n, (long long)*d_n_jobs);
    const long long seg = ((n + NW - 1) / NW + 32 * U - 1) / (32 * U) * (32 * U);
    const long long a = min((long long)warp * seg, n), b = min(a + seg, n);
    unsigned long long sum = 0;
    for (long long j0 = a; j0 < b; j0 += 32 * U) {
        uint32_t isz[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const long long j = j0 + k * 32 + lane;
            isz[k] = j < b ? jobs[j].isize : 0u;
        }
#pragma unroll
        for (int k = 0; k < U; k++) sum += j0 + k * 32 + lane < b ? (unsigned long long)slot_bytes(isz[k]) : 0ull;
    }
    for (int d = 16; d; d >>= 1) sum += __shfl_xor_sync(FULL, sum, d);
    if (lane == 0) wbase[warp] = sum;
    __syncthreads();
    if (warp == 0) {
        const unsigned long long x = lane < NW ? wbase[lane] : 0ull;
        unsigned long long tot;
        const unsigned long long e = warp_exclusive_scan(x, tot);
        __syncwarp();
        if (lane < NW) wbase[lane] = e;
    }
    __syncthreads();
    unsigned long long* slot = reinterpret_cast<unsigned long long*>(ws + WS_HEAD);
    unsigned long long carry = wbase[warp];
    for (long long j0 = a; j0 < b; j0 += 32 * U) {
        uint32_t isz[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const long long j = j0 + k * 32 + lane;
            isz[k] = j < b ? jobs[j].isize : 0u;
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            const long long j = j0 + k * 32 + lane;
            const unsigned long long v = j < b ? (unsigned long long)slot_bytes(isz[k]) : 0ull;
            unsigned long long t;
            const unsigned long long x = warp_exclusive_scan(v, t);
            if (j < b) slot[2 * j + 1] = carry + x;
            carry += t;
        }
    }
}

// ---------------------------------------------------------------- k_decode: one member per lane

template <int LB_, int DB_, int WARPS_>
struct DecCfg {
    static constexpr int LB = LB_, DB = DB_, WARPS = WARPS_;
    static constexpr int NLL = 15 - LB_, NLD = 15 - DB_;  // code lengths longer than the roots
    static constexpr uint32_t LMASK = (1u << LB_) - 1, DMASK = (1u << DB_) - 1;
    // One region per lane (bytes):
    //   LIT   u16[2^LB]  literal/length root entries
    //   DIST  u16[2^DB]  distance root entries
    //   DSYM  u16[32]    entries of the distance codes longer than DB, canonical order
    //   LSYM  u8[288]    low 8 bits of the symbols of literal/length codes longer than LB, canonical order
    //   LHI   u32[9]     bit i: symbol i of LSYM is 256 or more
    // While the lane reads a dynamic header: the code-length code's table (u16[128]) at 0, the
    // code lengths (up to 286 + 30 bytes) at LSYM, where the 19 lengths of the code-length code
    // wait first.
    static constexpr int LIT = 0, DIST = LIT + (2 << LB_), DSYM = DIST + (2 << DB_);
    static constexpr int LSYM = DSYM + 64 > 256 ? DSYM + 64 : 256;
    static constexpr int LHI = LSYM + 288;
    static constexpr int STRIDE = (LHI + 36 + 7) & ~7;
    static_assert(LSYM + 320 <= STRIDE && NLL <= 9 && NLD <= 10 && LB_ >= 5 && DB_ >= 4, "table sizes");
    struct WarpSmem {
        alignas(16) uint8_t lane[32][STRIDE];
        uint8_t lens[320];         // the code lengths of the lane whose tables the warp builds
        uint32_t scratch[48];
        uint32_t lim[20];          // limits computed for that lane: NLL literal/length, then NLD distance
    };
    struct CtaSmem {
        WarpSmem w[WARPS_];
    };
};

enum : int { S_IDLE = 0, S_HDR = 1, S_BUILD_CL = 2, S_CLENS = 3, S_BUILD = 4, S_RUN = 5, S_STORED = 6, S_FIN = 7,
             S_DONE = 8 };

// Canonical table of lens[0:nsym) for one lane, built by the whole warp: tab[2^lb] indexed by the
// next lb bits (LSB first); codes longer than lb bits have their entries in sym[] in canonical
// order and, for code length lb + 1 + i, lim[i] = (end of the length's codes, left-justified to 15
// bits) | (index in sym[] of its first code minus that code) << 16.  Acceptance as zlib's inflate:
// an over-subscribed code is an error; an incomplete one too, except a literal/length or distance
// code whose longest code has length 1 (the code-length code must be complete).  Returns false on
// error (the same in every lane).
__device__ __noinline__ bool build_lane(const uint8_t* lens, int nsym, int lb, int kind, uint16_t* tab, uint32_t* lim,
                                        uint16_t* sym, uint8_t* sym8, uint32_t* hi8, uint32_t* scratch) {
    const int lane = threadIdx.x & 31;
    if (lane < 16) scratch[lane] = 0;
    if (hi8 && lane < 9) hi8[lane] = 0;
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
    if (kind == T_CL && (incomplete || maxlen == 0)) return false;
    if (incomplete && maxlen > 1) return false;
    const uint32_t nshort = __shfl_sync(FULL, my_index, lb < 15 ? lb + 1 : 15);
    if (lim && lane > lb && lane < 16) {
        const uint32_t limit = (my_first + cnt) << (15 - lane);
        const int base = (int)(my_index - nshort) - (int)my_first;
        lim[lane - lb - 1] = (limit & 0xFFFFu) | ((uint32_t)(uint16_t)(int16_t)base << 16);
    }
    if (lane >= 1 && lane < 16) {
        scratch[lane] = my_index;        // running insertion index of the length
        scratch[16 + lane] = my_first;   // first code of the length
        scratch[32 + lane] = my_index;   // first index of the length
    }
    // slots no code reaches (an incomplete code) decode as errors; complete codes cover every slot
    if (incomplete || maxlen == 0)
        for (int i = lane; i < (1 << lb); i += 32) tab[i] = E_BAD;
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
            const uint16_t e = sym_entry(kind, (uint32_t)s, L);
            if ((int)L <= lb) {
                const uint32_t r = __brev(c) >> (32 - L);
                for (uint32_t x = r; x < (1u << lb); x += (1u << L)) tab[x] = e;
            } else {
                const uint32_t li = idx - nshort;
                if (sym8) {  // literal/length: the symbol's low byte, and a bit for 256 and up
                    sym8[li] = (uint8_t)s;
                    if (s >= 256) atomicOr(&hi8[li >> 5], 1u << (li & 31));
                } else {
                    sym[li] = e;
                }
                tab[__brev(c >> (L - lb)) >> (32 - lb)] = E_LONG;
            }
        }
        __syncwarp();
    }
    return true;
}

// The entry of a code longer than the root bits from the lane's limits: x holds the next 15+ bits.
template <int N, int NSYM>
__device__ __forceinline__ uint32_t long_entry(uint32_t x, const uint32_t (&lim)[N], const uint16_t* sym) {
    const uint32_t c = __brev(x) >> 17;  // the next 15 bits, first bit highest
    int idx = -1;
#pragma unroll
    for (int i = N - 1; i >= 0; i--)
        if (c < (lim[i] & 0xFFFFu)) idx = (int)(int16_t)(lim[i] >> 16) + (int)(c >> (N - 1 - i));
    return (idx >= 0 && idx < NSYM) ? (uint32_t)sym[idx] : (uint32_t)E_BAD;
}

// The same for literal/length codes, whose long-code symbols are kept as a low byte and a high bit.
template <int N>
__device__ __forceinline__ uint32_t long_lit_entry(uint32_t x, const uint32_t (&lim)[N], const uint8_t* sym8,
                                                   const uint32_t* hi8) {
    const uint32_t c = __brev(x) >> 17;  // the next 15 bits, first bit highest
    int idx = -1;
    uint32_t L = 0;
#pragma unroll
    for (int i = N - 1; i >= 0; i--) {
        if (c < (lim[i] & 0xFFFFu)) {
            idx = (int)(int16_t)(lim[i] >> 16) + (int)(c >> (N - 1 - i));
            L = (uint32_t)(16 - N + i);
        }
    }
    if (idx < 0 || idx >= 288) return E_BAD;
    const uint32_t sym = (uint32_t)sym8[idx] | (((hi8[idx >> 5] >> (idx & 31)) & 1u) << 8);
    return sym_entry(T_LIT, sym, L);
}

__device__ __forceinline__ void report(cb_inflate_summary* summary, uint32_t* job_status, long long j, uint32_t st) {
    if (job_status) job_status[j] = st;
    if (st != CB_OK) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&summary->n_bad), 1ull);
        atomicMin(reinterpret_cast<long long*>(&summary->first_bad), j);
        atomicMax(&summary->status, (int)st);
    }
}

__device__ __forceinline__ uint32_t load_word(const uint32_t* wbase, uint32_t nvalid, uint32_t w) {
    return w < nvalid ? __ldg(wbase + w) : 0u;
}

// Block k (16 bytes, words 4k..4k+3) of a lane's input: one 16-byte load when the whole block lies
// within the nvalid readable words, else word by word (zero past the end).
__device__ __forceinline__ uint4 load_block(const uint32_t* base16, uint32_t nvalid, uint32_t k) {
    const uint32_t w = 4 * k;
    if (w + 3 < nvalid) return __ldg(reinterpret_cast<const uint4*>(base16) + k);
    uint4 v;
    v.x = w < nvalid ? __ldg(base16 + w) : 0u;
    v.y = w + 1 < nvalid ? __ldg(base16 + w + 1) : 0u;
    v.z = w + 2 < nvalid ? __ldg(base16 + w + 2) : 0u;
    v.w = w + 3 < nvalid ? __ldg(base16 + w + 3) : 0u;
    return v;
}

// A hint to bring the 128-byte line of p into L2 (a prefetch, no load into registers).
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

template <class C>
__global__ void __launch_bounds__(C::WARPS * 32)
    k_decode(const cb_member_job* __restrict__ jobs, int64_t n_jobs, const int64_t* __restrict__ d_n_jobs,
             uint32_t* job_status, cb_inflate_summary* summary, uint8_t* ws, unsigned long long arena_bytes,
             int steps, uint32_t ahead, long long j0, long long j1, int qi) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    typename C::CtaSmem& S = *reinterpret_cast<typename C::CtaSmem*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    typename C::WarpSmem& W = S.w[warp];
    unsigned long long* queue = reinterpret_cast<unsigned long long*>(ws) + qi;  // this launch's counter
    uint32_t* per_job = reinterpret_cast<uint32_t*>(ws + WS_HEAD);  // (units, status, slot lo, slot hi) per job
    uint8_t* arena = ws + arena_offset(n_jobs);
    long long n = n_jobs;
    if (d_n_jobs) n = min((long long)n, (long long)*d_n_jobs);
    n = min(n, j1);  // this launch's jobs: [j0, j1)

    uint8_t* const my_base = W.lane[lane];
    const uint16_t* my_lit = reinterpret_cast<const uint16_t*>(my_base + C::LIT);
    const uint16_t* my_dist = reinterpret_cast<const uint16_t*>(my_base + C::DIST);
    const uint16_t* my_dsym = reinterpret_cast<const uint16_t*>(my_base + C::DSYM);
    const uint8_t* my_lsym = my_base + C::LSYM;
    const uint32_t* my_lhi = reinterpret_cast<const uint32_t*>(my_base + C::LHI);
    const uint16_t* my_cltab = reinterpret_cast<const uint16_t*>(my_base);  // while a header is read
    uint8_t* my_lens = my_base + C::LSYM;  // code lengths while a header is read (after the 19 below)

    // the member of this lane
    int st = S_IDLE;
    long long j = 0;
    // bit reader: bb holds bc bits (LSB first), fed from registers: a0-a3 the words left of the current
    // 16-byte block (acnt of them, a0 next), blk the next block, loaded a block ahead (nb: the block
    // after it); wfed words went into bb so far
    const uint32_t* wbase = nullptr;  // 16-byte aligned start at or before the payload
    uint64_t bb = 0;
    uint32_t bc = 0, a0 = 0, a1 = 0, a2 = 0, a3 = 0, acnt = 0, nb = 0, wfed = 0, nvalid = 0;
    uint4 blk = make_uint4(0, 0, 0, 0);
    uint32_t s0 = 0, in_bits = 0, isize = 0, pos = 0;
    bool final_block = false;
    uint32_t rem = 0, hlit = 0, total = 0, ci = 0;  // stored bytes left; code lengths read
    uint32_t* slot = nullptr;
    uint32_t nunits = 0, nwords = 0, half = 0, has = 0;  // units written, u32 words stored, a pending unit
    uint32_t err = CB_OK;
    uint32_t llim[C::NLL], dlim[C::NLD];
#pragma unroll
    for (int i = 0; i < C::NLL; i++) llim[i] = 0;
#pragma unroll
    for (int i = 0; i < C::NLD; i++) dlim[i] = 0;

    auto next_word = [&]() {  // a0 went into bb: the next word becomes a0
        a0 = a1;
        a1 = a2;
        a2 = a3;
        wfed++;
        if (--acnt == 0) {
            a0 = blk.x;
            a1 = blk.y;
            a2 = blk.z;
            a3 = blk.w;
            acnt = 4;
            blk = load_block(wbase, nvalid, nb);
            // entering a new 128-byte line of input: ask L2 for the line `ahead` lines further on, so
            // that the block loads find the lane's stream in L2 rather than DRAM
            if (ahead && (nb & 7u) == 0 && 4 * (nb + 8 * ahead) < nvalid) prefetch_l2(wbase + 4 * (nb + 8 * ahead));
            nb++;
        }
    };
    auto refill = [&]() {  // afterwards bc >= 33
        if (bc <= 32) {
            bb |= (uint64_t)a0 << bc;
            bc += 32;
            next_word();
        }
    };
    auto consume = [&](uint32_t k) {  // k <= bc
        bb >>= k;
        bc -= k;
    };
    auto consumed = [&]() { return wfed * 32u - bc - s0; };  // bits of the payload used
    auto put = [&](uint32_t v, uint32_t k) {  // append k (0, 1 or 2) units, packed low unit first
        if (k) {
            const uint32_t wv = has ? (half | (v << 16)) : v;
            if (k == 2 || has) slot[nwords++] = wv;
            half = has ? (v >> 16) : v;
            has ^= k & 1u;
            nunits += k;
        }
    };
    auto fail = [&](uint32_t code) {
        err = code;
        st = S_FIN;
    };

    for (;;) {
        // ---- lanes without a member take the next ones (one atomic per warp)
        const unsigned idle = __ballot_sync(FULL, st == S_IDLE);
        if (idle) {
            const int leader = __ffs(idle) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(queue, (unsigned long long)__popc(idle));
            base = __shfl_sync(FULL, base, leader);
            if (st == S_IDLE) {
                j = j0 + (long long)base + __popc(idle & ((1u << lane) - 1u));
                if (j >= n) {
                    st = S_DONE;
                } else {
                    const cb_member_job job = jobs[j];
                    const uintptr_t in = (uintptr_t)job.in;
                    wbase = reinterpret_cast<const uint32_t*>(in & ~(uintptr_t)15);
                    s0 = (uint32_t)(in & 15) * 8;  // bits of the first block before the payload
                    nvalid = (uint32_t)((in + job.in_len + 8 - (uintptr_t)wbase) >> 2);
                    in_bits = job.in_len * 8u;
                    isize = job.isize;
                    bb = 0;
                    bc = 0;
                    wfed = 0;
                    const uint4 b0 = load_block(wbase, nvalid, 0);
                    a0 = b0.x;
                    a1 = b0.y;
                    a2 = b0.z;
                    a3 = b0.w;
                    acnt = 4;
                    blk = load_block(wbase, nvalid, 1);
                    nb = 2;
                    for (uint32_t q = 0; q < (s0 >> 5); q++) next_word();  // whole words before the payload
                    refill();
                    refill();
                    consume(s0 & 31u);
                    pos = 0;
                    final_block = false;
                    nunits = nwords = half = has = 0;
                    err = CB_OK;
                    st = S_HDR;
                    const unsigned long long so = reinterpret_cast<const unsigned long long*>(per_job)[2 * j + 1];
                    slot = reinterpret_cast<uint32_t*>(arena + so);
                    if (so + slot_bytes(isize) > arena_bytes) fail(CB_ERR_CAPACITY);
                }
            }
        }
        if (__all_sync(FULL, st == S_DONE)) break;

        // ---- code tables, built by the whole warp for one lane at a time
        for (unsigned b = __ballot_sync(FULL, st == S_BUILD_CL || st == S_BUILD); b; b &= b - 1) {
            const int t = __ffs(b) - 1;
            const int tst = __shfl_sync(FULL, st, t);
            bool ok;
            uint8_t* tb = W.lane[t];
            if (tst == S_BUILD_CL) {
                // the code-length code: its 19 lengths wait at LSYM; its table goes to the region's start,
                // then the code lengths to come start from zero (runs of zeros are not written)
                if (lane < 19) W.lens[lane] = tb[C::LSYM + lane];
                __syncwarp();
                ok = build_lane(W.lens, 19, 7, T_CL, reinterpret_cast<uint16_t*>(tb), nullptr, nullptr, nullptr,
                                nullptr, W.scratch);
                for (int k = lane; k < 80; k += 32) reinterpret_cast<uint32_t*>(tb + C::LSYM)[k] = 0;
            } else {
                // literal/length and distance codes: fixed (hlit 0 marks a fixed block) or lane t's lengths
                const uint32_t th = __shfl_sync(FULL, hlit, t);
                const uint32_t ttot = __shfl_sync(FULL, total, t);
                int nl, nd;
                if (th == 0) {
                    for (int s = lane; s < 320; s += 32)
                        W.lens[s] = s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : s < 288 ? 8 : 5;
                    nl = 288;
                    nd = 32;
                } else {
                    for (uint32_t s = lane; s < ttot; s += 32) W.lens[s] = tb[C::LSYM + s];
                    nl = (int)th;
                    nd = (int)(ttot - th);
                }
                __syncwarp();
                ok = build_lane(W.lens, nl, C::LB, T_LIT, reinterpret_cast<uint16_t*>(tb + C::LIT), W.lim, nullptr,
                                tb + C::LSYM, reinterpret_cast<uint32_t*>(tb + C::LHI), W.scratch) &&
                     build_lane(W.lens + nl, nd, C::DB, T_DIST, reinterpret_cast<uint16_t*>(tb + C::DIST),
                                W.lim + C::NLL, reinterpret_cast<uint16_t*>(tb + C::DSYM), nullptr, nullptr, W.scratch);
            }
            __syncwarp();
            if (lane == t) {
                if (!ok) {
                    fail(CB_ERR_INFLATE);
                } else if (tst == S_BUILD_CL) {
                    st = S_CLENS;
                    ci = 0;
                } else {
#pragma unroll
                    for (int i = 0; i < C::NLL; i++) llim[i] = W.lim[i];
#pragma unroll
                    for (int i = 0; i < C::NLD; i++) dlim[i] = W.lim[C::NLL + i];
                    st = S_RUN;
                }
            }
            __syncwarp();
        }

        // ---- block headers and member ends (each lane its own; rare)
        if (st == S_HDR) {
            if (consumed() > in_bits) {
                fail(CB_ERR_INFLATE);
            } else {
                refill();
                const uint32_t h = (uint32_t)bb & 7u;
                consume(3);
                final_block = (h & 1u) != 0;
                const uint32_t btype = h >> 1;
                if (btype == 0) {
                    consume(bc & 7u);  // to a byte boundary: whole words are loaded, so bc & 7 bits remain
                    refill();
                    const uint32_t x = (uint32_t)bb;
                    const uint32_t len = x & 0xFFFFu, nlen = x >> 16;
                    consume(32);
                    if (len != (~nlen & 0xFFFFu) || len > isize - pos || consumed() + 8ull * len > in_bits) {
                        fail(CB_ERR_INFLATE);
                    } else {
                        rem = len;
                        st = len ? S_STORED : (final_block ? S_FIN : S_HDR);
                    }
                } else if (btype == 1) {
                    hlit = 0;  // fixed codes
                    st = S_BUILD;
                } else if (btype == 2) {
                    refill();
                    const uint32_t x = (uint32_t)bb;
                    hlit = (x & 31u) + 257;
                    const uint32_t hdist = ((x >> 5) & 31u) + 1, hclen = ((x >> 10) & 15u) + 4;
                    consume(14);
                    if (hlit > 286 || hdist > 30) {
                        fail(CB_ERR_INFLATE);
                    } else {
                        total = hlit + hdist;
                        uint32_t* zc = reinterpret_cast<uint32_t*>(my_lens);
#pragma unroll
                        for (int k = 0; k < 5; k++) zc[k] = 0;
                        for (uint32_t i = 0; i < hclen; i++) {
                            refill();
                            my_lens[kClOrder[i]] = (uint8_t)(bb & 7u);
                            consume(3);
                        }
                        st = S_BUILD_CL;
                    }
                } else {
                    fail(CB_ERR_INFLATE);
                }
            }
        }
        if (st == S_FIN) {
            if (err == CB_OK && (consumed() > in_bits || pos != isize)) err = CB_ERR_INFLATE;
            if (err == CB_OK && has) slot[nwords] = half;  // the last unit (the slot has 8 spare bytes)
            per_job[4 * j] = nunits;
            per_job[4 * j + 1] = err;
            report(summary, job_status, j, err);
            st = S_IDLE;
        }

        // ---- decode steps (lock step over the lanes' own streams); one straight path per symbol
#pragma unroll 1
        for (int k = 0; k < steps; k++) {
            if (st == S_RUN) {
                refill();
                const uint32_t x = (uint32_t)bb;
                uint32_t e = my_lit[x & C::LMASK];
                if (e == E_LONG) e = long_lit_entry<C::NLL>(x, llim, my_lsym, my_lhi);
                const uint32_t L = e_len(e);
                const bool is_len = (e & 0x8000u) != 0;
                const bool is_lit = e < 0x1000u;
                const bool is_eob = !is_len && e_kind(e) == E_EOB;
                const uint32_t ext = is_len ? (e >> 12) & 7u : 0u;
                const uint32_t len = (e & 255u) + 3 + ((x >> L) & ((1u << ext) - 1u));
                const uint32_t n1 = L + ext;  // <= 20 < bc
                // the distance (used by lengths only) from the 32 bits after n1: the rest of bb and,
                // past its bc bits, the next word a0 -- no refill inside the step
                const uint32_t avail = bc - n1;
                const uint32_t y = (uint32_t)(bb >> n1) | (avail < 32 ? a0 << avail : 0u);
                uint32_t d = my_dist[y & C::DMASK];
                if (is_len && d == E_LONG) d = long_entry<C::NLD, 32>(y, dlim, my_dsym);
                const uint32_t dl = e_len(d);
                uint32_t dbase, dext;
                dist_code(d & 31u, dbase, dext);
                const uint32_t dist = dbase + ((y >> dl) & ((1u << dext) - 1u));
                // a literal may take the next code too when it is a literal of the root table: at most 15
                // bits went to the first, and bb holds 33 or more (the step's second symbol)
                const uint32_t xb = (uint32_t)(bb >> L);
                const uint32_t eb = my_lit[xb & C::LMASK];
                const bool two = is_lit && eb < 0x1000u && pos + 1 < isize;
                const uint32_t k = n1 + (is_len ? dl + dext : two ? e_len(eb) : 0u);  // <= 48
                if (k < bc) {
                    consume(k);
                } else {  // the step used bits of a0: it becomes the buffer
                    const uint32_t r = k - bc;  // < 16
                    bb = (uint64_t)(a0 >> r);
                    bc = 32 - r;
                    next_word();
                }
                const bool bad = (!is_len && !is_lit && !is_eob) || (is_lit && pos >= isize) ||
                                 (is_len && (e_kind(d) != E_DIST || (d & 0x8000u) || dist > pos || len > isize - pos));
                if (bad) {
                    fail(CB_ERR_INFLATE);
                } else {
                    put(is_len ? unit_match(len, dist) : two ? ((e & 255u) | ((eb & 255u) << 16)) : (e & 255u),
                        is_len ? 2u : two ? 2u : is_lit ? 1u : 0u);
                    pos += is_len ? len : two ? 2u : is_lit ? 1u : 0u;
                    if (is_eob) st = final_block ? S_FIN : S_HDR;
                }
            } else if (st == S_CLENS) {
                refill();
                const uint32_t x = (uint32_t)bb;
                const uint32_t e = my_cltab[x & 127u];
                const uint32_t L = e_len(e), s = e & 255u;
                const uint32_t eb = s < 16 ? 0u : s == 16 ? 2u : s == 17 ? 3u : 7u;
                const uint32_t rep = s < 16 ? 1u : (s == 18 ? 11u : 3u) + ((x >> L) & ((1u << eb) - 1u));
                // a second plain length in the same step when its code follows (14 bits at most went to
                // the first, bb holds 33 or more)
                const uint32_t e2 = my_cltab[(uint32_t)(bb >> (L + eb)) & 127u];
                const uint32_t s2 = e2 & 255u, L2 = e_len(e2);
                const bool two = e_kind(e2) == E_CL && !(e2 & 0x8000u) && L2 != 0 && s2 < 16 && ci + rep < total;
                consume(L + eb + (two ? L2 : 0u));
                if (e_kind(e) != E_CL || (e & 0x8000u) || L == 0 || (s == 16 && ci == 0) || ci + rep > total) {
                    fail(CB_ERR_INFLATE);
                } else {
                    if (s < 16) {
                        my_lens[ci] = (uint8_t)s;
                    } else if (s == 16) {
                        const uint8_t v = my_lens[ci - 1];
                        for (uint32_t r = 0; r < rep; r++) my_lens[ci + r] = v;  // 3-6 copies
                    }
                    ci += rep;
                    if (two) my_lens[ci++] = (uint8_t)s2;
                    if (ci == total) {
                        if (my_lens[256] == 0) fail(CB_ERR_INFLATE);  // no end-of-block code
                        else st = S_BUILD;
                    }
                }
            } else if (st == S_STORED) {
                refill();
                const uint32_t x = (uint32_t)bb;
                const uint32_t k2 = rem >= 2 ? 2u : 1u;
                consume(8 * k2);
                put(k2 == 2 ? ((x & 255u) | ((x << 8) & 0xFF0000u)) : (x & 255u), k2);
                pos += k2;
                rem -= k2;
                if (rem == 0) st = final_block ? S_FIN : S_HDR;
            }
        }
    }
}

// ---------------------------------------------------------------- k_copy: one member per warp

constexpr int WIN = 1024;                 // flush and CRC window
static_assert(WIN == 32 * 32, "one 32-byte CRC column per lane");

// WARPS_ warps per CTA, each with a ring of RING_ bytes: sources up to RING_ - 32 bytes back read
// the ring, older ones the output already stored in HBM.
template <int WARPS_, uint32_t RING_, int UPL_ = 1>
struct CopyCfg {
    static constexpr int WARPS = WARPS_;
    static constexpr int UPL = UPL_;              // units per lane in a group
    static constexpr uint32_t GU = 32 * UPL_;     // units per group
    static constexpr uint32_t RING = RING_, RMASK = RING_ - 1;
    // a group's tokens start within GMAX bytes: its output (GMAX + 258 at most) and the unflushed
    // window before it (under WIN bytes) stay in the ring while the group is written
    static constexpr uint32_t GMAX = RING_ - WIN - 258 - 64;
    static_assert((RING_ & (RING_ - 1)) == 0 && RING_ >= 4096, "ring size");
    struct CtaSmem {
        uint32_t crc8[8][256];
        uint32_t mulk[4][256];   // x * x^(8 (WIN - 32)) by bytes: moves a column past the other lanes
        uint32_t tok[WARPS_][32 * UPL_];  // the tokens of the warp's current group, in order
        alignas(16) uint8_t ring[WARPS_][RING_];
    };
};

template <class S>
__device__ __forceinline__ uint32_t mulk(const S& s, uint32_t x) {
    return s.mulk[0][x & 255] ^ s.mulk[1][(x >> 8) & 255] ^ s.mulk[2][(x >> 16) & 255] ^ s.mulk[3][x >> 24];
}

// Store output bytes [ws, we) from the ring (byte p at slot p + a) to out, and fold them into this
// lane's CRC column (window kwin; windows are aligned to the end of the member, the first one
// padded by `pad` zero bytes in front).
template <uint32_t RMASK, class S>
__device__ __noinline__ uint32_t flush_window(uint8_t* out, uint32_t a, uint32_t ws, uint32_t we, uint32_t kwin,
                                              uint32_t pad, uint32_t col, const uint8_t* ring, const S& s, bool crc) {
    const int lane = threadIdx.x & 31;
    const uintptr_t o16 = (uintptr_t)out & ~(uintptr_t)15;
    const uintptr_t lo = (uintptr_t)out + ws, hi = (uintptr_t)out + we;
    const uintptr_t A0 = lo & ~(uintptr_t)15;
    const uint32_t nunits = (uint32_t)(((hi + 15) & ~(uintptr_t)15) - A0) >> 4;
    for (uint32_t u = lane; u < nunits; u += 32) {
        const uintptr_t ga = A0 + 16 * (uintptr_t)u;
        const uint32_t sl = (uint32_t)(ga - o16) & RMASK;
        if (ga >= lo && ga + 16 <= hi) {
            *reinterpret_cast<uint4*>(ga) = *reinterpret_cast<const uint4*>(ring + sl);
        } else {
            for (uint32_t k = 0; k < 16; k++)
                if (ga + k >= lo && ga + k < hi) *reinterpret_cast<uint8_t*>(ga + k) = ring[(sl + k) & RMASK];
        }
    }
    if (crc) {
        uint32_t c = mulk(s, col);
        const long long v0 = (long long)kwin * WIN + 32 * lane - (long long)pad;  // position of the column
        uint32_t wv[8];
        if (v0 >= 0) {
            // the column's 32 bytes from 9 aligned ring words (funnel shifts for the byte phase)
            const uint32_t sl = (uint32_t)(v0 + a) & RMASK, w = sl >> 2, sh = (sl & 3u) * 8;
            const uint32_t* rw = reinterpret_cast<const uint32_t*>(ring);
            uint32_t r[9];
#pragma unroll
            for (int k = 0; k < 9; k++) r[k] = rw[(w + k) & (RMASK >> 2)];
#pragma unroll
            for (int k = 0; k < 8; k++) wv[k] = __funnelshift_r(r[k], r[k + 1], sh);
        } else {
            // the first window: zero bytes stand before the member's start
#pragma unroll
            for (int k = 0; k < 8; k++) {
                uint32_t v = 0;
#pragma unroll
                for (int t = 0; t < 4; t++) {
                    const long long r0 = v0 + 4 * k + t;
                    v |= (r0 >= 0 ? (uint32_t)ring[(uint32_t)(r0 + a) & RMASK] : 0u) << (8 * t);
                }
                wv[k] = v;
            }
        }
#pragma unroll
        for (int q = 0; q < 8; q += 2) c = crc_step8(s.crc8, c, wv[q], wv[q + 1]);
        col = c;
    }
    __syncwarp();
    return col;
}

// zlib's CRC32 of the member from the lane columns.
__device__ __noinline__ uint32_t finish_crc(uint32_t col, uint32_t isize) {
    const int lane = threadIdx.x & 31;
    uint32_t v = col;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const int d = 1 << k;
        const uint32_t other = __shfl_down_sync(FULL, v, d);
        if ((lane & (2 * d - 1)) == 0) v = gf_mul(v, kCrc.seg[k]) ^ other;
    }
    v = __shfl_sync(FULL, v, 0);
    return crc_finish(v, isize);
}

template <class C>
__global__ void __launch_bounds__(C::WARPS * 32)
    k_copy(const cb_member_job* __restrict__ jobs, int64_t n_jobs, const int64_t* __restrict__ d_n_jobs,
           uint8_t* out_base, int check_crc, uint32_t* job_status, cb_inflate_summary* summary, uint8_t* ws,
           long long j0, long long j1, int qi) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    typename C::CtaSmem& S = *reinterpret_cast<typename C::CtaSmem*>(smem_raw);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
#pragma unroll
        for (int b = 0; b < 4; b++) S.mulk[b][i] = gf_mul((uint32_t)i << (8 * b), kCrc.k992);
    }
    init_crc8(S.crc8);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint8_t* ring = S.ring[warp];
    uint32_t* tokw = S.tok[warp];
    const uint32_t incl = lane == 31 ? 0xFFFFFFFFu : (2u << lane) - 1u;  // lanes 0..lane
    unsigned long long* queue = reinterpret_cast<unsigned long long*>(ws) + qi;  // this launch's counter
    const uint32_t* per_job = reinterpret_cast<const uint32_t*>(ws + WS_HEAD);
    const uint8_t* arena = ws + arena_offset(n_jobs);
    long long n = n_jobs;
    if (d_n_jobs) n = min((long long)n, (long long)*d_n_jobs);
    n = min(n, j1);  // this launch's jobs: [j0, j1)
    const bool crc = check_crc != 0;

    for (;;) {
        unsigned long long jj = 0;
        if (lane == 0) jj = atomicAdd(queue, 1ull);
        const long long j = j0 + (long long)__shfl_sync(FULL, jj, 0);
        if (j >= n) break;
        if (per_job[4 * j + 1] != CB_OK) continue;  // k_decode reported it
        const cb_member_job job = jobs[j];
        const uint32_t nu = per_job[4 * j];
        const uint16_t* U =
            reinterpret_cast<const uint16_t*>(arena + reinterpret_cast<const unsigned long long*>(per_job)[2 * j + 1]);
        uint8_t* out = out_base + job.out_off;
        const uint32_t a = (uint32_t)((uintptr_t)out & 15);
        const uint32_t isize = job.isize;
        const uint32_t pad = (uint32_t)(-(int32_t)isize) & (WIN - 1);
        uint32_t p = 0, ws_ = 0, we = min((uint32_t)WIN - pad, isize), kwin = 0, col = 0;
        uint32_t st = (nu > isize) ? (uint32_t)CB_ERR_INFLATE : (uint32_t)CB_OK;
        // groups of GU = 32 * UPL units, lane l holding units UPL * l ... UPL * l + UPL - 1 of the group
        constexpr int UPL = C::UPL;
        constexpr uint32_t GU = C::GU;
        uint32_t g = 0;
        uint32_t u[UPL];
#pragma unroll
        for (int h = 0; h < UPL; h++) {
            const uint32_t i = UPL * lane + h;
            u[h] = (i < nu && st == CB_OK) ? (uint32_t)__ldcs(U + i) : 0u;
        }
        while (st == CB_OK && g < nu) {
            // this group: units [g, g + cnt); a match head as the group's last unit waits for the next group
            const uint32_t avail = min(GU, nu - g);
            const uint32_t nl = __shfl_down_sync(FULL, u[0], 1);  // the unit after this lane's last
            const bool head_last = avail == GU && (__shfl_sync(FULL, u[UPL - 1], 31) & 0xC000u) == 0x8000u;
            uint32_t cnt = avail - (head_last ? 1u : 0u);
            uint32_t len[UPL], ex[UPL];
            uint32_t glen;
            auto lengths = [&](uint32_t c) {  // bytes of each unit's token, and where each starts
                uint32_t tot = 0;
#pragma unroll
                for (int h = 0; h < UPL; h++) {
                    const uint32_t x = u[h];
                    len[h] = UPL * lane + h < c ? (!(x & 0x8000u) ? 1u : (x & 0xC000u) == 0x8000u ? ((x >> 6) & 255u) + 3 : 0u)
                                                : 0u;
                    tot += len[h];
                }
                uint32_t e0 = warp_exclusive_scan(tot, glen);
#pragma unroll
                for (int h = 0; h < UPL; h++) {
                    ex[h] = e0;
                    e0 += len[h];
                }
            };
            lengths(cnt);
            if (glen > C::GMAX) {
                // keep the units whose token starts within GMAX bytes (a tail goes with its head); the
                // starts only grow along the units, so the kept units are a prefix
                const uint32_t prev_ex = __shfl_up_sync(FULL, ex[UPL - 1], 1);
                uint32_t kept = 0;
#pragma unroll
                for (int h = 0; h < UPL; h++) {
                    const bool tail = (u[h] & 0xC000u) == 0xC000u;
                    const uint32_t start = tail ? (h > 0 ? ex[h > 0 ? h - 1 : 0] : (lane > 0 ? prev_ex : ex[h])) : ex[h];
                    kept += __popc(__ballot_sync(FULL, UPL * lane + h < cnt && start < C::GMAX));
                }
                cnt = kept;
                lengths(cnt);
            }
            // match heads: the distance from the head and its tail (the next unit; a head that is the
            // last of the units, or not followed by a tail, is an error)
            bool bad = false;
            uint32_t tokv[UPL], myr[UPL], mybit[UPL];
            bool is_tok[UPL];
#pragma unroll
            for (int h = 0; h < UPL; h++) {
                const uint32_t i = UPL * lane + h;
                const uint32_t x = u[h];
                const uint32_t nx = h + 1 < UPL ? u[h + 1 < UPL ? h + 1 : 0] : nl;
                const bool head = i < cnt && (x & 0xC000u) == 0x8000u;
                const uint32_t dist = head ? ((((x & 63u) << 9) | (nx & 511u)) + 1) : 0u;
                bad |= (head && (i + 1 >= cnt || (nx & 0xC000u) != 0xC000u)) || (head && dist > p + ex[h]);
                is_tok[h] = len[h] != 0;
                tokv[h] = head ? (0x80000000u | dist) : (x & 255u);
                // a token starts in round ex >> 5 of the group, at bit ex & 31 of that round's start mask
                myr[h] = is_tok[h] ? ex[h] >> 5 : 0xFFFFFFFFu;
                mybit[h] = 1u << (ex[h] & 31u);
            }
            // the next group's units are loaded while this one is written
            const uint32_t g2 = g + cnt;
            uint32_t u2[UPL];
#pragma unroll
            for (int h = 0; h < UPL; h++) {
                const uint32_t i = g2 + UPL * lane + h;
                u2[h] = i < nu ? (uint32_t)__ldcs(U + i) : 0u;
            }
            if (__any_sync(FULL, bad) || glen > isize - p) {
                st = CB_ERR_INFLATE;
                break;
            }
            // the group's tokens in order (tails are not tokens): literal byte, or 0x80000000 | distance
            {
                uint32_t ord = 0;
                const uint32_t lower = (1u << lane) - 1u;
#pragma unroll
                for (int h = 0; h < UPL; h++) ord += __popc(__ballot_sync(FULL, is_tok[h]) & lower);
#pragma unroll
                for (int h = 0; h < UPL; h++)
                    if (is_tok[h]) tokw[ord++] = tokv[h];
            }
            __syncwarp();
            uint32_t before = 0;  // tokens that start before this round
            uint32_t ri = 0;
#pragma unroll 2
            for (uint32_t r0 = 0; r0 < glen; r0 += 32, ri++) {
                const uint32_t rel = r0 + lane;
                // the token of byte rel: tokens starting in this round set bits of a mask; the byte's
                // token is the last one starting at or before it
                uint32_t mine = 0;
#pragma unroll
                for (int h = 0; h < UPL; h++) mine |= myr[h] == ri ? mybit[h] : 0u;
                const uint32_t sm = __reduce_or_sync(FULL, mine);
                const uint32_t ord = before + __popc(sm & incl) - 1;
                before += __popc(sm);
                const uint32_t t = tokw[ord & (GU - 1)];
                const uint32_t b = p + rel;
                uint32_t val = t & 255u;
                int src = lane;  // the lane of this round holding the byte's source
                if (rel < glen && (t & 0x80000000u)) {
                    const uint32_t x = b - (t & 0x7FFFFFFFu);
                    if (x >= p + r0) src = (int)(x - (p + r0));
                    else if (x + C::RING >= p + r0 + 32) val = ring[(x + a) & C::RMASK];
                    else val = __ldcg(out + x);  // flushed long ago (the ring keeps the last RING - 32 bytes)
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
                if (rel < glen) ring[(b + a) & C::RMASK] = (uint8_t)val;
                __syncwarp();
            }
            __syncwarp();  // the round loop read tokw; the next group writes it
            p += glen;
            while (we > ws_ && p >= we) {
                col = flush_window<C::RMASK>(out, a, ws_, we, kwin, pad, col, ring, S, crc);
                ws_ = we;
                we = min(we + WIN, isize);
                kwin++;
            }
            g = g2;
#pragma unroll
            for (int h = 0; h < UPL; h++) u[h] = u2[h];
        }
        if (st == CB_OK && p != isize) st = CB_ERR_INFLATE;
        if (st == CB_OK && crc && finish_crc(col, isize) != job.crc) st = CB_ERR_CRC;
        if (lane == 0 && st != CB_OK) report(summary, job_status, j, st);
        __syncwarp();
    }
}

__global__ void k_split_init(cb_inflate_summary* summary, unsigned long long* queue) {
    summary->status = CB_OK;
    summary->reserved = 0;
    summary->n_bad = 0;
    summary->first_bad = INT64_MAX;
    for (int q = 0; q < 4; q++) queue[q] = 0;  // decode and copy counters of up to two job ranges
}

__global__ void k_split_finish(cb_inflate_summary* summary) {
    if (summary->first_bad == INT64_MAX) summary->first_bad = -1;
}

}  // namespace split
}  // namespace cb

using namespace cb;

int cb_set_error(cudaError_t e);  // abi.cu

namespace {

constexpr int MAX_DEVICES = 64;

// CTAs per SM of a kernel on the current device, setting its shared memory size once per device.
template <class K>
int occupancy(int (&cache)[MAX_DEVICES], K kernel, int threads, size_t smem) {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= MAX_DEVICES) return -1;
    int& b = cache[d];
    if (b > 0) return b;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int occ = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem);
    if (e != cudaSuccess) return -(int)e;
    b = occ > 0 ? occ : 1;
    return b;
}

int fail_occ(int o) { return cb_set_error(o == -1 ? cudaErrorInvalidDevice : (cudaError_t)(-o)); }

// One launch's jobs: [j0, j1) of the table, and its queue counters (decode at qd, copy at qd + 1).
struct Range {
    long long j0, j1;
    int qd;
};

template <class D>
int launch_decode(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint32_t* job_status,
                  cb_inflate_summary* summary, uint8_t* ws, unsigned long long arena_bytes, Range r, cudaStream_t s) {
    static int cache[MAX_DEVICES];
    const size_t smem = sizeof(typename D::CtaSmem);
    const int o = occupancy(cache, split::k_decode<D>, D::WARPS * 32, smem);
    if (o <= 0) return fail_occ(o);
    long long grid = (long long)cb_device_sm_count() * o;
    const long long by_work = (r.j1 - r.j0 + 32 * D::WARPS - 1) / (32 * D::WARPS);
    if (!d_n_jobs && by_work < grid) grid = by_work;
    split::k_decode<D><<<(unsigned)(grid < 1 ? 1 : grid), D::WARPS * 32, smem, s>>>(
        jobs, n_jobs, d_n_jobs, job_status, summary, ws, arena_bytes, (int)cb_param(CB_PARAM_DECODE_STEPS),
        (uint32_t)cb_param(CB_PARAM_DECODE_PREFETCH), r.j0, r.j1, r.qd);
    return CB_OK;
}

template <class C>
int launch_copy(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint8_t* out_base, int check_crc,
                uint32_t* job_status, cb_inflate_summary* summary, uint8_t* ws, Range r, cudaStream_t s) {
    static int cache[MAX_DEVICES];
    const size_t smem = sizeof(typename C::CtaSmem);
    const int o = occupancy(cache, split::k_copy<C>, C::WARPS * 32, smem);
    if (o <= 0) return fail_occ(o);
    long long grid = (long long)cb_device_sm_count() * o;
    const long long by_work = (r.j1 - r.j0 + C::WARPS - 1) / C::WARPS;
    if (!d_n_jobs && by_work < grid) grid = by_work;
    split::k_copy<C><<<(unsigned)(grid < 1 ? 1 : grid), C::WARPS * 32, smem, s>>>(
        jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, ws, r.j0, r.j1, r.qd + 1);
    return CB_OK;
}

int decode_range(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint32_t* job_status,
                 cb_inflate_summary* summary, uint8_t* ws, unsigned long long arena_bytes, Range r, cudaStream_t s) {
    const int rb = (int)cb_param(CB_PARAM_DECODE_ROOT);
    if (rb == 8)
        return launch_decode<split::DecCfg<8, 6, 1>>(jobs, n_jobs, d_n_jobs, job_status, summary, ws, arena_bytes, r, s);
    if (rb == 7)
        return launch_decode<split::DecCfg<7, 5, 1>>(jobs, n_jobs, d_n_jobs, job_status, summary, ws, arena_bytes, r, s);
    return launch_decode<split::DecCfg<6, 5, 1>>(jobs, n_jobs, d_n_jobs, job_status, summary, ws, arena_bytes, r, s);
}

int copy_range(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint8_t* out_base, int check_crc,
               uint32_t* job_status, cb_inflate_summary* summary, uint8_t* ws, Range r, cudaStream_t s) {
    const int cw = (int)cb_param(CB_PARAM_COPY_WARPS);
    const int units = (int)cb_param(CB_PARAM_COPY_UNITS);
#define CB_COPY(W, R, UPL) \
    launch_copy<split::CopyCfg<W, R, UPL>>(jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, ws, r, s)
    if (cw == 2) return CB_COPY(2, 16384, 1);
    if (cw == 3) return CB_COPY(3, 16384, 1);
    if (cw == 12) return units == 4 ? CB_COPY(12, 8192, 4) : units == 2 ? CB_COPY(12, 8192, 2) : CB_COPY(12, 8192, 1);
    if (cw == 24) return units >= 2 ? CB_COPY(24, 4096, 2) : CB_COPY(24, 4096, 1);
    return units == 4 ? CB_COPY(6, 16384, 4) : units == 2 ? CB_COPY(6, 16384, 2) : CB_COPY(6, 16384, 1);
#undef CB_COPY
}

// Two side streams per device for the pipelined form, and the events that join them to the caller's
// stream; the mutex keeps each call's records and waits together (a wait takes the event's state
// when it is called), so calls from several host threads may share them.
struct Side {
    cudaStream_t x = nullptr, y = nullptr;
    cudaEvent_t start = nullptr, done_x = nullptr, done_y = nullptr;
    bool ready = false;
};
Side g_side[MAX_DEVICES];
std::mutex g_side_mu;

int side_for(int dev, Side*& out) {
    Side& sd = g_side[dev];
    if (!sd.ready) {
        cudaError_t e = cudaStreamCreateWithFlags(&sd.x, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sd.y, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sd.start, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sd.done_x, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sd.done_y, cudaEventDisableTiming);
        if (e != cudaSuccess) return cb_set_error(e);
        sd.ready = true;
    }
    out = &sd;
    return CB_OK;
}

}  // namespace

extern "C" size_t cb_inflate_split_workspace_bytes(int64_t n_jobs, int64_t out_bytes) {
    if (n_jobs < 0 || out_bytes < 0) return 0;
    return split::arena_offset(n_jobs) + 2 * (size_t)out_bytes + 16 * (size_t)n_jobs + 16;
}

extern "C" int cb_inflate_split(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint8_t* out_base,
                                int check_crc, uint32_t* job_status, cb_inflate_summary* summary, void* workspace,
                                size_t workspace_bytes, void* stream) {
    if (!summary || !workspace || n_jobs < 0 || workspace_bytes < split::arena_offset(n_jobs) + 16) return CB_ERR_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint8_t* ws = reinterpret_cast<uint8_t*>(workspace);
    const unsigned long long arena_bytes = workspace_bytes - split::arena_offset(n_jobs);
    split::k_split_init<<<1, 1, 0, s>>>(summary, reinterpret_cast<unsigned long long*>(ws));
    if (n_jobs > 0) {
        split::k_slots<<<1, split::SLOT_NT, 0, s>>>(jobs, n_jobs, d_n_jobs, ws);
        // Pipelined: the jobs in two ranges, each decoded and then copied on its own stream, so that
        // the second range's decode and the first range's copy take the GPU while the other decode
        // runs out of members (one member per lane leaves lanes idle at its end).  Only with the job
        // count known on the host.
        const long long pipe = cb_param(CB_PARAM_DECODE_PIPELINE);
        const bool two = !d_n_jobs && n_jobs >= 2 && (pipe == 2 || (pipe == 1 && n_jobs >= 65536));
        int rc = CB_OK;
        if (!two) {
            const Range all{0, n_jobs, 0};
            rc = decode_range(jobs, n_jobs, d_n_jobs, job_status, summary, ws, arena_bytes, all, s);
            if (rc == CB_OK) rc = copy_range(jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, ws, all, s);
            if (rc != CB_OK) return rc;
        } else {
            int dev = 0;
            cudaError_t e = cudaGetDevice(&dev);
            if (e != cudaSuccess) return cb_set_error(e);
            if (dev < 0 || dev >= MAX_DEVICES) return CB_ERR_ARG;
            std::lock_guard<std::mutex> lock(g_side_mu);
            Side* sd = nullptr;
            if ((rc = side_for(dev, sd)) != CB_OK) return rc;
            const long long cut = n_jobs - n_jobs / 4;  // three quarters first
            const Range ra{0, cut, 0}, rb{cut, n_jobs, 2};
            e = cudaEventRecord(sd->start, s);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(sd->x, sd->start, 0);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(sd->y, sd->start, 0);
            if (e != cudaSuccess) return cb_set_error(e);
            rc = decode_range(jobs, n_jobs, d_n_jobs, job_status, summary, ws, arena_bytes, ra, sd->x);
            if (rc == CB_OK) rc = decode_range(jobs, n_jobs, d_n_jobs, job_status, summary, ws, arena_bytes, rb, sd->y);
            if (rc == CB_OK)
                rc = copy_range(jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, ws, ra, sd->x);
            if (rc == CB_OK)
                rc = copy_range(jobs, n_jobs, d_n_jobs, out_base, check_crc, job_status, summary, ws, rb, sd->y);
            // join both side streams back to the caller's stream whatever happened above
            e = cudaEventRecord(sd->done_x, sd->x);
            if (e == cudaSuccess) e = cudaEventRecord(sd->done_y, sd->y);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, sd->done_x, 0);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, sd->done_y, 0);
            if (rc != CB_OK) return rc;
            if (e != cudaSuccess) return cb_set_error(e);
        }
    }
    split::k_split_finish<<<1, 1, 0, s>>>(summary);
    return cb_set_error(cudaGetLastError());
}
