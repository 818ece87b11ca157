// BGZF member scan on B200: replaces bgzf_candidates, bgzf_sizes, the chain and the checks of
// _inflate_blocks (src/cubam/_kernels.py:69-89, src/cubam/_kernels.py:662-702,
// src/cubam/bgzf.py:542-586).
//
//  1. k_scan_count: a warp per 4 KB tile; each lane loads its eight 16-byte chunks with 128-bit
//     loads, then __vcmpeq4 finds 0x1f bytes (about 1 in 256 in compressed data) and only those
//     offsets get the full header test.  The count of every tile goes to the workspace.
//  2. k_scan_tiles: one block turns the tile counts into tile offsets (prefix sum; each warp
//     takes a contiguous segment, read coalesced with eight loads per lane in flight).
//  3. k_scan_write: tiles with candidates are tested again and their offsets written in order
//     (block prefix sum of the per-thread counts); no sort is needed.
//  4. k_fin_sums, k_scan_finish, k_fin_jobs: the chain from offset 0 (all candidates in the usual
//     case, checked and summed per block of candidates by a grid; otherwise a walk in one block),
//     the reference's checks in the reference's order, and the inflate jobs of the non-empty members
//     with their output offsets (prefix sum of ISIZE), written by a grid.

#include <atomic>

#include "common.cuh"

namespace cb {
namespace scan {

constexpr int NT = 256;
constexpr int FIN_NT = 1024;
constexpr long long MAX_ISIZE = 1 << 16;

struct Ws {
    uint32_t* tile_count;
    int64_t* tile_off;
    int64_t* cand;
    uint8_t* keep;
    int64_t* meta;  // [0] candidates, [1] status
    long long ntiles, cap;
};

__host__ __device__ inline long long n_tiles(const uint8_t* buf, long long n) {
    uintptr_t base = (uintptr_t)buf & ~(uintptr_t)15;
    long long chunks = (long long)(((uintptr_t)buf + n + 15 - base) >> 4);
    return (chunks + NT - 1) / NT + 1;
}

__host__ __device__ inline long long cand_cap(long long n) { return n / 28 + 1024; }

__host__ __device__ inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

__host__ __device__ inline Ws carve(void* ws, const uint8_t* buf, long long n) {
    Ws w;
    w.ntiles = n_tiles(buf, n);
    w.cap = cand_cap(n);
    uint8_t* p = reinterpret_cast<uint8_t*>(ws);
    w.meta = reinterpret_cast<int64_t*>(p);
    p += 256;
    w.tile_count = reinterpret_cast<uint32_t*>(p);
    p += align256(w.ntiles * 4);
    w.tile_off = reinterpret_cast<int64_t*>(p);
    p += align256(w.ntiles * 8);
    w.cand = reinterpret_cast<int64_t*>(p);
    p += align256(w.cap * 8);
    w.keep = p;
    return w;
}

__host__ inline size_t ws_bytes(long long n) {
    // worst case alignment of buf shifts the tile count by one
    long long ntiles = (n + 15 + 16) / 16 / NT + 2;
    long long cap = cand_cap(n);
    return 256 + align256(ntiles * 4) + align256(ntiles * 8) + align256(cap * 8) + align256(cap) + 256;
}

__device__ __forceinline__ bool member_at(const uint8_t* b, long long n, long long o) {
    if (o < 0 || o + 18 > n) return false;
    if (b[o] != 31 || b[o + 1] != 139 || b[o + 2] != 8 || b[o + 3] != 4) return false;
    if (b[o + 10] != 6 || b[o + 11] != 0 || b[o + 12] != 66 || b[o + 13] != 67 || b[o + 14] != 2 || b[o + 15] != 0)
        return false;
    long long bs = (long long)ld_u16(b, o + 16) + 1;
    return bs >= 26 && o + bs <= n;
}

// The 16 bytes of chunk c of the aligned view of buf (bytes outside [0, n) read as 0), and the
// offset of its first byte.
__device__ __forceinline__ uint4 chunk_load(const uint8_t* buf, long long n, long long c, long long& start) {
    const uintptr_t base = (uintptr_t)buf & ~(uintptr_t)15;
    const uintptr_t a = base + 16 * (uintptr_t)c;
    start = (long long)(a - (uintptr_t)buf);
    if (start >= 0 && start + 16 <= n) return __ldg(reinterpret_cast<const uint4*>(a));
    uint32_t w[4] = {0, 0, 0, 0};
    if (start < n && start + 16 > 0) {
        for (int k = 0; k < 4; k++) {
            uint32_t x = 0;
            for (int t = 0; t < 4; t++) {
                const long long o = start + 4 * k + t;
                if (o >= 0 && o < n) x |= (uint32_t)buf[o] << (8 * t);
            }
            w[k] = x;
        }
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// Bit mask (bit k = offset start + k) of the members that start in a chunk: __vcmpeq4 finds the
// 0x1f bytes, and only those get the full header test.
__device__ __forceinline__ uint32_t chunk_mask(const uint8_t* buf, long long n, long long start, uint4 v) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    uint32_t mask = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        uint32_t eq = __vcmpeq4(w[k], 0x1f1f1f1fu);
        while (eq) {
            const int t = (__ffs(eq) - 1) >> 3;
            eq &= ~(0xffu << (8 * t));
            const int q = 4 * k + t;  // the byte's place in the chunk
            if (q <= 12) {
                // the next three header bytes (8b 08 04) are in this chunk: test them from the registers
                // first (the chunk as a 128-bit value shifted right by q + 1 bytes), so that most 0x1f
                // bytes need no further load
                const unsigned sh = 8u * (unsigned)(q + 1);  // 8..104
                const unsigned long long lo = (unsigned long long)w[0] | ((unsigned long long)w[1] << 32);
                const unsigned long long hi = (unsigned long long)w[2] | ((unsigned long long)w[3] << 32);
                const unsigned long long x = sh < 64 ? (lo >> sh) | (hi << (64 - sh)) : hi >> (sh - 64);
                if ((x & 0xFFFFFFull) != 0x04088Bull) continue;
            }
            const long long o = start + q;
            if (member_at(buf, n, o)) mask |= 1u << q;
        }
    }
    return mask;
}

__device__ __forceinline__ uint32_t chunk_candidates(const uint8_t* buf, long long n, long long c) {
    long long start;
    const uint4 v = chunk_load(buf, n, c, start);
    return chunk_mask(buf, n, start, v);
}

// A warp per tile (NT chunks): each lane loads its NT / 32 chunks first, then tests them.
__global__ void __launch_bounds__(NT) k_scan_count(const uint8_t* buf, long long n, Ws w) {
    constexpr int PER = NT / 32;
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (NT / 32);
    for (long long t = (long long)blockIdx.x * (NT / 32) + (threadIdx.x >> 5); t < w.ntiles; t += nwarps) {
        uint4 v[PER];
        long long start[PER];
#pragma unroll
        for (int k = 0; k < PER; k++) v[k] = chunk_load(buf, n, t * NT + k * 32 + lane, start[k]);
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k < PER; k++) c += __popc(chunk_mask(buf, n, start[k], v[k]));
        c = __reduce_add_sync(FULL, c);
        if (lane == 0) w.tile_count[t] = c;
    }
}

// Exclusive prefix sum of the tile counts (one block); meta[0] = total, meta[1] = status.  Each warp
// takes a contiguous segment of tiles, read coalesced with eight loads per lane in flight: a first
// pass sums the segment, the warps' sums are scanned, and a second pass writes the offsets.
__global__ void __launch_bounds__(FIN_NT) k_scan_tiles(Ws w, long long too_many) {
    constexpr int NW = FIN_NT / 32, U = 8;
    __shared__ int64_t wbase[NW + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long seg = ((w.ntiles + NW - 1) / NW + 32 * U - 1) / (32 * U) * (32 * U);
    const long long a = min((long long)warp * seg, w.ntiles), b = min(a + seg, w.ntiles);
    int64_t sum = 0;
    for (long long i0 = a; i0 < b; i0 += 32 * U) {
        uint32_t v[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const long long i = i0 + k * 32 + lane;
            v[k] = i < b ? w.tile_count[i] : 0u;
        }
#pragma unroll
        for (int k = 0; k < U; k++) sum += v[k];
    }
    for (int d = 16; d; d >>= 1) sum += __shfl_xor_sync(FULL, sum, d);
    if (lane == 0) wbase[warp] = sum;
    __syncthreads();
    if (warp == 0) {
        const int64_t x = lane < NW ? wbase[lane] : 0;
        int64_t tot;
        const int64_t e = warp_exclusive_scan(x, tot);
        __syncwarp();
        if (lane < NW) wbase[lane] = e;
        if (lane == 0) wbase[NW] = tot;
    }
    __syncthreads();
    int64_t carry = wbase[warp];
    for (long long i0 = a; i0 < b; i0 += 32 * U) {
        uint32_t v[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const long long i = i0 + k * 32 + lane;
            v[k] = i < b ? w.tile_count[i] : 0u;
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            const long long i = i0 + k * 32 + lane;
            int64_t t;
            const int64_t x = warp_exclusive_scan((int64_t)v[k], t);
            if (i < b) w.tile_off[i] = carry + x;
            carry += t;
        }
    }
    if (threadIdx.x == 0) {
        const int64_t tot = wbase[NW];
        w.meta[2] = 0;  // set by the finish when k_fin_jobs is to write the jobs
        w.meta[0] = tot;
        w.meta[1] = tot > too_many ? CB_ERR_TOO_MANY : (tot > w.cap ? CB_ERR_CAPACITY : CB_OK);
    }
}

__global__ void __launch_bounds__(NT) k_scan_write(const uint8_t* buf, long long n, Ws w) {
    __shared__ int64_t sm[33];
    if (w.meta[1] != CB_OK) return;
    for (long long t = blockIdx.x; t < w.ntiles; t += gridDim.x) {
        if (w.tile_count[t] == 0) continue;
        long long c = t * NT + threadIdx.x;
        uint32_t mask = chunk_candidates(buf, n, c);
        int64_t tot;
        int64_t pos = w.tile_off[t] + block_exclusive_scan<NT>((int64_t)__popc(mask), tot, sm);
        long long start = (long long)(((uintptr_t)buf & ~(uintptr_t)15) + 16 * (uintptr_t)c - (uintptr_t)buf);
        while (mask) {
            int k = __ffs(mask) - 1;
            mask &= mask - 1;
            w.cand[pos++] = start + k;
        }
    }
}

__device__ __forceinline__ long long lower_bound(const int64_t* a, long long m, long long x) {
    long long lo = 0, hi = m;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// ---- the finish: chain check, the reference's checks, the job table
//
// The usual case is that every candidate ends where the next one starts.  k_fin_sums (a grid) checks
// that for blocks of FIN_NT candidates and sums each block's jobs and output bytes into the tile
// arrays (free once the candidates are written); k_scan_finish (one block) scans those sums and
// applies the checks, or, when a link breaks, keeps the chain from offset 0 by a walk and writes the
// jobs itself; k_fin_jobs (a grid) writes the jobs of the all-chained case.

// Candidates' block b: sums at tile_off[2b] (jobs) and tile_off[2b + 1] (output bytes); flags at
// tile_count[b]: bit 0 a broken link, bit 1 a bad member (ISIZE too large, or an empty member that is
// not the EOF block's form).
__device__ __forceinline__ void member_fields(const uint8_t* buf, const Ws& w, long long i, long long& c,
                                              long long& bs, int64_t& isz, bool& bad) {
    c = w.cand[i];
    bs = (long long)ld_u16(buf, c + 16) + 1;
    isz = (int64_t)ld_u32(buf, c + bs - 4);
    bad = isz > MAX_ISIZE || (isz == 0 && (bs != 28 || buf[c + 18] != 3 || buf[c + 19] != 0));
}

// Whether the block sums of m candidates fit the tile arrays (2 per block in tile_off); below about
// 17 KB of input they may not, and the finish takes the single-block path.
__device__ __forceinline__ bool fin_sums_fit(const Ws& w, long long m) {
    return 2 * ((m + FIN_NT - 1) / FIN_NT) <= w.ntiles;
}

__global__ void __launch_bounds__(FIN_NT) k_fin_sums(const uint8_t* buf, Ws w) {
    __shared__ int64_t sm[33];
    __shared__ uint32_t s_flags;
    if (w.meta[1] != CB_OK) return;
    const long long m = w.meta[0];
    if (!fin_sums_fit(w, m)) return;
    const long long nb = (m + FIN_NT - 1) / FIN_NT;
    for (long long b = blockIdx.x; b < nb; b += gridDim.x) {
        if (threadIdx.x == 0) s_flags = 0;
        __syncthreads();
        const long long i = b * FIN_NT + threadIdx.x;
        int64_t is_job = 0, out = 0;
        uint32_t flags = 0;
        if (i < m) {
            long long c, bs;
            int64_t isz;
            bool bad;
            member_fields(buf, w, i, c, bs, isz, bad);
            if (i + 1 < m && c + bs != w.cand[i + 1]) flags |= 1;
            if (bad) flags |= 2;
            is_job = isz > 0 && isz <= MAX_ISIZE;
            out = is_job ? isz : 0;
        }
        if (flags) atomicOr(&s_flags, flags);
        int64_t tj, to;
        block_exclusive_scan<FIN_NT>(is_job, tj, sm);
        block_exclusive_scan<FIN_NT>(out, to, sm);
        if (threadIdx.x == 0) {
            w.tile_off[2 * b] = tj;
            w.tile_off[2 * b + 1] = to;
            w.tile_count[b] = s_flags;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(FIN_NT) k_fin_jobs(const uint8_t* buf, long long out_base, cb_member_job* jobs,
                                                    long long jobs_cap, Ws w) {
    __shared__ int64_t sm[33];
    if (w.meta[1] != CB_OK || w.meta[2] != 1) return;  // not the all-chained case, or already failed
    const long long m = w.meta[0];
    const long long nb = (m + FIN_NT - 1) / FIN_NT;
    for (long long b = blockIdx.x; b < nb; b += gridDim.x) {
        const long long i = b * FIN_NT + threadIdx.x;
        int64_t is_job = 0, out = 0;
        long long c = 0, bs = 0;
        int64_t isz = 0;
        if (i < m) {
            bool bad;
            member_fields(buf, w, i, c, bs, isz, bad);
            is_job = isz > 0 && isz <= MAX_ISIZE;
            out = is_job ? isz : 0;
        }
        int64_t tj, to;
        const int64_t xj = block_exclusive_scan<FIN_NT>(is_job, tj, sm);
        const int64_t xo = block_exclusive_scan<FIN_NT>(out, to, sm);
        if (is_job) {
            const long long k = w.tile_off[2 * b] + xj;
            if (k < jobs_cap) {
                cb_member_job j;
                j.in = buf + c + 18;
                j.out_off = out_base + w.tile_off[2 * b + 1] + xo;
                j.in_len = (uint32_t)(bs - 26);
                j.isize = (uint32_t)isz;
                j.crc = ld_u32(buf, c + bs - 8);
                j.reserved = 0;
                jobs[k] = j;
            }
        }
    }
}

__global__ void __launch_bounds__(FIN_NT) k_scan_finish(const uint8_t* buf, long long n, int eof, long long out_base,
                                                       cb_member_job* jobs, long long jobs_cap,
                                                       cb_scan_summary* summary, Ws w) {
    __shared__ int64_t sm[33];
    __shared__ int s_breaks;
    __shared__ long long s_last;
    const long long m = w.meta[0];
    int status = (int)w.meta[1];
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_breaks = 0;
        s_last = 0;  // raised with an unsigned atomicMax below; candidate 0 is always kept
        summary->n_members = 0;
        summary->n_jobs = 0;
        summary->used = 0;
        summary->total_out = 0;
        summary->n_candidates = m;
        summary->chained = 1;
    }
    __syncthreads();
    if (status == CB_OK && m == 0 && eof && n > 0) status = CB_ERR_TRUNCATED;
    if (status == CB_OK && m > 0 && w.cand[0] != 0) status = CB_ERR_NO_CHAIN;
    if (status != CB_OK || m == 0) {
        if (tid == 0) summary->status = status;
        return;
    }
    // does every candidate end where the next starts?  From the block flags of k_fin_sums, or (chunks
    // too small for its sums to fit the tile arrays) by this block
    const long long nb = (m + FIN_NT - 1) / FIN_NT;
    const bool sums = fin_sums_fit(w, m);
    uint32_t local = 0;
    if (sums) {
        for (long long b = tid; b < nb; b += FIN_NT) local |= w.tile_count[b];
    } else {
        for (long long i = tid; i + 1 < m; i += FIN_NT) {
            const long long c = w.cand[i];
            if (c + (long long)ld_u16(buf, c + 16) + 1 != w.cand[i + 1]) local |= 1;
        }
    }
    if (local & 1) atomicOr(&s_breaks, 1);
    __syncthreads();
    if (sums && s_breaks == 0) {
        // all chained: scan the block sums into block bases (k_fin_jobs writes the jobs)
        int64_t cj = 0, co = 0;
        for (long long b0 = 0; b0 < nb; b0 += FIN_NT) {
            const long long b = b0 + tid;
            const int64_t vj = b < nb ? w.tile_off[2 * b] : 0, vo = b < nb ? w.tile_off[2 * b + 1] : 0;
            int64_t tj, to;
            const int64_t xj = block_exclusive_scan<FIN_NT>(vj, tj, sm);
            const int64_t xo = block_exclusive_scan<FIN_NT>(vo, to, sm);
            if (b < nb) {
                w.tile_off[2 * b] = cj + xj;
                w.tile_off[2 * b + 1] = co + xo;
            }
            cj += tj;
            co += to;
        }
        if (tid == 0) {
            const long long c = w.cand[m - 1];
            const long long used = c + (long long)ld_u16(buf, c + 16) + 1;
            int st = CB_OK;
            if (eof && used != n) st = CB_ERR_TRUNCATED;
            else if (local & 2) st = CB_ERR_CORRUPT_BLOCK;
            else if (cj > jobs_cap) st = CB_ERR_CAPACITY;
            summary->status = st;
            if (st != CB_ERR_TRUNCATED) {
                summary->n_members = m;
                summary->n_jobs = cj;
                summary->used = used;
                summary->total_out = co;
                w.meta[2] = 1;  // k_fin_jobs writes the jobs (those below jobs_cap)
            }
        }
        return;
    }
    if (s_breaks) {
        for (long long i = tid; i < m; i += FIN_NT) w.keep[i] = 0;
        __syncthreads();
        if (tid == 0) {
            long long i = 0;
            for (;;) {
                w.keep[i] = 1;
                long long c = w.cand[i];
                long long nx = c + (long long)ld_u16(buf, c + 16) + 1;
                long long j = lower_bound(w.cand, m, nx);
                if (j >= m || w.cand[j] != nx) break;
                i = j;
            }
            summary->chained = 0;
        }
        __syncthreads();
    }
    const bool all = s_breaks == 0;
    // last kept member -> used (every candidate is kept on the fast path)
    if (!all) {
        long long mine = -1;
        for (long long i = tid; i < m; i += FIN_NT)
            if (w.keep[i]) mine = i;
        for (int d = 16; d; d >>= 1) {
            const long long y = __shfl_down_sync(FULL, mine, d);
            if (y > mine) mine = y;
        }
        if ((tid & 31) == 0 && mine > 0) atomicMax(reinterpret_cast<unsigned long long*>(&s_last), (unsigned long long)mine);
        __syncthreads();
    }
    const long long last = all ? m - 1 : s_last;
    const long long used = w.cand[last] + (long long)ld_u16(buf, w.cand[last] + 16) + 1;
    if (eof && used != n) {
        if (tid == 0) summary->status = CB_ERR_TRUNCATED;
        return;
    }
    // checks and jobs
    int bad = 0;
    int64_t carry_jobs = 0, carry_out = 0, kept = 0;
    for (long long b = 0; b <= last; b += FIN_NT) {
        long long i = b + tid;
        int64_t is_job = 0, isz = 0;
        long long c = 0, bs = 0;
        if (i <= last && (all || w.keep[i])) {
            c = w.cand[i];
            bs = (long long)ld_u16(buf, c + 16) + 1;
            isz = (int64_t)ld_u32(buf, c + bs - 4);
            kept++;
            if (isz > MAX_ISIZE) bad = 1;
            if (isz == 0 && (bs != 28 || buf[c + 18] != 3 || buf[c + 19] != 0)) bad = 1;
            is_job = isz > 0 && isz <= MAX_ISIZE;
        }
        int64_t tj, to;
        int64_t xj = block_exclusive_scan<FIN_NT>(is_job, tj, sm);
        int64_t xo = block_exclusive_scan<FIN_NT>(is_job ? isz : 0, to, sm);
        if (is_job) {
            long long k = carry_jobs + xj;
            if (k < jobs_cap) {
                cb_member_job j;
                j.in = buf + c + 18;
                j.out_off = out_base + carry_out + xo;
                j.in_len = (uint32_t)(bs - 26);
                j.isize = (uint32_t)isz;
                j.crc = ld_u32(buf, c + bs - 8);
                j.reserved = 0;
                jobs[k] = j;
            }
        }
        carry_jobs += tj;
        carry_out += to;
    }
    if (bad) atomicOr(&s_breaks, 2);
    __syncthreads();
    int64_t tot_kept;
    block_exclusive_scan<FIN_NT>(kept, tot_kept, sm);
    if (tid == 0) {
        int st = (s_breaks & 2) ? CB_ERR_CORRUPT_BLOCK : (carry_jobs > jobs_cap ? CB_ERR_CAPACITY : CB_OK);
        summary->status = st;
        summary->n_members = tot_kept;
        summary->n_jobs = carry_jobs;
        summary->used = used;
        summary->total_out = carry_out;
    }
}

}  // namespace scan
}  // namespace cb

using namespace cb;

int cb_set_error(cudaError_t e);  // abi.cu

extern "C" size_t cb_scan_workspace_bytes(int64_t n) { return scan::ws_bytes(n < 0 ? 0 : n); }

extern "C" int cb_scan_members(const uint8_t* buf, int64_t n, int eof, int64_t out_base_off, cb_member_job* jobs,
                               int64_t cap, cb_scan_summary* summary, void* workspace, size_t workspace_bytes,
                               void* stream) {
    if (n < 0 || !summary || !workspace || (n > 0 && !buf) || cap < 0) return CB_ERR_ARG;
    if (workspace_bytes < scan::ws_bytes(n)) return CB_ERR_CAPACITY;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    scan::Ws w = scan::carve(workspace, buf, n);
    int sms = cb_device_sm_count();
    long long grid = w.ntiles < (long long)sms * 8 ? w.ntiles : (long long)sms * 8;
    if (grid < 1) grid = 1;
    long long cgrid = (w.ntiles + scan::NT / 32 - 1) / (scan::NT / 32);
    if (cgrid > (long long)sms * 16) cgrid = (long long)sms * 16;
    if (cgrid < 1) cgrid = 1;
    scan::k_scan_count<<<(unsigned)cgrid, scan::NT, 0, s>>>(buf, n, w);
    scan::k_scan_tiles<<<1, scan::FIN_NT, 0, s>>>(w, scan::cand_cap(n));
    scan::k_scan_write<<<(unsigned)grid, scan::NT, 0, s>>>(buf, n, w);
    long long fgrid = (long long)sms * 2;
    scan::k_fin_sums<<<(unsigned)fgrid, scan::FIN_NT, 0, s>>>(buf, w);
    scan::k_scan_finish<<<1, scan::FIN_NT, 0, s>>>(buf, n, eof, out_base_off, jobs, cap, summary, w);
    scan::k_fin_jobs<<<(unsigned)fgrid, scan::FIN_NT, 0, s>>>(buf, out_base_off, jobs, cap, w);
    return cb_set_error(cudaGetLastError());
}

// ---------------------------------------------------------------- the scan without allocation
// cb_scan_members with its scratch in a file-scope device array (see the header): the array holds
// the workspace of an input of CB_NOALLOC_SCAN_MAX_BYTES bytes, laid out as scan::carve lays out a
// caller's workspace.

namespace cb {
namespace scan {

constexpr size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr long long NOALLOC_TILES = (CB_NOALLOC_SCAN_MAX_BYTES + 15 + 16) / 16 / NT + 2;
constexpr long long NOALLOC_CAP = CB_NOALLOC_SCAN_MAX_BYTES / 28 + 1024;
constexpr size_t NOALLOC_SCRATCH_BYTES =
    256 + a256(NOALLOC_TILES * 4) + a256(NOALLOC_TILES * 8) + a256(NOALLOC_CAP * 8) + a256(NOALLOC_CAP) + 256;

static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// The array's device address, per device, looked up on the first call on that device.  Atomic, so
// that host threads calling at once on one device agree (each stores the same address).  The address
// belongs to the device's primary context: after cudaDeviceReset it is stale, which the header
// states as unsupported.
static std::atomic<void*> g_noalloc_ptr[64];

}  // namespace scan
}  // namespace cb

int cb_set_error_text(int code, const char* text);  // abi.cu

extern "C" int cb_scan_members_noalloc(const uint8_t* buf, int64_t n, int eof, int64_t out_base_off,
                                       cb_member_job* jobs, int64_t cap, cb_scan_summary* summary, void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n > CB_NOALLOC_SCAN_MAX_BYTES || scan::ws_bytes(n) > scan::NOALLOC_SCRATCH_BYTES)
        return cb_set_error_text(CB_ERR_CAPACITY,
                                 "cb_scan_members_noalloc: input larger than its fixed scratch (16 MiB at most)");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cb_set_error(e);
    if (dev < 0 || dev >= 64) return cb_set_error_text(CB_ERR_ARG, "cb_scan_members_noalloc: device index >= 64");
    void* p = scan::g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!p) {
        e = cudaGetSymbolAddress(&p, scan::g_noalloc_scratch);
        if (e != cudaSuccess) return cb_set_error(e);
        scan::g_noalloc_ptr[dev].store(p, std::memory_order_release);
    }
    return cb_scan_members(buf, n, eof, out_base_off, jobs, cap, summary, p, scan::NOALLOC_SCRATCH_BYTES, stream);
}
