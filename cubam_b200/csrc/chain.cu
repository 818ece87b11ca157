// The record chain of an inflated chunk on B200: replaces record_candidates + record_ends + chain
// (src/cubam/_kernels.py:250-289, src/cubam/_kernels.py:676-702, src/cubam/bam.py:403-418).
//
// cubam tests the record predicate (is_record, src/cubam/_kernels.py:250-278) at every byte offset and
// keeps the chain from offset 0.  Only offsets on that chain matter: the result is the walk from 0 that
// follows block_size while the predicate holds, which is O(records), not O(bytes).  It is walked in
// parallel by tiles of CB_PARAM_CHAIN_TILE bytes (by default 64 KB, less for small chunks):
//
//  1. k_walk: one warp per tile, the tile staged in shared memory 8 KB at a time (coalesced
//     asynchronous 16-byte copies; the window slides on as the walk passes it).  The lanes test 32
//     offsets at a time for the tile's first offset that passes the predicate; one lane follows the
//     block_size links from it through the window up to the first offset past the tile; the lanes
//     test the predicate on each window's records in parallel.  Out: first[t], count[t] (up to the
//     first record that fails), exit[t], whether the walk broke inside the tile, and the records'
//     offsets in the tile (16-bit, relative to it).  Tiles of 64 KB hold about 256 records, so one
//     first-record search serves many links.
//  2. k_check: tile t's walk is the true chain when its first offset is where the previous non-empty
//     tile's walk left (exit); a tile whose candidate is not on the chain (a spurious match of the
//     predicate) makes the chunk take the serial path.  With none (the usual case, none were seen in
//     hundreds of MB of BAM data), the chain is the union of the tile walks up to the first broken one.
//  3. k_count_* : prefix sum of the tile counts (three kernels), then k_emit writes each tile's
//     offsets from its relative ones (no second walk); k_finish writes the summary (records, tail,
//     errors).
//  4. k_serial: the chain walked by one thread, for chunks where the tile walks disagree.

#include <atomic>

#include "common.cuh"

namespace cb {
namespace chain {

constexpr long long T_MIN = 2048;   // smallest tile
constexpr long long T_MAX = 65536;  // largest tile (record offsets are kept as 16 bits from the tile start)
constexpr int NT = 256;
constexpr int WW = 4;               // warps per block of k_walk
constexpr int WIN = 8192;           // bytes of a tile staged at a time (the walk slides the window)
constexpr int HALO = 512;           // bytes staged after the window (headers of records that cross its end)
constexpr int HEAD = 40;            // bytes of a record header the hop loop wants inside the window
constexpr int SCAN = 1024;          // tiles per block of the count scan
constexpr int MIN_RECORD = 37;      // bytes of the shortest record the predicate accepts (block_size >= 33)

// Record offsets one tile can hold (records are at least MIN_RECORD bytes apart).
__host__ __device__ inline long long rel_cap(long long T) { return T / MIN_RECORD + 2; }
// Shared memory of one k_walk warp: the staged window (plus slack for word reads) and the offsets of
// the records that start in it.
constexpr int STAGE_BYTES = ((WIN + HALO + 32 + 15) / 16) * 16;
constexpr int LIST = (WIN + HALO) / MIN_RECORD + 2;
constexpr int WARP_SMEM = STAGE_BYTES + ((LIST * 2 + 15) / 16) * 16;

struct Ws {
    int64_t* first;    // per tile
    int64_t* exit;
    int32_t* count;    // records; bit 31: the walk broke inside the tile
    int64_t* base;     // exclusive prefix of the counts
    int64_t* bsum;     // per scan block
    int64_t* meta;     // [0] inconsistent tile (min) [1] first broken tile (min) [2] any candidate [3] total
    uint16_t* rel;     // per tile: its records' offsets relative to the tile start, rel_cap(T) slots
    long long ntiles, nblocks;
    long long T;       // bytes per tile
    long long rcap;    // rel_cap(T)
};

__host__ __device__ inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

__host__ __device__ inline Ws carve(void* ws, long long n, long long T) {
    Ws w;
    w.T = T;
    w.ntiles = (n + T - 1) / T;
    if (w.ntiles < 1) w.ntiles = 1;
    w.nblocks = (w.ntiles + SCAN - 1) / SCAN;
    uint8_t* p = reinterpret_cast<uint8_t*>(ws);
    w.meta = reinterpret_cast<int64_t*>(p);
    p += 256;
    w.first = reinterpret_cast<int64_t*>(p);
    p += align256(w.ntiles * 8);
    w.exit = reinterpret_cast<int64_t*>(p);
    p += align256(w.ntiles * 8);
    w.count = reinterpret_cast<int32_t*>(p);
    p += align256(w.ntiles * 4);
    w.base = reinterpret_cast<int64_t*>(p);
    p += align256(w.ntiles * 8);
    w.bsum = reinterpret_cast<int64_t*>(p);
    p += align256(w.nblocks * 8);
    w.rcap = rel_cap(T);
    w.rel = reinterpret_cast<uint16_t*>(p);
    return w;
}

__host__ inline size_t ws_bytes_for(long long n, long long T) {
    long long ntiles = (n + T - 1) / T;
    if (ntiles < 1) ntiles = 1;
    long long nblocks = (ntiles + SCAN - 1) / SCAN;
    return 256 + 3 * align256(ntiles * 8) + align256(ntiles * 4) + align256(nblocks * 8) +
           align256(ntiles * rel_cap(T) * 2) + 256;
}

// Workspace for any tile size: the largest over the allowed sizes.
__host__ inline size_t ws_bytes(long long n) {
    size_t m = 0;
    for (long long T = T_MIN; T <= T_MAX; T *= 2) {
        const size_t b = ws_bytes_for(n, T);
        if (b > m) m = b;
    }
    return m;
}

__device__ __forceinline__ int reg2bin(int beg, int end) {
    --end;
    if (beg >> 14 == end >> 14) return 4681 + (beg >> 14);
    if (beg >> 17 == end >> 17) return 585 + (beg >> 17);
    if (beg >> 20 == end >> 20) return 73 + (beg >> 20);
    if (beg >> 23 == end >> 23) return 9 + (beg >> 23);
    if (beg >> 26 == end >> 26) return 1 + (beg >> 26);
    return 0;
}

// The reference's record predicate at offset o (src/cubam/_kernels.py:250-278), on the bytes of
// accessor A (GlobalBytes or StagedBytes with 64-bit offsets I, WindowBytes with 32-bit offsets from
// its window; n is the data's end in the same offsets).
template <class A, class I> __device__ __forceinline__ bool is_record_at(const A& b, I n, I o, int n_ref) {
    if (o < 0 || o + 36 > n) return false;
    const int bs = (int)b.u32(o);
    if (bs < 33 || bs > (1 << 22) || o + 4 + (I)bs > n) return false;
    const int ref = (int)b.u32(o + 4), pos = (int)b.u32(o + 8);
    const int nref = (int)b.u32(o + 24), npos = (int)b.u32(o + 28);
    if (ref < -1 || ref >= n_ref || pos < -1 || nref < -1 || nref >= n_ref || npos < -1) return false;
    const uint32_t w12 = b.u32(o + 12), w16 = b.u32(o + 16), lseq = b.u32(o + 20);
    const uint32_t lrn = w12 & 255, ncig = w16 & 0xffff, flag = w16 >> 16;
    if (lrn < 2 || flag >= 4096 || lseq > (1u << 22)) return false;
    if (32LL + lrn + 4LL * ncig + (lseq + 1) / 2 + lseq > (long long)bs) return false;
    const I nm = o + 36;
    if (b.u8(nm + (I)lrn - 1) != 0) return false;
    // the name's characters (all but its NUL): each in 33..126 and not '@', four at a time while a
    // word holds only name characters, then one at a time (no byte past the name is read)
    uint32_t i = 0;
    for (; i + 4 < lrn; i += 4) {
        const uint32_t x = b.u32(nm + (I)i);
        if (__vcmpltu4(x, 0x21212121u) | __vcmpgtu4(x, 0x7E7E7E7Eu) | __vcmpeq4(x, 0x40404040u)) return false;
    }
    for (; i + 1 < lrn; i++) {
        const uint32_t c = b.u8(nm + (I)i);
        if (c < 33 || c > 126 || c == '@') return false;
    }
    const I cg = nm + (I)lrn;
    long long rlen = 0;
    for (uint32_t q = 0; q < ncig; q++) {
        const uint32_t v = b.u32(cg + 4 * (I)q), op = v & 15;
        if (op > 8) return false;
        if (op == 0 || op == 2 || op == 3 || op == 7 || op == 8) rlen += v >> 4;
    }
    if (pos >= 0) {
        const int end = pos + (int)(rlen > 0 ? rlen : 1);
        if ((w12 >> 16) != (uint32_t)reg2bin(pos, end)) return false;
    }
    return true;
}

__device__ __forceinline__ bool is_record(const uint8_t* b, long long n, long long o, int n_ref) {
    return is_record_at<GlobalBytes, long long>(GlobalBytes{b}, n, o, n_ref);
}

__global__ void k_init(Ws w) {
    w.meta[0] = INT64_MAX;
    w.meta[1] = INT64_MAX;
    w.meta[2] = 0;
    w.meta[3] = 0;
}

// A warp per tile, the tile's bytes staged a window at a time.
__global__ void __launch_bounds__(WW * 32) k_walk(const uint8_t* __restrict__ b, long long n, int n_ref, Ws w) {
    extern __shared__ uint4 walk_mem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint4* st = walk_mem + (size_t)warp * (WARP_SMEM / 16);
    uint16_t* list = reinterpret_cast<uint16_t*>(reinterpret_cast<uint8_t*>(st) + STAGE_BYTES);
    const uint8_t* sb = reinterpret_cast<const uint8_t*>(st);
    for (long long t = (long long)blockIdx.x * WW + warp; t < w.ntiles; t += (long long)gridDim.x * WW) {
        const long long T = w.T, ts = t * T, te = min(ts + T, n);
        long long hi = min(ts + WIN + HALO, n);
        long long r0 = stage_bytes(b, ts, hi, st);
        // the tile's first offset that passes the predicate, 32 offsets at a time (the window slides
        // on when the search passes it)
        long long c = -1;
        for (long long base = ts; base < te; base += 32) {
            if (base + 32 + HEAD > hi && hi < n) {
                __syncwarp();
                hi = min(base + WIN + HALO, n);
                r0 = stage_bytes(b, base, hi, st);
            }
            // the window's bytes by 32-bit offsets from r0 (the data's end past 2^30 is never near)
            const WindowBytes d{b + r0, sb, (int)(hi - r0)};
            const int nr = (int)min(n - r0, (long long)(1 << 30));
            const long long o = base + lane;
            bool ok = false;
            if (o < te && o + 4 <= n) {
                const int x = (int)(o - r0);
                const uint32_t bs = d.u32(x);
                if (bs - 33u <= (1u << 22) - 33u) ok = is_record_at(d, nr, x, n_ref);
            }
            const unsigned m = __ballot_sync(FULL, ok);
            if (m) {
                c = base + __ffs(m) - 1;
                break;
            }
        }
        int cnt = 0;
        bool broken = false;
        long long exit = -1;
        if (c >= 0) {
            long long o = c;
            for (;;) {
                if (o + HEAD > hi && hi < n) {  // the next header is past the window: slide it on
                    __syncwarp();
                    hi = min(o + WIN + HALO, n);
                    r0 = stage_bytes(b, o, hi, st);
                }
                // one lane follows the links while their headers are in the window; a link that cannot
                // be a record ends the list (the predicate fails there below)
                int m = 0;
                bool stop = false;
                if (lane == 0) {
                    // in 32-bit offsets from the window start r0: x while x <= xmax (before the tile's
                    // end, and the header inside the window unless the window reaches the data's end)
                    const int wlen = (int)(hi - r0);
                    const int xmax = (int)(min(te - 1, hi >= n ? te - 1 : hi - HEAD) - r0);
                    const int nr = (int)min(n - r0, (long long)(1 << 30));  // the data's end (past 2^30: never near)
                    const int base = (int)(r0 - ts);
                    int x = (int)(o - r0);
                    while (x <= xmax) {
                        list[m++] = (uint16_t)(x + base);
                        if (x + 4 > wlen) {  // at the data's end: not a record
                            stop = true;
                            break;
                        }
                        const uint32_t* wd = reinterpret_cast<const uint32_t*>(sb + (x & ~3));
                        const uint32_t bs = __funnelshift_r(wd[0], wd[1], (unsigned)(x & 3) * 8);
                        if (bs - 33u > (1u << 22) - 33u || x + 36 > nr || x + 4 + (int)bs > nr) {
                            stop = true;
                            break;
                        }
                        x += 4 + (int)bs;
                    }
                    o = r0 + x;
                }
                m = __shfl_sync(FULL, m, 0);
                o = __shfl_sync(FULL, o, 0);
                stop = __shfl_sync(FULL, (int)stop, 0) != 0;
                __syncwarp();
                // the predicate on the listed records, in parallel: the count ends at the first failure
                const WindowBytes d{b + r0, sb, (int)(hi - r0)};
                const int nr = (int)min(n - r0, (long long)(1 << 30));
                const int xt = (int)(ts - r0);  // the tile start from the window start (may be negative)
                int f = m;
                for (int j0 = 0; j0 < m; j0 += 32) {
                    const int j = j0 + lane;
                    const bool ok = j >= m || is_record_at(d, nr, xt + (int)list[j], n_ref);
                    const unsigned bad = __ballot_sync(FULL, !ok);
                    if (bad) {
                        f = j0 + __ffs(bad) - 1;
                        break;
                    }
                }
                if (stop && f == m) f = m - 1;  // a link that fails its checks fails the predicate too
                for (int j = lane; j < f; j += 32) w.rel[t * w.rcap + cnt + j] = list[j];
                cnt += f;
                __syncwarp();
                if (f < m) {
                    broken = true;
                    exit = ts + list[f];
                    break;
                }
                if (o >= te) {
                    exit = o;
                    break;
                }
            }
        }
        if (lane == 0) {
            // one flag for the whole chunk: read it first, so that the tiles do not all queue on one
            // address
            if (c >= 0 && *reinterpret_cast<volatile int64_t*>(&w.meta[2]) == 0)
                atomicOr(reinterpret_cast<unsigned long long*>(&w.meta[2]), 1ull);
            if (broken) atomicMin(reinterpret_cast<long long*>(&w.meta[1]), t);
            w.first[t] = c;
            w.exit[t] = exit;
            w.count[t] = cnt | (broken ? (int)0x80000000 : 0);
        }
        __syncwarp();
    }
}

// Is each non-empty tile entered by the chain at its first candidate?
__global__ void __launch_bounds__(NT) k_check(Ws w) {
    const long long end = w.meta[1];  // the chain ends in this tile (if any)
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < w.ntiles;
         t += (long long)gridDim.x * blockDim.x) {
        const long long f = w.first[t];
        if (f < 0 || t > end) continue;
        long long entry = 0;
        for (long long u = t - 1; u >= 0; u--) {
            if (w.first[u] >= 0) {
                entry = w.exit[u];
                break;
            }
        }
        if (entry != f) atomicMin(reinterpret_cast<long long*>(&w.meta[0]), t);
    }
}

// Prefix sum of the tile counts (tiles after the end of the chain count 0).
__global__ void __launch_bounds__(SCAN) k_count_blocks(Ws w) {
    __shared__ int64_t sm[33];
    const long long end = w.meta[1];
    const long long t = (long long)blockIdx.x * SCAN + threadIdx.x;
    int64_t v = (t < w.ntiles && t <= end) ? (int64_t)(w.count[t] & 0x7fffffff) : 0;
    int64_t tot;
    const int64_t x = block_exclusive_scan<SCAN>(v, tot, sm);
    if (t < w.ntiles) w.base[t] = x;
    if (threadIdx.x == 0) w.bsum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN) k_count_top(Ws w) {
    __shared__ int64_t sm[33];
    int64_t carry = 0;
    for (long long b0 = 0; b0 < w.nblocks; b0 += SCAN) {
        const long long i = b0 + threadIdx.x;
        const int64_t v = i < w.nblocks ? w.bsum[i] : 0;
        int64_t tot;
        const int64_t x = block_exclusive_scan<SCAN>(v, tot, sm);
        if (i < w.nblocks) w.bsum[i] = carry + x;
        carry += tot;
    }
    if (threadIdx.x == 0) w.meta[3] = carry;
}

__global__ void __launch_bounds__(SCAN) k_count_add(Ws w) {
    const long long t = (long long)blockIdx.x * SCAN + threadIdx.x;
    if (t < w.ntiles) w.base[t] += w.bsum[blockIdx.x];
}

// Each tile's offsets, from its relative ones, at its place in the chain (a warp per tile).
__global__ void __launch_bounds__(NT) k_emit(Ws w, int64_t* out, long long cap) {
    if (w.meta[0] != INT64_MAX || w.meta[3] > cap) return;
    const long long end = w.meta[1];
    if (w.first[0] != 0) return;
    const int lane = threadIdx.x & 31;
    for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < w.ntiles;
         t += ((long long)gridDim.x * blockDim.x) >> 5) {
        if (t > end) break;
        const int cnt = w.count[t] & 0x7fffffff;
        const long long k = w.base[t], ts = t * w.T;
        const uint16_t* r = w.rel + t * w.rcap;
        for (int j = lane; j < cnt; j += 32) out[k + j] = ts + r[j];
    }
}

// The chain walked by one thread (tiles that disagree).
__global__ void k_serial(const uint8_t* b, long long n, int n_ref, Ws w, int64_t* out, long long cap,
                         cb_chain_summary* summary) {
    if (w.meta[0] == INT64_MAX || w.first[0] != 0) return;
    long long o = 0, k = 0;
    while (is_record(b, n, o, n_ref)) {
        if (k < cap) out[k] = o;
        k++;
        o += 4 + (long long)ld_u32(b, o);
    }
    summary->n_records = k;
    summary->tail = o;
    summary->n_candidates = -1;
    summary->chained = 0;
    summary->status = k > cap ? CB_ERR_CAPACITY : CB_OK;
}

__global__ void k_finish(long long n, Ws w, long long cap, cb_chain_summary* summary) {
    if (n == 0 || w.meta[2] == 0) {  // no record candidate anywhere: nothing on the chain, carry all
        summary->n_records = 0;
        summary->tail = 0;
        summary->n_candidates = 0;
        summary->chained = 1;
        summary->status = CB_OK;
        return;
    }
    if (w.first[0] != 0) {  // offset 0 is not a record while another offset is
        summary->n_records = 0;
        summary->tail = 0;
        summary->n_candidates = -1;
        summary->chained = 1;
        summary->status = CB_ERR_NO_CHAIN;
        return;
    }
    if (w.meta[0] != INT64_MAX) return;  // k_serial writes the summary
    const long long end = w.meta[1];
    long long last = end;
    if (last == INT64_MAX) {  // the chain runs to the end of the data: its last non-empty tile
        last = w.ntiles - 1;
        while (last > 0 && w.first[last] < 0) last--;
    }
    summary->n_records = w.meta[3];
    summary->tail = w.exit[last];
    summary->n_candidates = -1;
    summary->chained = 1;
    summary->status = w.meta[3] > cap ? CB_ERR_CAPACITY : CB_OK;
}

// The first offset below `limit` where a record passes the predicate and the next `hops` records
// (following block_size) pass it too, or the data ends on the way (a record that runs past the end is
// taken as the start of an incomplete one): the speculative start of a shard's first record.
__global__ void __launch_bounds__(NT) k_first(const uint8_t* b, long long n, int n_ref, long long limit, int hops,
                                              unsigned long long* best) {
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < limit;
         o += (long long)gridDim.x * blockDim.x) {
        if ((unsigned long long)o >= *(volatile unsigned long long*)best) break;
        if (o + 4 > n) break;
        const uint32_t bs = ld_u32(b, o);
        if (bs - 33u > (1u << 22) - 33u) continue;
        if (!is_record(b, n, o, n_ref)) continue;
        long long q = o + 4 + (long long)bs;
        bool ok = true;
        for (int h = 0; h < hops && q + 4 <= n; h++) {
            const uint32_t bq = ld_u32(b, q);
            if (q + 4 + (long long)bq > n) {  // runs past the end: an incomplete record, if plausible
                ok = bq >= 33u && bq <= (1u << 22);
                break;
            }
            if (!is_record(b, n, q, n_ref)) {
                ok = false;
                break;
            }
            q += 4 + (long long)bq;
        }
        if (ok) atomicMin(best, (unsigned long long)o);
    }
}

__global__ void k_first_init(unsigned long long* best) { *best = ~0ull; }

}  // namespace chain
}  // namespace cb

using namespace cb;

int cb_set_error(cudaError_t e);  // abi.cu

extern "C" size_t cb_record_chain_workspace_bytes(int64_t n) { return chain::ws_bytes(n < 0 ? 0 : n); }

extern "C" int cb_record_chain(const uint8_t* data, int64_t n, int32_t n_ref, int64_t* offsets, int64_t cap,
                               cb_chain_summary* summary, void* workspace, size_t workspace_bytes, void* stream) {
    if (n < 0 || !summary || !workspace || (n > 0 && (!data || !offsets)) || cap < 0) return CB_ERR_ARG;
    if (workspace_bytes < chain::ws_bytes(n)) return CB_ERR_CAPACITY;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    long long tile = cb_param(CB_PARAM_CHAIN_TILE);
    const long long sms = cb_device_sm_count();
    if (tile == 0) {
        // 64 KB tiles (about 256 records: one first-record search per tile), smaller ones for chunks
        // too small to give 16 tiles per SM
        tile = chain::T_MAX;
        while (tile > chain::T_MIN && n / tile < sms * 16) tile /= 2;
    }
    if (tile < chain::T_MIN || tile > chain::T_MAX || (tile & (tile - 1))) return CB_ERR_ARG;
    chain::Ws w = chain::carve(workspace, n, tile);
    const size_t smem = (size_t)chain::WW * chain::WARP_SMEM;
    {
        static std::atomic<bool> attr_set[64];
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64 || !attr_set[dev].load(std::memory_order_acquire)) {
            const cudaError_t e = cudaFuncSetAttribute(chain::k_walk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)smem);
            if (e != cudaSuccess) return cb_set_error(e);
            if (dev >= 0 && dev < 64) attr_set[dev].store(true, std::memory_order_release);
        }
    }
    long long grid = (w.ntiles + chain::NT - 1) / chain::NT;
    if (grid > sms * 16) grid = sms * 16;
    if (grid < 1) grid = 1;
    long long wgrid = (w.ntiles + chain::WW - 1) / chain::WW;
    if (wgrid > sms * 32) wgrid = sms * 32;
    if (wgrid < 1) wgrid = 1;
    long long egrid = (w.ntiles + chain::NT / 32 - 1) / (chain::NT / 32);
    if (egrid > sms * 16) egrid = sms * 16;
    if (egrid < 1) egrid = 1;
    chain::k_init<<<1, 1, 0, s>>>(w);
    if (n > 0) {
        chain::k_walk<<<(unsigned)wgrid, chain::WW * 32, smem, s>>>(data, n, n_ref, w);
        chain::k_check<<<(unsigned)grid, chain::NT, 0, s>>>(w);
        chain::k_count_blocks<<<(unsigned)w.nblocks, chain::SCAN, 0, s>>>(w);
        chain::k_count_top<<<1, chain::SCAN, 0, s>>>(w);
        chain::k_count_add<<<(unsigned)w.nblocks, chain::SCAN, 0, s>>>(w);
        chain::k_emit<<<(unsigned)egrid, chain::NT, 0, s>>>(w, offsets, cap);
        chain::k_serial<<<1, 1, 0, s>>>(data, n, n_ref, w, offsets, cap, summary);
    }
    chain::k_finish<<<1, 1, 0, s>>>(n, w, cap, summary);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_first_record(const uint8_t* data, int64_t n, int32_t n_ref, int64_t limit, int32_t hops,
                               int64_t* first, void* stream) {
    if (n < 0 || limit < 0 || hops < 0 || !first || (n > 0 && !data)) return CB_ERR_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned long long* best = reinterpret_cast<unsigned long long*>(first);
    chain::k_first_init<<<1, 1, 0, s>>>(best);
    const long long lim = limit < n ? limit : n;
    if (lim > 0) {
        long long grid = (lim + chain::NT - 1) / chain::NT;
        const long long cap = (long long)cb_device_sm_count() * 8;
        if (grid > cap) grid = cap;
        chain::k_first<<<(unsigned)grid, chain::NT, 0, s>>>(data, n, n_ref, lim, hops, best);
    }
    return cb_set_error(cudaGetLastError());
}
