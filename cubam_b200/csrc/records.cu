// BAM records on B200: the record chain (src/cubam/_kernels.py:250-289, src/cubam/bam.py:403-418),
// the fixed columns (src/cubam/_kernels.py:292-319), the aux tags (src/cubam/_kernels.py:334-388) and
// the on-request decoders (src/cubam/_kernels.py:322-620, src/cubam/bam.py:299-400).
//
// Record chain:
//  1. k_rec_count: every byte offset of the inflated chunk is tested with the reference's record
//     predicate.  Each thread loads 16 bytes with one 128-bit load plus the next 4 bytes of its
//     neighbour, so the block_size window of all 16 offsets is in registers; most offsets fail the
//     33 <= block_size <= 2^22 test there.  Survivors get the full predicate.  Counts per 4 KB tile.
//  2. k_rec_tiles: prefix sum of the tile counts (one block).
//  3. k_rec_write: the candidates, in order, straight into the caller's offset array.
//  4. k_rec_links: does each candidate end where the next starts (grid)?
//  5. k_rec_finish: one block: in the usual case the candidates are the records; otherwise the
//     reference's pointer jumping from offset 0 runs in this block and the chain is compacted in place.

#include "common.cuh"

namespace cb {
namespace rec {

constexpr int NT = 256;
constexpr int TILE = NT * 16;
constexpr int FIN_NT = 1024;

struct Ws {
    uint32_t* tile_count;
    int64_t* tile_off;
    int64_t* meta;     // [0] candidates, [1] status, [2] breaks
    int64_t* jump;     // pointer jumping (slow path)
    int64_t* jump2;
    uint8_t* mark;
    long long ntiles, cap;
};

__host__ __device__ inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

__host__ __device__ inline long long n_tiles(const uint8_t* buf, long long n) {
    uintptr_t base = (uintptr_t)buf & ~(uintptr_t)15;
    long long chunks = (long long)(((uintptr_t)buf + n + 15 - base) >> 4);
    return (chunks + NT - 1) / NT + 1;
}

__host__ __device__ inline long long too_many(long long n) { return n / 32 + 1024; }

__host__ __device__ inline Ws carve(void* ws, const uint8_t* buf, long long n) {
    Ws w;
    w.ntiles = n_tiles(buf, n);
    w.cap = too_many(n);
    uint8_t* p = reinterpret_cast<uint8_t*>(ws);
    w.meta = reinterpret_cast<int64_t*>(p);
    p += 256;
    w.tile_count = reinterpret_cast<uint32_t*>(p);
    p += align256(w.ntiles * 4);
    w.tile_off = reinterpret_cast<int64_t*>(p);
    p += align256(w.ntiles * 8);
    w.jump = reinterpret_cast<int64_t*>(p);
    p += align256((w.cap + 1) * 8);
    w.jump2 = reinterpret_cast<int64_t*>(p);
    p += align256((w.cap + 1) * 8);
    w.mark = p;
    return w;
}

__host__ inline size_t ws_bytes(long long n) {
    long long ntiles = (n + 32) / 16 / NT + 2;
    long long cap = too_many(n);
    return 256 + align256(ntiles * 4) + align256(ntiles * 8) + 2 * align256((cap + 1) * 8) + align256(cap + 1) + 256;
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

__device__ __forceinline__ bool ref_consuming(uint32_t op) {
    return op == 0 || op == 2 || op == 3 || op == 7 || op == 8;  // M D N = X
}

// The reference's record predicate (src/cubam/_kernels.py:250-278), after block_size `bs`
// (read by the caller) passed 33 <= bs <= 2^22.
__device__ bool record_rest(const uint8_t* b, long long n, long long o, int bs, int n_ref) {
    if (o + 36 > n || o + 4 + (long long)bs > n) return false;
    int ref = (int)ld_u32(b, o + 4), pos = (int)ld_u32(b, o + 8);
    int nref = (int)ld_u32(b, o + 24), npos = (int)ld_u32(b, o + 28);
    if (ref < -1 || ref >= n_ref || pos < -1 || nref < -1 || nref >= n_ref || npos < -1) return false;
    uint32_t lrn = b[o + 12], ncig = ld_u16(b, o + 16), flag = ld_u16(b, o + 18), lseq = ld_u32(b, o + 20);
    if (lrn < 2 || flag >= 4096 || lseq > (1u << 22)) return false;
    if (32LL + lrn + 4LL * ncig + (lseq + 1) / 2 + lseq > (long long)bs) return false;
    const long long nm = o + 36;
    if (b[nm + lrn - 1] != 0) return false;
    for (uint32_t i = 0; i + 1 < lrn; i++) {
        uint8_t c = b[nm + i];
        if (c < 33 || c > 126 || c == '@') return false;
    }
    const long long cg = nm + lrn;
    long long rlen = 0;
    for (uint32_t i = 0; i < ncig; i++) {
        uint32_t v = ld_u32(b, cg + 4LL * i), op = v & 15;
        if (op > 8) return false;
        if (ref_consuming(op)) rlen += v >> 4;
    }
    if (pos >= 0) {
        int end = pos + (int)(rlen > 0 ? rlen : 1);
        if (ld_u16(b, o + 14) != (uint32_t)reg2bin(pos, end)) return false;
    }
    return true;
}

__device__ __forceinline__ bool is_record(const uint8_t* b, long long n, long long o, int n_ref) {
    if (o < 0 || o + 36 > n) return false;
    int bs = (int)ld_u32(b, o);
    if (bs < 33 || bs > (1 << 22)) return false;
    return record_rest(b, n, o, bs, n_ref);
}

// Candidate mask of 16-byte chunk c of the aligned view of data.
__device__ __forceinline__ uint32_t chunk_records(const uint8_t* buf, long long n, long long c, int n_ref) {
    uintptr_t base = (uintptr_t)buf & ~(uintptr_t)15;
    uintptr_t a = base + 16 * (uintptr_t)c;
    long long start = (long long)(a - (uintptr_t)buf);
    uint32_t w[5];
    bool inside = start >= 0 && start + 20 <= n;
    if (inside) {
        uint4 v = __ldg(reinterpret_cast<const uint4*>(a));
        w[0] = v.x;
        w[1] = v.y;
        w[2] = v.z;
        w[3] = v.w;
    }
    // the next 4 bytes come from the neighbouring lane's first word when that lane loaded it
    uint32_t nxt = __shfl_down_sync(FULL, w[0], 1);
    const bool nb_inside = __shfl_down_sync(FULL, inside ? 1 : 0, 1) != 0;
    if (!inside) {
        for (int k = 0; k < 5; k++) {
            uint32_t x = 0;
            for (int t = 0; t < 4; t++) {
                long long o = start + 4 * k + t;
                if (o >= 0 && o < n) x |= (uint32_t)buf[o] << (8 * t);
            }
            w[k] = x;
        }
    } else {
        w[4] = ((threadIdx.x & 31) == 31 || !nb_inside) ? ld_u32(buf, start + 16) : nxt;
    }
    if (start >= n || start + 16 <= 0) return 0;
    uint32_t mask = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        uint32_t bs = __funnelshift_r(w[k >> 2], w[(k >> 2) + 1], 8 * (k & 3));
        if (bs - 33u <= (1u << 22) - 33u) {
            long long o = start + k;
            if (o >= 0 && record_rest(buf, n, o, (int)bs, n_ref)) mask |= 1u << k;
        }
    }
    return mask;
}

__global__ void __launch_bounds__(NT) k_rec_count(const uint8_t* buf, long long n, int n_ref, Ws w) {
    __shared__ uint32_t red[NT / 32];
    for (long long t = blockIdx.x; t < w.ntiles; t += gridDim.x) {
        uint32_t c = __popc(chunk_records(buf, n, t * NT + threadIdx.x, n_ref));
        for (int d = 16; d; d >>= 1) c += __shfl_down_sync(FULL, c, d);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t s = 0;
            for (int i = 0; i < NT / 32; i++) s += red[i];
            w.tile_count[t] = s;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(FIN_NT) k_rec_tiles(Ws w, long long cap) {
    __shared__ int64_t sm[33];
    int64_t carry = 0;
    for (long long b = 0; b < w.ntiles; b += FIN_NT) {
        long long i = b + threadIdx.x;
        int64_t v = i < w.ntiles ? (int64_t)w.tile_count[i] : 0;
        int64_t tot;
        int64_t x = block_exclusive_scan<FIN_NT>(v, tot, sm);
        if (i < w.ntiles) w.tile_off[i] = carry + x;
        carry += tot;
    }
    if (threadIdx.x == 0) {
        w.meta[0] = carry;
        w.meta[1] = carry > w.cap ? CB_ERR_TOO_MANY : (carry > cap ? CB_ERR_CAPACITY : CB_OK);
        w.meta[2] = 0;
    }
}

__global__ void __launch_bounds__(NT) k_rec_write(const uint8_t* buf, long long n, int n_ref, int64_t* out, Ws w) {
    __shared__ int64_t sm[33];
    if (w.meta[1] != CB_OK) return;
    for (long long t = blockIdx.x; t < w.ntiles; t += gridDim.x) {
        if (w.tile_count[t] == 0) continue;
        long long c = t * NT + threadIdx.x;
        uint32_t mask = chunk_records(buf, n, c, n_ref);
        int64_t tot;
        int64_t pos = w.tile_off[t] + block_exclusive_scan<NT>((int64_t)__popc(mask), tot, sm);
        long long start = (long long)(((uintptr_t)buf & ~(uintptr_t)15) + 16 * (uintptr_t)c - (uintptr_t)buf);
        while (mask) {
            int k = __ffs(mask) - 1;
            mask &= mask - 1;
            out[pos++] = start + k;
        }
    }
}

__global__ void k_rec_links(const uint8_t* buf, const int64_t* cand, Ws w) {
    if (w.meta[1] != CB_OK) return;
    const long long m = w.meta[0];
    int local = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i + 1 < m; i += (long long)gridDim.x * blockDim.x) {
        long long c = cand[i];
        if (c + 4 + (long long)ld_u32(buf, c) != cand[i + 1]) local = 1;
    }
    if (__any_sync(FULL, local) && (threadIdx.x & 31) == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&w.meta[2]), 1ull);
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

__global__ void __launch_bounds__(FIN_NT) k_rec_finish(const uint8_t* buf, int64_t* cand, cb_chain_summary* summary,
                                                      Ws w) {
    __shared__ int64_t sm[33];
    const int tid = threadIdx.x;
    const long long m = w.meta[0];
    int status = (int)w.meta[1];
    if (status == CB_OK && m > 0 && cand[0] != 0) status = CB_ERR_NO_CHAIN;
    if (status != CB_OK || m == 0) {
        if (tid == 0) {
            summary->status = status;
            summary->n_records = 0;
            summary->tail = 0;
            summary->n_candidates = m;
            summary->chained = 1;
        }
        return;
    }
    if (w.meta[2] == 0) {
        if (tid == 0) {
            long long c = cand[m - 1];
            summary->status = CB_OK;
            summary->n_records = m;
            summary->tail = c + 4 + (long long)ld_u32(buf, c);
            summary->n_candidates = m;
            summary->chained = 1;
        }
        return;
    }
    // pointer jumping from candidate 0 (src/cubam/_kernels.py:692-702): jump[i] is the candidate
    // where candidate i ends, or m; mark[] the candidates reached from 0.
    for (long long i = tid; i <= m; i += FIN_NT) {
        long long j = m;
        if (i < m) {
            long long c = cand[i];
            long long nx = c + 4 + (long long)ld_u32(buf, c);
            if (i + 1 < m && cand[i + 1] == nx) j = i + 1;
            else {
                long long k = lower_bound(cand, m, nx);
                if (k < m && cand[k] == nx) j = k;
            }
        }
        w.jump[i] = j;
        w.mark[i] = i == 0 ? 1 : 0;
    }
    __syncthreads();
    int64_t* jp = w.jump;
    int64_t* jq = w.jump2;
    for (long long span = 1; span < m; span *= 2) {
        for (long long i = tid; i < m; i += FIN_NT)
            if (w.mark[i]) w.mark[jp[i]] = 1;
        __syncthreads();
        for (long long i = tid; i <= m; i += FIN_NT) jq[i] = jp[jp[i]];
        __syncthreads();
        int64_t* t = jp;
        jp = jq;
        jq = t;
    }
    // compact in place (reads of a chunk happen before its writes; writes never pass reads)
    int64_t carry = 0, last = -1;
    for (long long b = 0; b < m; b += FIN_NT) {
        long long i = b + tid;
        int64_t keep = (i < m && w.mark[i]) ? 1 : 0;
        long long v = keep ? cand[i] : 0;
        int64_t tot;
        int64_t x = block_exclusive_scan<FIN_NT>(keep, tot, sm);
        if (keep) {
            cand[carry + x] = v;
            if (carry + x + 1 == carry + tot) last = v;
        }
        carry += tot;
        __syncthreads();
    }
    __shared__ long long s_last;
    if (tid == 0) s_last = 0;  // raised with an unsigned atomicMax; candidate 0 is always on the chain
    __syncthreads();
    if (last >= 0) atomicMax(reinterpret_cast<unsigned long long*>(&s_last), (unsigned long long)last);
    __syncthreads();
    if (tid == 0) {
        summary->status = CB_OK;
        summary->n_records = carry;
        summary->tail = s_last + 4 + (long long)ld_u32(buf, s_last);
        summary->n_candidates = m;
        summary->chained = 0;
    }
}

// ---------------------------------------------------------------- columns

__global__ void k_decode_fixed(const uint8_t* __restrict__ b, const int64_t* __restrict__ off, long long n,
                               int32_t* ref, int32_t* pos, int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref,
                               int32_t* npos, int32_t* tlen, int32_t* l_seq, uint16_t* clip_left,
                               uint16_t* clip_right) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long o = off[i];
        const int p = (int)ld_u32(b, o + 8);
        ref[i] = (int)ld_u32(b, o + 4);
        pos[i] = p;
        mapq[i] = b[o + 13];
        flag[i] = (uint16_t)ld_u16(b, o + 18);
        nref[i] = (int)ld_u32(b, o + 24);
        npos[i] = (int)ld_u32(b, o + 28);
        tlen[i] = (int)ld_u32(b, o + 32);
        l_seq[i] = (int)ld_u32(b, o + 20);
        const uint32_t lrn = b[o + 12], ncig = ld_u16(b, o + 16);
        const long long cg = o + 36 + lrn;
        long long rlen = 0;
        uint32_t cl = 0, cr = 0;
        for (uint32_t k = 0; k < ncig; k++) {
            uint32_t v = ld_u32(b, cg + 4LL * k), op = v & 15, len = v >> 4;
            if (ref_consuming(op)) rlen += len;
            if (op == 4) {
                if (k == 0) cl = len;
                else cr = len;
            }
        }
        end[i] = p + (int)rlen;
        clip_left[i] = (uint16_t)(cl > 65535 ? 65535 : cl);
        clip_right[i] = (uint16_t)(cr > 65535 ? 65535 : cr);
    }
}

struct TagNames {
    uint8_t c[32];
};

// One aux walk per record (src/cubam/_kernels.py:334-388) that fills k tags.
__global__ void k_find_tags(const uint8_t* __restrict__ b, const int64_t* __restrict__ off, long long n, TagNames names,
                            int k, uint8_t* type, int64_t* voff, int32_t* vlen, int64_t* ival) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long o = off[i];
        const long long rec_end = o + 4 + (long long)ld_u32(b, o);
        const uint32_t lrn = b[o + 12], ncig = ld_u16(b, o + 16), lseq = ld_u32(b, o + 20);
        long long a = o + 36 + lrn + 4LL * ncig + (lseq + 1) / 2 + lseq;
        uint32_t found = 0, want = (k >= 32 ? 0xffffffffu : ((1u << k) - 1u));
        for (int t = 0; t < k; t++) {
            type[(long long)t * n + i] = 0;
            voff[(long long)t * n + i] = 0;
            vlen[(long long)t * n + i] = 0;
            ival[(long long)t * n + i] = 0;
        }
        while (a + 3 <= rec_end && found != want) {
            const uint8_t ty = b[a + 2];
            const long long v = a + 3;
            long long nx;
            switch (ty) {
                case 'A': case 'c': case 'C': nx = v + 1; break;
                case 's': case 'S': nx = v + 2; break;
                case 'i': case 'I': case 'f': nx = v + 4; break;
                case 'Z': case 'H':
                    nx = v;
                    while (nx < rec_end && b[nx] != 0) nx++;
                    nx++;
                    break;
                case 'B': {
                    if (v + 5 > rec_end) {
                        nx = -1;
                        break;
                    }
                    const uint8_t sub = b[v];
                    const long long cnt = (long long)ld_u32(b, v + 1);
                    const int sz = (sub == 'c' || sub == 'C') ? 1 : (sub == 's' || sub == 'S') ? 2 : 4;
                    nx = v + 5 + cnt * sz;
                    break;
                }
                default: nx = -1;
            }
            if (nx < 0 || nx > rec_end) {
                // malformed: every tag not found yet gets 255
                for (int t = 0; t < k; t++)
                    if (!(found >> t & 1)) type[(long long)t * n + i] = 255;
                break;
            }
            for (int t = 0; t < k; t++) {
                if ((found >> t & 1) || b[a] != names.c[2 * t] || b[a + 1] != names.c[2 * t + 1]) continue;
                found |= 1u << t;
                long long iv = 0;
                int vl = 0;
                switch (ty) {
                    case 'c': iv = (signed char)b[v]; break;
                    case 'C': case 'A': iv = b[v]; break;
                    case 's': iv = (short)ld_u16(b, v); break;
                    case 'S': iv = ld_u16(b, v); break;
                    case 'i': iv = (int)ld_u32(b, v); break;
                    case 'I': iv = ld_u32(b, v); break;
                    case 'Z': case 'H': vl = (int)(nx - 1 - v); break;
                    case 'B': vl = (int)(nx - v); break;
                    default: break;
                }
                type[(long long)t * n + i] = ty;
                voff[(long long)t * n + i] = v;
                vlen[(long long)t * n + i] = vl;
                ival[(long long)t * n + i] = iv;
            }
            a = nx;
        }
    }
}

constexpr unsigned long long FNV_OFFSET = 1469598103934665603ULL;
constexpr unsigned long long FNV_PRIME = 1099511628211ULL;

__global__ void k_name_hash(const uint8_t* __restrict__ b, const int64_t* __restrict__ off, long long n, uint64_t* h) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long o = off[i];
        const uint32_t lrn = b[o + 12];
        unsigned long long x = FNV_OFFSET;
        for (uint32_t k = 0; k + 1 < lrn; k++) {
            x ^= b[o + 36 + k];
            x *= FNV_PRIME;
        }
        h[i] = x;
    }
}

__global__ void k_hash_spans(const uint8_t* __restrict__ b, const int64_t* __restrict__ voff,
                             const int32_t* __restrict__ vlen, long long n, uint64_t* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int l = vlen[i];
        if (l < 0) {
            out[i] = 0;
            continue;
        }
        unsigned long long x = FNV_OFFSET;
        const long long o = voff[i];
        for (int k = 0; k < l; k++) {
            x ^= b[o + k];
            x *= FNV_PRIME;
        }
        out[i] = x;
    }
}

__global__ void k_pack_acgt(const uint8_t* __restrict__ b, const int64_t* __restrict__ voff,
                            const int32_t* __restrict__ vlen, long long n, uint64_t* out, uint8_t* ok) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long k = voff[i];
        const long long e = voff[i] + vlen[i];
        unsigned long long code = 0, suffix = 0;
        uint32_t nb = 0;
        bool good = vlen[i] > 0;
        for (; good && k < e && b[k] != '-'; k++) {
            const uint8_t c = b[k];
            const uint32_t x = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : c == 'T' ? 3 : 4;
            if (x == 4 || nb == 24) good = false;
            else code |= (unsigned long long)x << (2 * nb++);
        }
        if (good && k < e) {
            k++;
            uint32_t nd = 0;
            for (; k < e; k++, nd++) {
                if (b[k] < '0' || b[k] > '9' || nd == 3) {
                    good = false;
                    break;
                }
                suffix = suffix * 10 + (b[k] - '0');
            }
            if (nd == 0) good = false;
            suffix += 1;
        }
        if (nb == 0) good = false;
        out[i] = good ? (code | ((unsigned long long)nb << 48) | (suffix << 53)) : 0;
        ok[i] = good;
    }
}

__global__ void k_unpack_acgt(const uint64_t* __restrict__ codes, const int64_t* __restrict__ dst_off, long long n,
                              uint8_t* chars) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long c = codes[i];
        const uint32_t nb = (uint32_t)((c >> 48) & 31), suffix = (uint32_t)(c >> 53);
        uint8_t* d = chars + dst_off[i];
        for (uint32_t k = 0; k < nb; k++) d[k] = "ACGT"[(c >> (2 * k)) & 3];
        if (suffix) {
            uint32_t s = suffix - 1, nd = s >= 100 ? 3 : s >= 10 ? 2 : 1;
            d[nb] = '-';
            for (uint32_t k = 0; k < nd; k++) {
                d[nb + nd - k] = '0' + s % 10;
                s /= 10;
            }
        }
    }
}

__global__ void k_aligned_length(const uint8_t* __restrict__ b, const int64_t* __restrict__ off, long long n,
                                 int32_t* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long o = off[i];
        const uint32_t lrn = b[o + 12], ncig = ld_u16(b, o + 16);
        const long long cg = o + 36 + lrn;
        uint32_t s = 0;
        for (uint32_t k = 0; k < ncig; k++) {
            uint32_t v = ld_u32(b, cg + 4LL * k), op = v & 15;
            if (op == 0 || op == 7 || op == 8) s += v >> 4;
        }
        out[i] = (int32_t)s;
    }
}

__global__ void k_blocks(const uint8_t* __restrict__ b, const int64_t* __restrict__ off, long long n, int split_del,
                         int fill, const int64_t* first, int32_t* cnt, int64_t* rec, int32_t* start, int32_t* end) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long o = off[i];
        const uint32_t lrn = b[o + 12], ncig = ld_u16(b, o + 16);
        const long long cg = o + 36 + lrn;
        uint32_t x = ld_u32(b, o + 8), s = x;
        int k = 0;
        const long long w = fill ? first[i] : 0;
        for (uint32_t c = 0; c < ncig; c++) {
            const uint32_t v = ld_u32(b, cg + 4LL * c), op = v & 15, l = v >> 4;
            const bool aligned = op == 0 || op == 7 || op == 8 || (op == 2 && !split_del);
            const bool gap = op == 3 || (op == 2 && split_del);
            if (aligned) {
                x += l;
            } else if (gap) {
                if ((int)x > (int)s) {
                    if (fill) {
                        rec[w + k] = i;
                        start[w + k] = (int)s;
                        end[w + k] = (int)x;
                    }
                    k++;
                }
                x += l;
                s = x;
            }
        }
        if ((int)x > (int)s) {
            if (fill) {
                rec[w + k] = i;
                start[w + k] = (int)s;
                end[w + k] = (int)x;
            }
            k++;
        }
        if (!fill) cnt[i] = k;
    }
}

__global__ void k_base_at(const uint8_t* __restrict__ b, const int64_t* __restrict__ off, const int64_t* __restrict__ rec,
                          const int32_t* __restrict__ refpos, long long m, int8_t* base) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (long long)gridDim.x * blockDim.x) {
        const long long o = off[rec[j]];
        const int target = refpos[j];
        const uint32_t lrn = b[o + 12], ncig = ld_u16(b, o + 16), lseq = ld_u32(b, o + 20);
        const long long cg = o + 36 + lrn, sq = cg + 4LL * ncig;
        long long x = (int)ld_u32(b, o + 8), y = 0;
        int8_t r = -3;
        for (uint32_t k = 0; k < ncig; k++) {
            const uint32_t v = ld_u32(b, cg + 4LL * k), op = v & 15, l = v >> 4;
            if (op == 0 || op == 7 || op == 8) {
                if (target < x + l) {
                    const long long q = y + (target - x);
                    if (target >= x && q < (long long)lseq) {
                        const uint32_t c = (b[sq + q / 2] >> ((q & 1) ? 0 : 4)) & 15;
                        r = c == 1 ? 0 : c == 2 ? 1 : c == 4 ? 2 : c == 8 ? 3 : 4;
                    }
                    break;
                }
                x += l;
                y += l;
            } else if (op == 2 || op == 3) {
                if (target < x + l) {
                    r = target >= x ? (op == 2 ? -1 : -2) : -3;
                    break;
                }
                x += l;
            } else if (op == 1 || op == 4) {
                y += l;
            }
        }
        base[j] = r;
    }
}

// One warp per span; 16-byte copies when source and destination share their alignment.
__global__ void k_copy_spans(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst,
                             const int64_t* __restrict__ src_off, const int64_t* __restrict__ dst_off,
                             const int64_t* __restrict__ size, long long n) {
    const int lane = threadIdx.x & 31;
    for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n;
         w += ((long long)gridDim.x * blockDim.x) >> 5) {
        const uint8_t* s = src + src_off[w];
        uint8_t* d = dst + dst_off[w];
        const long long len = size[w];
        long long i = 0;
        if (((uintptr_t)s & 15) == ((uintptr_t)d & 15) && len >= 64) {
            const long long head = (16 - ((uintptr_t)s & 15)) & 15;
            for (long long k = lane; k < head; k += 32) d[k] = s[k];
            const long long nv = (len - head) >> 4;
            const uint4* sv = reinterpret_cast<const uint4*>(s + head);
            uint4* dv = reinterpret_cast<uint4*>(d + head);
            for (long long k = lane; k < nv; k += 32) dv[k] = sv[k];
            i = head + nv * 16;
        }
        for (long long k = i + lane; k < len; k += 32) d[k] = s[k];
    }
}

__global__ void k_record_sizes(const uint8_t* __restrict__ b, const int64_t* __restrict__ off, long long n, int64_t* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = 4 + (long long)ld_u32(b, off[i]);
}

}  // namespace rec
}  // namespace cb

using namespace cb;

int cb_set_error(cudaError_t e);  // abi.cu

static unsigned grid_for(long long items, int threads) {
    long long g = (items + threads - 1) / threads;
    long long cap = (long long)cb_device_sm_count() * 16;
    if (g > cap) g = cap;
    return (unsigned)(g < 1 ? 1 : g);
}

extern "C" size_t cb_record_chain_workspace_bytes(int64_t n) { return rec::ws_bytes(n < 0 ? 0 : n); }

extern "C" int cb_record_chain(const uint8_t* data, int64_t n, int32_t n_ref, int64_t* offsets, int64_t cap,
                               cb_chain_summary* summary, void* workspace, size_t workspace_bytes, void* stream) {
    if (n < 0 || !summary || !workspace || (n > 0 && (!data || !offsets)) || cap < 0) return CB_ERR_ARG;
    if (workspace_bytes < rec::ws_bytes(n)) return CB_ERR_CAPACITY;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    rec::Ws w = rec::carve(workspace, data, n);
    long long grid = w.ntiles < (long long)cb_device_sm_count() * 8 ? w.ntiles : (long long)cb_device_sm_count() * 8;
    if (grid < 1) grid = 1;
    rec::k_rec_count<<<(unsigned)grid, rec::NT, 0, s>>>(data, n, n_ref, w);
    rec::k_rec_tiles<<<1, rec::FIN_NT, 0, s>>>(w, cap);
    rec::k_rec_write<<<(unsigned)grid, rec::NT, 0, s>>>(data, n, n_ref, offsets, w);
    rec::k_rec_links<<<grid_for(n / 37 + 1, 256), 256, 0, s>>>(data, offsets, w);
    rec::k_rec_finish<<<1, rec::FIN_NT, 0, s>>>(data, offsets, summary, w);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_decode_fixed(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* ref, int32_t* pos,
                               int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos,
                               int32_t* tlen, int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right,
                               void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_decode_fixed<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        data, offsets, n, ref, pos, end, mapq, flag, nref, npos, tlen, l_seq, clip_left, clip_right);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_find_tags(const uint8_t* data, const int64_t* offsets, int64_t n, const char* names, int32_t k,
                            uint8_t* type, int64_t* voff, int32_t* vlen, int64_t* value, void* stream) {
    if (n < 0 || k < 1 || k > 16 || !names) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::TagNames t{};
    for (int i = 0; i < 2 * k; i++) t.c[i] = (uint8_t)names[i];
    rec::k_find_tags<<<grid_for(n, 128), 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(data, offsets, n, t, k,
                                                                                            type, voff, vlen, value);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_name_hash(const uint8_t* data, const int64_t* offsets, int64_t n, uint64_t* out, void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_name_hash<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(data, offsets, n, out);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_hash_spans(const uint8_t* data, const int64_t* voff, const int32_t* vlen, int64_t n, uint64_t* out,
                             void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_hash_spans<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(data, voff, vlen, n, out);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_pack_acgt(const uint8_t* data, const int64_t* voff, const int32_t* vlen, int64_t n, uint64_t* out,
                            uint8_t* ok, void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_pack_acgt<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(data, voff, vlen, n, out,
                                                                                            ok);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_unpack_acgt(const uint64_t* codes, const int64_t* dst_off, int64_t n, uint8_t* chars, void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_unpack_acgt<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(codes, dst_off, n,
                                                                                              chars);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_aligned_length(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* out, void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_aligned_length<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(data, offsets, n,
                                                                                                 out);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_blocks(const uint8_t* data, const int64_t* offsets, int64_t n, int split_del, int fill,
                         const int64_t* first, int32_t* cnt, int64_t* recs, int32_t* start, int32_t* end,
                         void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_blocks<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        data, offsets, n, split_del, fill, first, cnt, recs, start, end);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_base_at(const uint8_t* data, const int64_t* offsets, const int64_t* recs, const int32_t* refpos,
                          int64_t m, int8_t* out, void* stream) {
    if (m < 0) return CB_ERR_ARG;
    if (m == 0) return CB_OK;
    rec::k_base_at<<<grid_for(m, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(data, offsets, recs, refpos,
                                                                                          m, out);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_copy_spans(const uint8_t* src, uint8_t* dst, const int64_t* src_off, const int64_t* dst_off,
                             const int64_t* size, int64_t n, void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_copy_spans<<<grid_for(n * 32, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(src, dst, src_off,
                                                                                                  dst_off, size, n);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_record_sizes(const uint8_t* data, const int64_t* offsets, int64_t n, int64_t* out, void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_record_sizes<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(data, offsets, n, out);
    return cb_set_error(cudaGetLastError());
}
