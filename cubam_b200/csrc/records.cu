// BAM record columns on B200: the fixed columns (src/cubam/_kernels.py:292-319), the aux tags
// (src/cubam/_kernels.py:334-388) and the on-request decoders (src/cubam/_kernels.py:322-620,
// src/cubam/bam.py:299-400).  The record chain itself is in chain.cu.

#include <atomic>

#include "common.cuh"

namespace cb {
namespace rec {

__device__ __forceinline__ bool ref_consuming(uint32_t op) {
    return op == 0 || op == 2 || op == 3 || op == 7 || op == 8;  // M D N = X
}

// ---------------------------------------------------------------- columns

constexpr unsigned long long FNV_OFFSET = 1469598103934665603ULL;
constexpr unsigned long long FNV_PRIME = 1099511628211ULL;

// ---------------------------------------------------------------- the record pass
//
// One warp decodes 32 consecutive entries of `off`.  The bytes from the group's first record to the
// next group's first record (the group's records, when the offsets are a record chain) are first
// copied to shared memory with 16-byte loads (coalesced, each byte read once from HBM); each lane
// then parses its record from there: the fixed columns (src/cubam/_kernels.py:292-319), the
// aligned length and read-name hash (src/cubam/_kernels.py:322-330, :391-403) and k aux tags in one
// walk (src/cubam/_kernels.py:334-388).  Any byte outside the staged window (a record longer than
// the window, offsets that are not ascending, as after a take) is read from global memory, so the
// result never depends on the window.

constexpr int RW = 4;           // warps per block
constexpr int STAGE = 12288;    // bytes staged per warp (32 records of up to 384 bytes)

struct Cols {
    int32_t *ref, *pos, *end;
    uint8_t* mapq;
    uint16_t* flag;
    int32_t *nref, *npos, *tlen, *l_seq;
    uint16_t *clip_left, *clip_right;
    int32_t* aligned;
    uint64_t* name_hash;
    int32_t* nblk;        // aligned blocks per read, deletions inside a block (as blocks(split_deletions=0))
    int32_t* nblk_split;  // the same with deletions splitting blocks
};

// Aligned blocks of one read in the two modes of blocks() (src/cubam/_kernels.py:408-437): a block
// ends at an N (and, splitting, at a D) and is counted when it covers a reference base.
struct BlockCount {
    uint32_t x = 0, s = 0;
    int k = 0;
    __device__ __forceinline__ void start(uint32_t pos) { x = s = pos; }
    __device__ __forceinline__ void op(uint32_t op, uint32_t l, bool split) {
        const bool aligned = op == 0 || op == 7 || op == 8 || (op == 2 && !split);
        const bool gap = op == 3 || (op == 2 && split);
        if (aligned) {
            x += l;
        } else if (gap) {
            if ((int)x > (int)s) k++;
            x += l;
            s = x;
        }
    }
    __device__ __forceinline__ int end() const { return k + ((int)x > (int)s ? 1 : 0); }
};

struct TagNames {
    uint8_t c[32];
};

struct TagOut {
    uint8_t* type;
    int64_t* voff;
    int32_t* vlen;
    int64_t* ival;
    long long stride;  // entries between tags (tag-major)
};

using Win = StagedBytes;

// Offset just past the NUL that ends the string at v, or rec_end + 1 when none comes before rec_end
// (the reference's byte loop, src/cubam/_kernels.py:356-359), four bytes at a time in the window.
__device__ __forceinline__ long long str_end(const Win& w, long long v, long long rec_end) {
    long long p = v;
    while (p < rec_end) {
        if (w.in(p, 4)) {
            const uint32_t x = w.u32(p);
            const uint32_t z = (x - 0x01010101u) & ~x & 0x80808080u;  // its lowest set bit marks the first 0 byte
            if (z) {
                const long long q = p + ((__ffs(z) - 1) >> 3);
                return q < rec_end ? q + 1 : rec_end + 1;
            }
            p += 4;
        } else {
            if (w.u8(p) == 0) return p + 1;
            p++;
        }
    }
    return rec_end + 1;
}

__device__ __forceinline__ void parse_record(const Win& w, long long o, long long i, const Cols& c, bool cols,
                                             const uint32_t* tag_code, int k, const TagOut& t) {
    const uint32_t w12 = w.u32(o + 12), w16 = w.u32(o + 16);
    const uint32_t lrn = w12 & 255, ncig = w16 & 0xffff;
    const uint32_t lseq = w.u32(o + 20);
    const bool blocks = c.nblk || c.nblk_split;
    if (cols || blocks) {
        const int p = (int)w.u32(o + 8);
        BlockCount b0, b1;
        b0.start((uint32_t)p);
        b1.start((uint32_t)p);
        if (cols) {
            c.ref[i] = (int)w.u32(o + 4);
            c.pos[i] = p;
            c.mapq[i] = (uint8_t)(w12 >> 8);
            c.flag[i] = (uint16_t)(w16 >> 16);
            c.nref[i] = (int)w.u32(o + 24);
            c.npos[i] = (int)w.u32(o + 28);
            c.tlen[i] = (int)w.u32(o + 32);
            c.l_seq[i] = (int)lseq;
        }
        const long long cg = o + 36 + lrn;
        long long rlen = 0;
        uint32_t cl = 0, cr = 0, al = 0;
        for (uint32_t q = 0; q < ncig; q++) {
            const uint32_t v = w.u32(cg + 4LL * q), op = v & 15, len = v >> 4;
            if (ref_consuming(op)) rlen += len;
            if (op == 0 || op == 7 || op == 8) al += len;
            if (op == 4) {
                if (q == 0) cl = len;
                else cr = len;
            }
            if (blocks) {
                b0.op(op, len, false);
                b1.op(op, len, true);
            }
        }
        if (cols) {
            c.end[i] = p + (int)rlen;
            c.clip_left[i] = (uint16_t)(cl > 65535 ? 65535 : cl);
            c.clip_right[i] = (uint16_t)(cr > 65535 ? 65535 : cr);
        }
        if (c.aligned) c.aligned[i] = (int32_t)al;
        if (c.nblk) c.nblk[i] = b0.end();
        if (c.nblk_split) c.nblk_split[i] = b1.end();
    } else if (c.aligned) {
        const long long cg = o + 36 + lrn;
        uint32_t al = 0;
        for (uint32_t q = 0; q < ncig; q++) {
            const uint32_t v = w.u32(cg + 4LL * q), op = v & 15;
            if (op == 0 || op == 7 || op == 8) al += v >> 4;
        }
        c.aligned[i] = (int32_t)al;
    }
    if (c.name_hash) {
        unsigned long long x = FNV_OFFSET;
        for (uint32_t q = 0; q + 1 < lrn; q++) {
            x ^= w.u8(o + 36 + q);
            x *= FNV_PRIME;
        }
        c.name_hash[i] = x;
    }
    if (k == 0) return;
    // the aux walk: one pass that fills k tags
    const long long rec_end = o + 4 + (long long)w.u32(o);
    long long a = o + 36 + lrn + 4LL * ncig + (lseq + 1) / 2 + lseq;
    const uint32_t want = (1u << k) - 1u;
    uint32_t found = 0;
    for (int q = 0; q < k; q++) {
        t.type[q * t.stride + i] = 0;
        t.voff[q * t.stride + i] = 0;
        t.vlen[q * t.stride + i] = 0;
        t.ival[q * t.stride + i] = 0;
    }
    while (a + 3 <= rec_end && found != want) {
        const uint32_t code = w.u8(a) | (w.u8(a + 1) << 8), ty = w.u8(a + 2);
        const long long v = a + 3;
        long long nx;
        switch (ty) {
            case 'A': case 'c': case 'C': nx = v + 1; break;
            case 's': case 'S': nx = v + 2; break;
            case 'i': case 'I': case 'f': nx = v + 4; break;
            case 'Z': case 'H': nx = str_end(w, v, rec_end); break;
            case 'B': {
                if (v + 5 > rec_end) {
                    nx = -1;
                    break;
                }
                const uint32_t sub = w.u8(v);
                const long long cnt = (long long)w.u32(v + 1);
                const int sz = (sub == 'c' || sub == 'C') ? 1 : (sub == 's' || sub == 'S') ? 2 : 4;
                nx = v + 5 + cnt * sz;
                break;
            }
            default: nx = -1;
        }
        if (nx < 0 || nx > rec_end) {
            // malformed: every tag not found yet gets 255
            for (int q = 0; q < k; q++)
                if (!(found >> q & 1)) t.type[q * t.stride + i] = 255;
            break;
        }
        for (int q = 0; q < k; q++) {
            if ((found >> q & 1) || code != tag_code[q]) continue;
            found |= 1u << q;
            long long iv = 0;
            int vl = 0;
            switch (ty) {
                case 'c': iv = (signed char)w.u8(v); break;
                case 'C': case 'A': iv = w.u8(v); break;
                case 's': iv = (short)w.u16(v); break;
                case 'S': iv = w.u16(v); break;
                case 'i': iv = (int)w.u32(v); break;
                case 'I': iv = w.u32(v); break;
                case 'Z': case 'H': vl = (int)(nx - 1 - v); break;
                case 'B': vl = (int)(nx - v); break;
                default: break;
            }
            t.type[q * t.stride + i] = (uint8_t)ty;
            t.voff[q * t.stride + i] = v;
            t.vlen[q * t.stride + i] = vl;
            t.ival[q * t.stride + i] = iv;
        }
        a = nx;
    }
}

__global__ void __launch_bounds__(RW * 32) k_records(const uint8_t* __restrict__ b, const int64_t* __restrict__ off,
                                                      long long n, Cols c, int cols, TagNames names, int k, TagOut t) {
    extern __shared__ uint4 stage_mem[];
    __shared__ uint32_t tag_code[16];  // the k tag names, two characters each
    if (threadIdx.x < 16) tag_code[threadIdx.x] = names.c[2 * threadIdx.x] | (names.c[2 * threadIdx.x + 1] << 8);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint4* st = stage_mem + (size_t)warp * (STAGE / 16);
    const long long groups = (n + 31) >> 5;
    for (long long g = (long long)blockIdx.x * RW + warp; g < groups; g += (long long)gridDim.x * RW) {
        const long long i0 = g << 5, i = i0 + lane;
        const bool valid = i < n;
        const long long o = valid ? off[i] : 0;
        // the window: from the group's first record to the next group's first (the last group: to the
        // end of its last entry's record); it stays 16 bytes short of the stage for the word reads
        const long long lo = __shfl_sync(FULL, o, 0);
        long long hi;
        if (i0 + 32 < n) {
            hi = off[i0 + 32];
        } else {
            const int last = (int)(n - 1 - i0);
            long long e = 0;
            if (lane == last) e = o + 4 + (long long)ld_u32(b, o);
            hi = __shfl_sync(FULL, e, last);
        }
        if (hi > lo + STAGE - 32) hi = lo + STAGE - 32;
        if (hi < lo) hi = lo;
        const long long r0 = stage_bytes(b, lo, hi, st);
        if (valid) {
            const Win w{b, reinterpret_cast<const uint8_t*>(st), r0, hi};
            parse_record(w, o, i, c, cols != 0, tag_code, k, t);
        }
        __syncwarp();
    }
}

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

// The record pass (k_records): every column group is optional; k = 0 for no tags.
static int launch_records(const uint8_t* data, const int64_t* offsets, int64_t n, const rec::Cols& c, bool cols,
                          const char* names, int32_t k, uint8_t* type, int64_t* voff, int32_t* vlen, int64_t* value,
                          void* stream) {
    if (n < 0 || k < 0 || k > 16 || (k > 0 && (!names || !type || !voff || !vlen || !value))) return CB_ERR_ARG;
    if (cols && !(c.ref && c.pos && c.end && c.mapq && c.flag && c.nref && c.npos && c.tlen && c.l_seq &&
                  c.clip_left && c.clip_right))
        return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    if (!data || !offsets) return CB_ERR_ARG;
    rec::TagNames tn{};
    for (int i = 0; i < 2 * k; i++) tn.c[i] = (uint8_t)names[i];
    const rec::TagOut t{type, voff, vlen, value, (long long)n};
    const size_t smem = (size_t)rec::RW * rec::STAGE;
    static std::atomic<bool> attr_set[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_set[dev].load(std::memory_order_acquire)) {
        const cudaError_t e = cudaFuncSetAttribute(rec::k_records, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cb_set_error(e);
        if (dev >= 0 && dev < 64) attr_set[dev].store(true, std::memory_order_release);
    }
    const long long groups = (n + 31) / 32;
    long long grid = (groups + rec::RW - 1) / rec::RW;
    const long long cap = (long long)cb_device_sm_count() * 8;
    if (grid > cap) grid = cap;
    rec::k_records<<<(unsigned)grid, rec::RW * 32, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        data, offsets, n, c, cols ? 1 : 0, tn, k, t);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_decode_columns(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* ref, int32_t* pos,
                                 int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos,
                                 int32_t* tlen, int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right,
                                 int32_t* aligned_length, uint64_t* name_hash, int32_t* n_blocks,
                                 int32_t* n_blocks_split, const char* names, int32_t k, uint8_t* type,
                                 int64_t* voff, int32_t* vlen, int64_t* value, void* stream) {
    const rec::Cols c{ref,       pos,        end,      mapq,           flag,     nref, npos,
                      tlen,      l_seq,      clip_left, clip_right,    aligned_length, name_hash,
                      n_blocks,  n_blocks_split};
    return launch_records(data, offsets, n, c, ref != nullptr, names, k, type, voff, vlen, value, stream);
}

extern "C" int cb_decode_fixed(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* ref, int32_t* pos,
                               int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos,
                               int32_t* tlen, int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right,
                               void* stream) {
    const rec::Cols c{ref, pos, end, mapq, flag, nref, npos, tlen, l_seq, clip_left, clip_right, nullptr, nullptr};
    return launch_records(data, offsets, n, c, true, nullptr, 0, nullptr, nullptr, nullptr, nullptr, stream);
}

extern "C" int cb_decode_records(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* ref, int32_t* pos,
                                 int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos,
                                 int32_t* tlen, int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right,
                                 int32_t* aligned_length, uint64_t* name_hash, void* stream) {
    const rec::Cols c{ref, pos, end, mapq, flag, nref, npos, tlen, l_seq, clip_left, clip_right, aligned_length,
                      name_hash};
    return launch_records(data, offsets, n, c, true, nullptr, 0, nullptr, nullptr, nullptr, nullptr, stream);
}

extern "C" int cb_find_tags(const uint8_t* data, const int64_t* offsets, int64_t n, const char* names, int32_t k,
                            uint8_t* type, int64_t* voff, int32_t* vlen, int64_t* value, void* stream) {
    if (k < 1) return CB_ERR_ARG;
    const rec::Cols c{};
    return launch_records(data, offsets, n, c, false, names, k, type, voff, vlen, value, stream);
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
