// BAM record columns on B200: the fixed columns (src/cubam/_kernels.py:292-319), the aux tags
// (src/cubam/_kernels.py:334-388) and the on-request decoders (src/cubam/_kernels.py:322-620,
// src/cubam/bam.py:299-400).  The record chain itself is in chain.cu.

#include "common.cuh"

namespace cb {
namespace rec {

__device__ __forceinline__ bool ref_consuming(uint32_t op) {
    return op == 0 || op == 2 || op == 3 || op == 7 || op == 8;  // M D N = X
}

// ---------------------------------------------------------------- columns

constexpr unsigned long long FNV_OFFSET = 1469598103934665603ULL;
constexpr unsigned long long FNV_PRIME = 1099511628211ULL;

// The fixed columns (src/cubam/_kernels.py:292-319) and, when their pointers are given, the
// aligned length and the read-name hash of each record in the same pass over its bytes (the values
// k_aligned_length and k_name_hash give).
__global__ void k_decode_fixed(const uint8_t* __restrict__ b, const int64_t* __restrict__ off, long long n,
                               int32_t* ref, int32_t* pos, int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref,
                               int32_t* npos, int32_t* tlen, int32_t* l_seq, uint16_t* clip_left,
                               uint16_t* clip_right, int32_t* aligned, uint64_t* name_hash) {
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
        uint32_t cl = 0, cr = 0, al = 0;
        for (uint32_t k = 0; k < ncig; k++) {
            uint32_t v = ld_u32(b, cg + 4LL * k), op = v & 15, len = v >> 4;
            if (ref_consuming(op)) rlen += len;
            if (op == 0 || op == 7 || op == 8) al += len;
            if (op == 4) {
                if (k == 0) cl = len;
                else cr = len;
            }
        }
        end[i] = p + (int)rlen;
        clip_left[i] = (uint16_t)(cl > 65535 ? 65535 : cl);
        clip_right[i] = (uint16_t)(cr > 65535 ? 65535 : cr);
        if (aligned) aligned[i] = (int32_t)al;
        if (name_hash) {
            unsigned long long x = FNV_OFFSET;
            for (uint32_t k = 0; k + 1 < lrn; k++) {
                x ^= b[o + 36 + k];
                x *= FNV_PRIME;
            }
            name_hash[i] = x;
        }
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

extern "C" int cb_decode_fixed(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* ref, int32_t* pos,
                               int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos,
                               int32_t* tlen, int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right,
                               void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_decode_fixed<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        data, offsets, n, ref, pos, end, mapq, flag, nref, npos, tlen, l_seq, clip_left, clip_right, nullptr, nullptr);
    return cb_set_error(cudaGetLastError());
}

extern "C" int cb_decode_records(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* ref, int32_t* pos,
                                 int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos,
                                 int32_t* tlen, int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right,
                                 int32_t* aligned_length, uint64_t* name_hash, void* stream) {
    if (n < 0) return CB_ERR_ARG;
    if (n == 0) return CB_OK;
    rec::k_decode_fixed<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        data, offsets, n, ref, pos, end, mapq, flag, nref, npos, tlen, l_seq, clip_left, clip_right, aligned_length,
        name_hash);
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
