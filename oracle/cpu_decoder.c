/* CPU decoder of BAM files: TEST INFRASTRUCTURE ONLY (the oracle for large inputs and the timed
 * CPU baseline).  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may load it.
 *
 * The same semantics as oracle/bam_oracle.py, in C, multithreaded with pthreads:
 *  - BGZF members (src/cubam/_kernels.py:69-89, src/cubam/bgzf.py:542-611): the chain of members
 *    from offset 0 (BSIZE), ISIZE <= 65536, the empty-member rule; every member inflated with the
 *    system zlib (inflateInit2 with -15 window bits: raw DEFLATE, RFC 1951), in parallel, CRC32
 *    optionally checked against the trailer;
 *  - records: the chain from the first record, under the record predicate of
 *    src/cubam/_kernels.py:250-278; the fixed columns of src/cubam/_kernels.py:292-319; tags by one
 *    aux walk per record with find_tag's rules (src/cubam/_kernels.py:334-388); FNV-1a 64 of names
 *    and of string tags (src/cubam/_kernels.py:322-330,532-540).
 * Over a whole file, the records and their columns are the concatenation over cubam's batches.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

enum { ORC_OK = 0, ORC_TRUNCATED = 1, ORC_NO_CHAIN = 2, ORC_CORRUPT = 3, ORC_INFLATE = 4, ORC_CRC = 5, ORC_CAPACITY = 7 };

static inline uint32_t u16(const uint8_t* b, int64_t o) { return (uint32_t)b[o] | ((uint32_t)b[o + 1] << 8); }
static inline uint32_t u32(const uint8_t* b, int64_t o) {
    return (uint32_t)b[o] | ((uint32_t)b[o + 1] << 8) | ((uint32_t)b[o + 2] << 16) | ((uint32_t)b[o + 3] << 24);
}

static int is_member(const uint8_t* b, int64_t n, int64_t o) {
    if (o + 18 > n) return 0;
    if (b[o] != 31 || b[o + 1] != 139 || b[o + 2] != 8 || b[o + 3] != 4) return 0;
    if (b[o + 10] != 6 || b[o + 11] != 0 || b[o + 12] != 66 || b[o + 13] != 67 || b[o + 14] != 2 || b[o + 15] != 0)
        return 0;
    int64_t bs = (int64_t)u16(b, o + 16) + 1;
    return bs >= 26 && o + bs <= n;
}

/* Members of a whole BGZF file (the file must start at one and end with a complete one, unless
 * `partial`: then the members of a prefix).  Writes up to cap (offset, bsize, isize, out_off) rows;
 * returns the count or -status. */
int64_t orc_scan_file(const uint8_t* f, int64_t n, int64_t* off, int64_t* bsize, int64_t* isize, int64_t* out_off,
                      int64_t cap, int partial) {
    int64_t o = 0, m = 0, total = 0;
    while (o < n) {
        if (!is_member(f, n, o)) {
            if (partial && o > 0) break; /* a prefix of the file: stop before the first incomplete member */
            return o == 0 ? -ORC_NO_CHAIN : -ORC_TRUNCATED;
        }
        int64_t bs = (int64_t)u16(f, o + 16) + 1;
        int64_t is = (int64_t)u32(f, o + bs - 4);
        if (is > 65536) return -ORC_CORRUPT;
        if (is == 0 && (bs != 28 || f[o + 18] != 3 || f[o + 19] != 0)) return -ORC_CORRUPT;
        if (m < cap) {
            off[m] = o;
            bsize[m] = bs;
            isize[m] = is;
            out_off[m] = total;
        }
        m++;
        total += is;
        o += bs;
    }
    return m > cap ? -ORC_CAPACITY : m;
}

typedef struct {
    const uint8_t* f;
    const int64_t *off, *bsize, *isize, *out_off;
    uint8_t* out;
    int64_t lo, hi;
    int check_crc;
    int status;
} inflate_task;

static void* inflate_worker(void* arg) {
    inflate_task* t = (inflate_task*)arg;
    z_stream z;
    memset(&z, 0, sizeof(z));
    if (inflateInit2(&z, -15) != Z_OK) {
        t->status = ORC_INFLATE;
        return NULL;
    }
    for (int64_t i = t->lo; i < t->hi && t->status == ORC_OK; i++) {
        int64_t is = t->isize[i];
        if (is == 0) continue;
        inflateReset(&z);
        z.next_in = (Bytef*)(t->f + t->off[i] + 18);
        z.avail_in = (uInt)(t->bsize[i] - 26);
        z.next_out = t->out + t->out_off[i];
        z.avail_out = (uInt)is;
        int rc = inflate(&z, Z_FINISH);
        if (rc != Z_STREAM_END || z.total_out != (uLong)is) {
            t->status = ORC_INFLATE;
            break;
        }
        if (t->check_crc) {
            uint32_t want = u32(t->f, t->off[i] + t->bsize[i] - 8);
            if ((uint32_t)crc32(0L, t->out + t->out_off[i], (uInt)is) != want) t->status = ORC_CRC;
        }
    }
    inflateEnd(&z);
    return NULL;
}

/* Inflate members [0, m) of the scan into out; n_threads workers over contiguous member ranges. */
int orc_inflate(const uint8_t* f, const int64_t* off, const int64_t* bsize, const int64_t* isize,
                const int64_t* out_off, int64_t m, uint8_t* out, int n_threads, int check_crc) {
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 1024) n_threads = 1024;
    pthread_t th[1024];
    inflate_task task[1024];
    for (int k = 0; k < n_threads; k++) {
        inflate_task t = {f, off, bsize, isize, out_off, out, m * k / n_threads, m * (k + 1) / n_threads, check_crc,
                          ORC_OK};
        task[k] = t;
        pthread_create(&th[k], NULL, inflate_worker, &task[k]);
    }
    int status = ORC_OK;
    for (int k = 0; k < n_threads; k++) {
        pthread_join(th[k], NULL);
        if (task[k].status > status) status = task[k].status;
    }
    return status;
}

/* ------------------------------------------------------------------ records */

static int reg2bin(int beg, int end) {
    --end;
    if (beg >> 14 == end >> 14) return 4681 + (beg >> 14);
    if (beg >> 17 == end >> 17) return 585 + (beg >> 17);
    if (beg >> 20 == end >> 20) return 73 + (beg >> 20);
    if (beg >> 23 == end >> 23) return 9 + (beg >> 23);
    if (beg >> 26 == end >> 26) return 1 + (beg >> 26);
    return 0;
}

static inline int ref_consuming(uint32_t op) { return op == 0 || op == 2 || op == 3 || op == 7 || op == 8; }

int orc_is_record(const uint8_t* b, int64_t n, int64_t o, int n_ref) {
    if (o + 36 > n) return 0;
    int32_t bs = (int32_t)u32(b, o);
    if (bs < 33 || bs > (1 << 22) || o + 4 + bs > n) return 0;
    int32_t ref = (int32_t)u32(b, o + 4), pos = (int32_t)u32(b, o + 8);
    int32_t nref = (int32_t)u32(b, o + 24), npos = (int32_t)u32(b, o + 28);
    if (ref < -1 || ref >= n_ref || pos < -1 || nref < -1 || nref >= n_ref || npos < -1) return 0;
    uint32_t lrn = b[o + 12], ncig = u16(b, o + 16), flag = u16(b, o + 18), lseq = u32(b, o + 20);
    if (lrn < 2 || flag >= 4096 || lseq > (1u << 22)) return 0;
    if (32LL + lrn + 4LL * ncig + (lseq + 1) / 2 + lseq > (int64_t)bs) return 0;
    int64_t nm = o + 36;
    if (b[nm + lrn - 1] != 0) return 0;
    for (uint32_t i = 0; i + 1 < lrn; i++) {
        uint8_t c = b[nm + i];
        if (c < 33 || c > 126 || c == '@') return 0;
    }
    int64_t cg = nm + lrn, rlen = 0;
    for (uint32_t i = 0; i < ncig; i++) {
        uint32_t v = u32(b, cg + 4LL * i), op = v & 15;
        if (op > 8) return 0;
        if (ref_consuming(op)) rlen += v >> 4;
    }
    if (pos >= 0) {
        int32_t end = (int32_t)((uint32_t)pos + (uint32_t)(int32_t)(rlen > 0 ? rlen : 1));
        if (u16(b, o + 14) != (uint32_t)reg2bin(pos, end)) return 0;
    }
    return 1;
}

/* Records of data[start:n) on the chain from `start`; returns the count (or -ORC_CAPACITY), *tail = end. */
int64_t orc_record_chain(const uint8_t* b, int64_t n, int64_t start, int n_ref, int64_t* off, int64_t cap,
                         int64_t* tail) {
    int64_t o = start, m = 0;
    while (orc_is_record(b, n, o, n_ref)) {
        if (m < cap) off[m] = o;
        m++;
        o += 4 + (int64_t)u32(b, o);
    }
    *tail = o;
    return m > cap ? -ORC_CAPACITY : m;
}

typedef struct {
    const uint8_t* b;
    const int64_t* off;
    int64_t lo, hi, n;
    int32_t *ref, *pos, *end;
    uint8_t* mapq;
    uint16_t* flag;
    int32_t *nref, *npos, *tlen, *l_seq;
    uint16_t *clip_left, *clip_right;
    uint64_t* name_hash;
    int k;
    const char* tags;
    uint8_t* ty;
    int64_t* voff;
    int32_t* vlen;
    int64_t* ival;
    uint64_t* thash; /* FNV-1a of Z/H values of each tag (0 otherwise) */
} decode_task;

#define FNV_OFFSET 1469598103934665603ULL
#define FNV_PRIME 1099511628211ULL

static void decode_one(decode_task* t, int64_t i) {
    const uint8_t* b = t->b;
    int64_t o = t->off[i];
    int32_t p = (int32_t)u32(b, o + 8);
    t->ref[i] = (int32_t)u32(b, o + 4);
    t->pos[i] = p;
    t->mapq[i] = b[o + 13];
    t->flag[i] = (uint16_t)u16(b, o + 18);
    t->nref[i] = (int32_t)u32(b, o + 24);
    t->npos[i] = (int32_t)u32(b, o + 28);
    t->tlen[i] = (int32_t)u32(b, o + 32);
    t->l_seq[i] = (int32_t)u32(b, o + 20);
    uint32_t lrn = b[o + 12], ncig = u16(b, o + 16), lseq = u32(b, o + 20);
    int64_t cg = o + 36 + lrn, rlen = 0;
    uint32_t cl = 0, cr = 0;
    for (uint32_t k = 0; k < ncig; k++) {
        uint32_t v = u32(b, cg + 4LL * k), op = v & 15, len = v >> 4;
        if (ref_consuming(op)) rlen += len;
        if (op == 4) {
            if (k == 0) cl = len;
            else cr = len;
        }
    }
    t->end[i] = (int32_t)((uint32_t)p + (uint32_t)rlen);
    t->clip_left[i] = (uint16_t)(cl > 65535 ? 65535 : cl);
    t->clip_right[i] = (uint16_t)(cr > 65535 ? 65535 : cr);
    uint64_t h = FNV_OFFSET;
    for (uint32_t k = 0; k + 1 < lrn; k++) h = (h ^ b[o + 36 + k]) * FNV_PRIME;
    t->name_hash[i] = h;
    if (!t->k) return;
    int64_t n = t->n;
    for (int q = 0; q < t->k; q++) {
        t->ty[q * n + i] = 0;
        t->voff[q * n + i] = 0;
        t->vlen[q * n + i] = 0;
        t->ival[q * n + i] = 0;
        t->thash[q * n + i] = 0;
    }
    int64_t rec_end = o + 4 + (int64_t)u32(b, o);
    int64_t a = cg + 4LL * ncig + (lseq + 1) / 2 + lseq;
    uint32_t found = 0, want = (1u << t->k) - 1u;
    while (a + 3 <= rec_end && found != want) {
        uint8_t ty = b[a + 2];
        int64_t v = a + 3, nx;
        switch (ty) {
            case 'A': case 'c': case 'C': nx = v + 1; break;
            case 's': case 'S': nx = v + 2; break;
            case 'i': case 'I': case 'f': nx = v + 4; break;
            case 'Z': case 'H':
                nx = v;
                while (nx < rec_end && b[nx] != 0) nx++;
                nx++;
                break;
            case 'B':
                if (v + 5 > rec_end) {
                    nx = -1;
                } else {
                    uint8_t sub = b[v];
                    int64_t cnt = (int64_t)u32(b, v + 1);
                    int sz = (sub == 'c' || sub == 'C') ? 1 : (sub == 's' || sub == 'S') ? 2 : 4;
                    nx = v + 5 + cnt * sz;
                }
                break;
            default: nx = -1;
        }
        if (nx < 0 || nx > rec_end) {
            for (int q = 0; q < t->k; q++)
                if (!(found >> q & 1)) t->ty[q * n + i] = 255;
            break;
        }
        for (int q = 0; q < t->k; q++) {
            if ((found >> q & 1) || b[a] != (uint8_t)t->tags[2 * q] || b[a + 1] != (uint8_t)t->tags[2 * q + 1]) continue;
            found |= 1u << q;
            int64_t iv = 0;
            int32_t vl = 0;
            switch (ty) {
                case 'c': iv = (int8_t)b[v]; break;
                case 'C': case 'A': iv = b[v]; break;
                case 's': iv = (int16_t)u16(b, v); break;
                case 'S': iv = u16(b, v); break;
                case 'i': iv = (int32_t)u32(b, v); break;
                case 'I': iv = u32(b, v); break;
                case 'Z': case 'H': vl = (int32_t)(nx - 1 - v); break;
                case 'B': vl = (int32_t)(nx - v); break;
                default: break;
            }
            t->ty[q * n + i] = ty;
            t->voff[q * n + i] = v;
            t->vlen[q * n + i] = vl;
            t->ival[q * n + i] = iv;
            if (ty == 'Z' || ty == 'H') {
                uint64_t x = FNV_OFFSET;
                for (int32_t c = 0; c < vl; c++) x = (x ^ b[v + c]) * FNV_PRIME;
                t->thash[q * n + i] = x;
            }
        }
        a = nx;
    }
}

static void* decode_worker(void* arg) {
    decode_task* t = (decode_task*)arg;
    for (int64_t i = t->lo; i < t->hi; i++) decode_one(t, i);
    return NULL;
}

/* Columns of n records at off[] of data b (k <= 16 tags named by tags[2k]). */
int orc_decode(const uint8_t* b, const int64_t* off, int64_t n, int n_threads, int32_t* ref, int32_t* pos,
               int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos, int32_t* tlen,
               int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right, uint64_t* name_hash, int k,
               const char* tags, uint8_t* ty, int64_t* voff, int32_t* vlen, int64_t* ival, uint64_t* thash) {
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 1024) n_threads = 1024;
    if (k < 0 || k > 16) return 9;
    pthread_t th[1024];
    decode_task task[1024];
    for (int q = 0; q < n_threads; q++) {
        decode_task t = {b, off, n * q / n_threads, n * (q + 1) / n_threads, n, ref, pos, end, mapq, flag, nref, npos,
                         tlen, l_seq, clip_left, clip_right, name_hash, k, tags, ty, voff, vlen, ival, thash};
        task[q] = t;
        pthread_create(&th[q], NULL, decode_worker, &task[q]);
    }
    for (int q = 0; q < n_threads; q++) pthread_join(th[q], NULL);
    return ORC_OK;
}
