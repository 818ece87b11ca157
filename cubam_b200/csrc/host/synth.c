/* Seeded synthetic BAM files of the shapes of the reader benchmarks (host code, C + zlib).
 *
 * Shapes:
 *   0  small single-end: 1 reference of 1,000,000 bp, 90 bp reads, CIGAR 90M, MAPQ 255, flag 0/16,
 *      CB:Z (16-mer + "-1" from n_barcodes) and UB:Z (random 12-mer);
 *   1  GEX: 25 references with the lengths of the human chromosomes (GRCh38), 91 bp reads, 75% 91M,
 *      20% with 1-2 N introns of log-uniform 100-50,000 bp, 10% with soft clips of 1-30 bp, MAPQ 255
 *      or 0 (9:1), CB/UB, GN:Z from 30,000 gene symbols, xf from {0,17,25}, NH 1-4;
 *   2  ATAC pairs: 50 bp mates, fragment length log-normal (median 150, clipped to 20-1,000), flags
 *      99/147 or 83/163, 5% of pairs duplicate-flagged, CB:Z from n_barcodes.
 * Records are coordinate-sorted, bases uniform ACGT, names 16 characters; qualities are uniform in
 * 2..41 for shape 0 and binned as NovaSeq writes them (37/23/12/2 at 80/10/7/3%) for shapes 1 and 2.
 * The record stream is cut into members of 0xFF00 bytes (as htslib writes) compressed with zlib at
 * `level` (or 1..9 at random per member when level < 0), a fraction `stored_frac` of members are
 * stored (BTYPE 0); the header is its own member and the file ends with the EOF member.
 * Work is spread over `n_threads` threads: record segments are generated in parallel (each from its
 * own seed, so the output does not depend on the thread count) and members compressed in parallel.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

#define BLOCK 0xFF00
#define SEG_RECORDS 131072

typedef struct {
    uint64_t s[4];
} rng_t;

static uint64_t splitmix(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static void rng_seed(rng_t* r, uint64_t seed, uint64_t stream) {
    uint64_t x = seed * 0x100000001B3ull ^ (stream + 0x632BE59BD9B4E019ull);
    for (int i = 0; i < 4; i++) r->s[i] = splitmix(&x);
}
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static inline uint64_t next_u64(rng_t* r) { /* xoshiro256** */
    uint64_t* s = r->s;
    uint64_t res = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return res;
}
static inline double unif(rng_t* r) { return (next_u64(r) >> 11) * (1.0 / 9007199254740992.0); }
static inline uint32_t below(rng_t* r, uint32_t n) { return (uint32_t)(((next_u64(r) >> 32) * (uint64_t)n) >> 32); }

static const int64_t HUMAN[25] = {248956422, 242193529, 198295559, 190214555, 181538259, 170805979, 159345973,
                                  145138636, 138394717, 133797422, 135086622, 133275309, 114364328, 107043718,
                                  101991189, 90338345,  83257441,  80373285,  58617616,  64444167,  46709983,
                                  50818468,  156040895, 57227415,  16569};
static const char* HUMAN_NAMES[25] = {"chr1",  "chr2",  "chr3",  "chr4",  "chr5",  "chr6",  "chr7",
                                      "chr8",  "chr9",  "chr10", "chr11", "chr12", "chr13", "chr14",
                                      "chr15", "chr16", "chr17", "chr18", "chr19", "chr20", "chr21",
                                      "chr22", "chrX",  "chrY",  "chrM"};

typedef struct {
    int shape, level, n_threads;
    int64_t n_records;
    uint64_t seed;
    double stored_frac;
    int n_barcodes;
    int n_refs;
    int64_t ref_len[25];
    int64_t genome;
    int64_t cum[26];
    char* barcodes; /* n_barcodes x 16 */
    char* genes;    /* 30000 x 12 (NUL padded) */
    uint8_t* gene_len;
} cfg_t;

static int reg2bin(int beg, int end) {
    --end;
    if (beg >> 14 == end >> 14) return 4681 + (beg >> 14);
    if (beg >> 17 == end >> 17) return 585 + (beg >> 17);
    if (beg >> 20 == end >> 20) return 73 + (beg >> 20);
    if (beg >> 23 == end >> 23) return 9 + (beg >> 23);
    if (beg >> 26 == end >> 26) return 1 + (beg >> 26);
    return 0;
}

typedef struct {
    uint8_t* p;
    int64_t n, cap;
} buf_t;

static void reserve(buf_t* b, int64_t more) {
    if (b->n + more <= b->cap) return;
    int64_t c = b->cap ? b->cap : 1 << 20;
    while (c < b->n + more) c *= 2;
    b->p = (uint8_t*)realloc(b->p, (size_t)c);
    b->cap = c;
}
static inline void put32(uint8_t* d, uint32_t v) {
    d[0] = v & 255;
    d[1] = (v >> 8) & 255;
    d[2] = (v >> 16) & 255;
    d[3] = v >> 24;
}
static inline void put16(uint8_t* d, uint32_t v) {
    d[0] = v & 255;
    d[1] = (v >> 8) & 255;
}

typedef struct {
    int32_t ref, pos, mate_pos, tlen;
    uint16_t flag;
    uint8_t mapq;
    uint8_t ncig;
    uint32_t cig[8];
    int32_t span;
    uint64_t name_id;
    uint32_t cb, gene;
    uint8_t xf, nh;
    int l_seq;
} rec_t;

static void emit(buf_t* out, const cfg_t* c, const rec_t* r, rng_t* g) {
    const int lrn = 17;
    int l_seq = r->l_seq;
    int aux = 0;
    if (c->shape == 0 || c->shape == 1) aux += 3 + 19 + 3 + 13;
    if (c->shape == 1) aux += 3 + c->gene_len[r->gene] + 1 + 4 + 4;
    if (c->shape == 2) aux += 3 + 19;
    int bs = 32 + lrn + 4 * r->ncig + (l_seq + 1) / 2 + l_seq + aux;
    reserve(out, 4 + bs);
    uint8_t* d = out->p + out->n;
    put32(d, (uint32_t)bs);
    put32(d + 4, (uint32_t)r->ref);
    put32(d + 8, (uint32_t)r->pos);
    d[12] = (uint8_t)lrn;
    d[13] = r->mapq;
    put16(d + 14, (uint32_t)reg2bin(r->pos, r->pos + (r->span > 0 ? r->span : 1)));
    put16(d + 16, r->ncig);
    put16(d + 18, r->flag);
    put32(d + 20, (uint32_t)l_seq);
    put32(d + 24, (uint32_t)(c->shape == 2 ? r->ref : -1));
    put32(d + 28, (uint32_t)(c->shape == 2 ? r->mate_pos : -1));
    put32(d + 32, (uint32_t)r->tlen);
    uint8_t* q = d + 36;
    static const char hex[] = "0123456789ABCDEF";
    q[0] = 'R';
    uint64_t id = r->name_id;
    for (int k = 15; k >= 1; k--) {
        q[k] = (uint8_t)hex[id & 15];
        id >>= 4;
    }
    q[16] = 0;
    q += lrn;
    for (int k = 0; k < r->ncig; k++, q += 4) put32(q, r->cig[k]);
    static const uint8_t code[4] = {1, 2, 4, 8};
    for (int k = 0; k < (l_seq + 1) / 2; k++) {
        uint64_t x = next_u64(g);
        uint8_t hi = code[x & 3], lo = (2 * k + 1 < l_seq) ? code[(x >> 2) & 3] : 0;
        *q++ = (uint8_t)((hi << 4) | lo);
    }
    if (c->shape == 0) {
        for (int k = 0; k < l_seq; k++) *q++ = (uint8_t)(2 + below(g, 40));
    } else {
        /* binned qualities as NovaSeq writes them: 37 / 23 / 12 / 2 */
        for (int k = 0; k < l_seq; k++) {
            uint32_t u = below(g, 100);
            *q++ = (uint8_t)(u < 80 ? 37 : u < 90 ? 23 : u < 97 ? 12 : 2);
        }
    }
    if (c->shape == 0 || c->shape == 1 || c->shape == 2) {
        q[0] = 'C';
        q[1] = 'B';
        q[2] = 'Z';
        memcpy(q + 3, c->barcodes + 16 * (size_t)r->cb, 16);
        q[19] = '-';
        q[20] = '1';
        q[21] = 0;
        q += 22;
    }
    if (c->shape == 0 || c->shape == 1) {
        static const char acgt[] = "ACGT";
        q[0] = 'U';
        q[1] = 'B';
        q[2] = 'Z';
        uint64_t x = next_u64(g);
        for (int k = 0; k < 12; k++) q[3 + k] = (uint8_t)acgt[(x >> (2 * k)) & 3];
        q[15] = 0;
        q += 16;
    }
    if (c->shape == 1) {
        int gl = c->gene_len[r->gene];
        q[0] = 'G';
        q[1] = 'N';
        q[2] = 'Z';
        memcpy(q + 3, c->genes + 12 * (size_t)r->gene, (size_t)gl);
        q[3 + gl] = 0;
        q += 4 + gl;
        q[0] = 'x';
        q[1] = 'f';
        q[2] = 'C';
        q[3] = r->xf;
        q[4] = 'N';
        q[5] = 'H';
        q[6] = 'C';
        q[7] = r->nh;
        q += 8;
    }
    out->n += 4 + bs;
}

static void global_to_ref(const cfg_t* c, int64_t gpos, int32_t* ref, int32_t* pos) {
    int lo = 0, hi = c->n_refs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) / 2;
        if (c->cum[mid] <= gpos) lo = mid;
        else hi = mid - 1;
    }
    *ref = lo;
    *pos = (int32_t)(gpos - c->cum[lo]);
}

static int cmp_i64(const void* a, const void* b) {
    int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return x < y ? -1 : x > y;
}

typedef struct {
    int64_t key, idx;
} keyed_t;
static int cmp_keyed(const void* a, const void* b) {
    const keyed_t *x = (const keyed_t*)a, *y = (const keyed_t*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->idx < y->idx ? -1 : x->idx > y->idx;
}

/* Records [seg * SEG_RECORDS, ...) of the file, in coordinate order. */
static void gen_segment(const cfg_t* c, int64_t seg, int64_t n_seg, buf_t* out) {
    rng_t g;
    rng_seed(&g, c->seed, (uint64_t)seg);
    int64_t r0 = seg * SEG_RECORDS, r1 = r0 + SEG_RECORDS < c->n_records ? r0 + SEG_RECORDS : c->n_records;
    int64_t n = r1 - r0;
    int64_t glo = c->genome * seg / n_seg, ghi = c->genome * (seg + 1) / n_seg;
    if (c->shape == 2) {
        int64_t pairs = n / 2;
        int64_t* gp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(pairs + 1));
        for (int64_t i = 0; i < pairs; i++) gp[i] = glo + (int64_t)(unif(&g) * (double)(ghi - glo - 1100));
        qsort(gp, (size_t)pairs, sizeof(int64_t), cmp_i64);
        rec_t* rs = (rec_t*)malloc(sizeof(rec_t) * (size_t)(2 * pairs + 1));
        for (int64_t i = 0; i < pairs; i++) {
            double z = sqrt(-2.0 * log(unif(&g) + 1e-300)) * cos(6.283185307179586 * unif(&g));
            int L = (int)(150.0 * exp(0.5 * z));
            if (L < 20) L = 20;
            if (L > 1000) L = 1000;
            int32_t ref, pos;
            global_to_ref(c, gp[i], &ref, &pos);
            if (pos + L + 60 > c->ref_len[ref]) pos = (int32_t)(c->ref_len[ref] - L - 60 > 0 ? c->ref_len[ref] - L - 60 : 0);
            int32_t mpos = pos + (L >= 50 ? L - 50 : 0);
            int rev = (int)(next_u64(&g) & 1);
            uint16_t dup = unif(&g) < 0.05 ? 0x400 : 0;
            uint32_t cb = below(&g, (uint32_t)c->n_barcodes);
            uint64_t id = (uint64_t)(r0 / 2 + i) * 0x9E3779B97F4A7C15ull;
            for (int m = 0; m < 2; m++) {
                rec_t* r = &rs[2 * i + m];
                memset(r, 0, sizeof(*r));
                r->ref = ref;
                r->pos = m ? mpos : pos;
                r->mate_pos = m ? pos : mpos;
                r->tlen = m ? -L : L;
                /* read1 forward + read2 reverse (99/147), or read1 reverse + read2 forward (83/163) */
                if (!rev) r->flag = (uint16_t)((m ? 147 : 99) | dup);
                else r->flag = (uint16_t)((m ? 163 : 83) | dup);
                r->mapq = 60;
                r->ncig = 1;
                r->cig[0] = (50u << 4) | 0;
                r->span = 50;
                r->l_seq = 50;
                r->name_id = id >> 4;
                r->cb = cb;
            }
        }
        /* coordinate order: key (ref, pos, index) */
        keyed_t* ord = (keyed_t*)malloc(sizeof(keyed_t) * (size_t)(2 * pairs + 1));
        for (int64_t i = 0; i < 2 * pairs; i++) {
            ord[i].key = ((int64_t)rs[i].ref << 32) | (int64_t)(uint32_t)rs[i].pos;
            ord[i].idx = i;
        }
        qsort(ord, (size_t)(2 * pairs), sizeof(keyed_t), cmp_keyed);
        for (int64_t i = 0; i < 2 * pairs; i++) emit(out, c, &rs[ord[i].idx], &g);
        free(ord);
        free(rs);
        free(gp);
        return;
    }
    int64_t* gp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
    for (int64_t i = 0; i < n; i++) gp[i] = glo + (int64_t)(unif(&g) * (double)(ghi - glo));
    qsort(gp, (size_t)n, sizeof(int64_t), cmp_i64);
    for (int64_t i = 0; i < n; i++) {
        rec_t r;
        memset(&r, 0, sizeof(r));
        int32_t ref, pos;
        global_to_ref(c, gp[i], &ref, &pos);
        r.ref = ref;
        r.tlen = 0;
        r.name_id = (uint64_t)(r0 + i) * 0x9E3779B97F4A7C15ull >> 4;
        r.cb = below(&g, (uint32_t)c->n_barcodes);
        if (c->shape == 0) {
            r.flag = (next_u64(&g) & 1) ? 16 : 0;
            r.mapq = 255;
            r.ncig = 1;
            r.cig[0] = (90u << 4) | 0;
            r.span = 90;
            r.l_seq = 90;
        } else {
            r.flag = (next_u64(&g) & 1) ? 16 : 0;
            r.mapq = unif(&g) < 0.9 ? 255 : 0;
            r.l_seq = 91;
            double u = unif(&g);
            int introns = u < 0.75 ? 0 : u < 0.95 ? 1 + (int)(next_u64(&g) & 1) : 0;
            int clip = (u >= 0.90) ? 1 + (int)below(&g, 30) : 0; /* 10%: 0.90-0.95 with an intron, 0.95-1 without */
            int aligned = 91 - clip;
            int nc = 0, span = 0;
            int left_clip = clip && (next_u64(&g) & 1);
            if (clip && left_clip) r.cig[nc++] = ((uint32_t)clip << 4) | 4;
            int seg_n = introns + 1, done = 0;
            for (int s = 0; s < seg_n; s++) {
                int m = (s == seg_n - 1) ? aligned - done : (aligned / seg_n);
                r.cig[nc++] = ((uint32_t)m << 4) | 0;
                done += m;
                span += m;
                if (s < seg_n - 1) {
                    int nlen = (int)exp(log(100.0) + unif(&g) * (log(50000.0) - log(100.0)));
                    r.cig[nc++] = ((uint32_t)nlen << 4) | 3;
                    span += nlen;
                }
            }
            if (clip && !left_clip) r.cig[nc++] = ((uint32_t)clip << 4) | 4;
            r.ncig = (uint8_t)nc;
            r.span = span;
            r.gene = below(&g, 30000);
            static const uint8_t xfs[3] = {0, 17, 25};
            r.xf = xfs[below(&g, 3)];
            r.nh = (uint8_t)(1 + below(&g, 4));
        }
        if (pos + r.span > c->ref_len[ref]) pos = (int32_t)(c->ref_len[ref] - r.span > 0 ? c->ref_len[ref] - r.span : 0);
        r.pos = pos;
        emit(out, c, &r, &g);
    }
    free(gp);
}

/* ------------------------------------------------------------------ BGZF */

static int64_t member(const uint8_t* data, int64_t n, int level, uint8_t* out) {
    /* out has room for n + 1024 bytes */
    z_stream z;
    memset(&z, 0, sizeof(z));
    deflateInit2(&z, level, Z_DEFLATED, -15, 8, Z_DEFAULT_STRATEGY);
    z.next_in = (Bytef*)data;
    z.avail_in = (uInt)n;
    z.next_out = out + 18;
    z.avail_out = (uInt)(n + 1024 - 26);
    deflate(&z, Z_FINISH);
    int64_t pay = (int64_t)z.total_out;
    deflateEnd(&z);
    int64_t bs = 18 + pay + 8;
    static const uint8_t h[16] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67, 2, 0};
    memcpy(out, h, 16);
    put16(out + 16, (uint32_t)(bs - 1));
    put32(out + 18 + pay, (uint32_t)crc32(0L, data, (uInt)n));
    put32(out + 22 + pay, (uint32_t)n);
    return bs;
}

typedef struct {
    const cfg_t* c;
    const uint8_t* data;
    int64_t n_members, total;
    int64_t lo, hi;
    uint8_t** out;
    int64_t* out_n;
    uint64_t wave;
    int64_t first_member;
} ztask_t;

static void* compress_worker(void* arg) {
    ztask_t* t = (ztask_t*)arg;
    for (int64_t k = t->lo; k < t->hi; k++) {
        int64_t a = k * BLOCK, n = a + BLOCK <= t->total ? BLOCK : t->total - a;
        rng_t g;
        rng_seed(&g, t->c->seed ^ 0xC0FFEEull, (uint64_t)(t->first_member + k));
        int level = t->c->level >= 0 ? t->c->level : 1 + (int)below(&g, 9);
        if (t->c->stored_frac > 0 && unif(&g) < t->c->stored_frac) level = 0;
        t->out[k] = (uint8_t*)malloc((size_t)(n + 1024));
        t->out_n[k] = member(t->data + a, n, level, t->out[k]);
    }
    return NULL;
}

typedef struct {
    const cfg_t* c;
    int64_t seg, n_seg;
    buf_t out;
} gtask_t;

static void* gen_worker(void* arg) {
    gtask_t* t = (gtask_t*)arg;
    gen_segment(t->c, t->seg, t->n_seg, &t->out);
    return NULL;
}

/* Write the BAM file; returns 0, and the uncompressed record bytes and member count. */
int synth_bam(const char* path, int shape, int64_t n_records, uint64_t seed, int level, double stored_frac,
              int n_barcodes, int n_threads, int64_t* out_record_bytes, int64_t* out_members,
              int64_t* out_file_bytes) {
    cfg_t c;
    memset(&c, 0, sizeof(c));
    c.shape = shape;
    c.level = level;
    c.n_records = n_records;
    c.seed = seed;
    c.stored_frac = stored_frac;
    c.n_threads = n_threads < 1 ? 1 : n_threads > 256 ? 256 : n_threads;
    c.n_barcodes = n_barcodes > 0 ? n_barcodes : 1000;
    if (shape == 0) {
        c.n_refs = 1;
        c.ref_len[0] = 1000000;
    } else {
        c.n_refs = 25;
        for (int i = 0; i < 25; i++) c.ref_len[i] = HUMAN[i];
    }
    for (int i = 0; i < c.n_refs; i++) c.cum[i + 1] = c.cum[i] + c.ref_len[i];
    c.genome = c.cum[c.n_refs];
    rng_t g;
    rng_seed(&g, seed, 0xFFFFFFFFull);
    c.barcodes = (char*)malloc((size_t)c.n_barcodes * 16);
    for (int i = 0; i < c.n_barcodes * 16; i++) c.barcodes[i] = "ACGT"[next_u64(&g) & 3];
    c.genes = (char*)calloc(30000, 12);
    c.gene_len = (uint8_t*)malloc(30000);
    static const char* syl[16] = {"A", "B", "C", "D", "E", "F", "G", "K", "L", "M", "N", "P", "R", "S", "T", "Z"};
    for (int i = 0; i < 30000; i++) {
        int len = 3 + (int)below(&g, 6);
        char* s = c.genes + 12 * i;
        int k = 0;
        for (; k < len - 2; k++) s[k] = syl[below(&g, 16)][0];
        snprintf(s + k, 12 - (size_t)k, "%d", (int)below(&g, 99) + 1);
        c.gene_len[i] = (uint8_t)strlen(s);
    }
    FILE* f = fopen(path, "wb");
    if (!f) return 1;
    /* header member */
    buf_t hdr = {0, 0, 0};
    char text[4096];
    int tl = snprintf(text, sizeof(text), "@HD\tVN:1.6\tSO:coordinate\n");
    for (int i = 0; i < c.n_refs; i++)
        tl += snprintf(text + tl, sizeof(text) - (size_t)tl, "@SQ\tSN:%s\tLN:%lld\n", shape == 0 ? "chr1" : HUMAN_NAMES[i],
                       (long long)c.ref_len[i]);
    reserve(&hdr, 12 + tl + 25 * 32);
    memcpy(hdr.p, "BAM\1", 4);
    put32(hdr.p + 4, (uint32_t)tl);
    memcpy(hdr.p + 8, text, (size_t)tl);
    hdr.n = 8 + tl;
    put32(hdr.p + hdr.n, (uint32_t)c.n_refs);
    hdr.n += 4;
    for (int i = 0; i < c.n_refs; i++) {
        const char* nm = shape == 0 ? "chr1" : HUMAN_NAMES[i];
        int ln = (int)strlen(nm) + 1;
        put32(hdr.p + hdr.n, (uint32_t)ln);
        memcpy(hdr.p + hdr.n + 4, nm, (size_t)ln);
        put32(hdr.p + hdr.n + 4 + ln, (uint32_t)c.ref_len[i]);
        hdr.n += 8 + ln;
    }
    uint8_t* hm = (uint8_t*)malloc((size_t)hdr.n + 1024);
    int64_t file_bytes = 0, members = 0, rec_bytes = 0;
    int64_t hb = member(hdr.p, hdr.n, level >= 0 ? level : 6, hm);
    fwrite(hm, 1, (size_t)hb, f);
    file_bytes += hb;
    members++;
    free(hm);
    free(hdr.p);
    /* records, wave by wave */
    int64_t n_seg = (n_records + SEG_RECORDS - 1) / SEG_RECORDS;
    buf_t carry = {0, 0, 0};
    int64_t member_index = 1;
    for (int64_t s0 = 0; s0 < n_seg; s0 += c.n_threads) {
        int64_t ns = n_seg - s0 < c.n_threads ? n_seg - s0 : c.n_threads;
        gtask_t* gt = (gtask_t*)calloc((size_t)ns, sizeof(gtask_t));
        pthread_t th[256];
        for (int64_t k = 0; k < ns; k++) {
            gt[k].c = &c;
            gt[k].seg = s0 + k;
            gt[k].n_seg = n_seg;
            pthread_create(&th[k], NULL, gen_worker, &gt[k]);
        }
        for (int64_t k = 0; k < ns; k++) pthread_join(th[k], NULL);
        buf_t all = {0, 0, 0};
        int64_t tot = carry.n;
        for (int64_t k = 0; k < ns; k++) tot += gt[k].out.n;
        reserve(&all, tot);
        memcpy(all.p, carry.p, (size_t)carry.n);
        all.n = carry.n;
        for (int64_t k = 0; k < ns; k++) {
            memcpy(all.p + all.n, gt[k].out.p, (size_t)gt[k].out.n);
            all.n += gt[k].out.n;
            rec_bytes += gt[k].out.n;
            free(gt[k].out.p);
        }
        free(gt);
        int last = s0 + ns >= n_seg;
        int64_t full = last ? (all.n + BLOCK - 1) / BLOCK : all.n / BLOCK;
        int64_t used = last ? all.n : full * BLOCK;
        uint8_t** outs = (uint8_t**)calloc((size_t)(full + 1), sizeof(uint8_t*));
        int64_t* outn = (int64_t*)calloc((size_t)(full + 1), sizeof(int64_t));
        ztask_t zt[256];
        int nt = c.n_threads;
        for (int k = 0; k < nt; k++) {
            ztask_t t = {&c, all.p, full, used, full * k / nt, full * (k + 1) / nt, outs, outn, 0, member_index};
            zt[k] = t;
            pthread_create(&th[k], NULL, compress_worker, &zt[k]);
        }
        for (int k = 0; k < nt; k++) pthread_join(th[k], NULL);
        for (int64_t k = 0; k < full; k++) {
            fwrite(outs[k], 1, (size_t)outn[k], f);
            file_bytes += outn[k];
            free(outs[k]);
        }
        members += full;
        member_index += full;
        free(outs);
        free(outn);
        carry.n = 0;
        reserve(&carry, all.n - used);
        memcpy(carry.p, all.p + used, (size_t)(all.n - used));
        carry.n = all.n - used;
        free(all.p);
    }
    static const uint8_t eofm[28] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67, 2, 0, 27, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    fwrite(eofm, 1, 28, f);
    file_bytes += 28;
    members++;
    fclose(f);
    free(carry.p);
    free(c.barcodes);
    free(c.genes);
    free(c.gene_len);
    if (out_record_bytes) *out_record_bytes = rec_bytes;
    if (out_members) *out_members = members;
    if (out_file_bytes) *out_file_bytes = file_bytes;
    return 0;
}
