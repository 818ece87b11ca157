// Host model of cb_deflate_spans' DEFLATE coder: the same algorithm as the k_deflate kernel
// (cubam_b200/csrc/deflate.cu), step by step on one thread, so that its output is the kernel's
// output byte for byte.  TEST INFRASTRUCTURE: built and run by tests/test_gpu_writer.py, which
// compares every stream the GPU writes with this one.
//
// Per span: 512-position tiles; per position the hash of its 4 bytes; candidates are the nearest
// earlier position of the same hash among the 32 positions of its warp and the hash head of
// earlier tiles (updated after the tile by the last position of each hash and warp, the larger
// position winning); the longer match of at least 4 bytes is kept (the warp's on ties); with
// level >= 2 a position whose successor has a longer match is a literal; the greedy parse follows
// the steps from the tile's entry.  Then minimum-redundancy code lengths limited to 15 / 7 bits,
// run-length coded lengths, and the smallest of a dynamic, a fixed and a stored block.
//
// usage: deflate_model <input file> <spans file: int64 off, int64 size pairs> <level> <output file>
// output: for each span a uint32 length then the stream's bytes.

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../cubam_b200/csrc/deflate_codes.cuh"

using namespace cb::dfl;

constexpr int NT = 512, HB = 13, NH = 1 << HB, MIN_MATCH = 4, MAX_MATCH = 258, WSIZE = 32768;

static uint32_t u32at(const std::vector<uint8_t>& b, uint32_t i) {
    uint32_t v = 0;
    for (int k = 0; k < 4; k++) v |= (uint32_t)(i + k < b.size() ? b[i + k] : 0) << (8 * k);
    return v;
}
static uint32_t match_len(const std::vector<uint8_t>& b, uint32_t p, uint32_t c, uint32_t maxl) {
    uint32_t L = 0;
    while (L < maxl && b[p + L] == b[c + L]) L++;
    return L;
}

struct Bits {
    std::vector<uint32_t> w;
    void put(uint32_t pos, uint32_t v, uint32_t nb) {
        if (!nb) return;
        uint32_t wi = pos >> 5, s = pos & 31;
        if (w.size() < wi + 3) w.resize(wi + 3, 0);
        uint64_t x = (uint64_t)v << s;
        w[wi] |= (uint32_t)x;
        if (s + nb > 32) w[wi + 1] |= (uint32_t)(x >> 32);
    }
};

std::vector<uint8_t> model(const std::vector<uint8_t>& in, int level, int* kind_out = nullptr) {
    const uint32_t n = in.size();
    std::vector<uint8_t> buf(in);
    buf.resize(n + 16, 0);
    std::vector<uint32_t> head(NH, 0), toks;
    uint32_t lfreq[288] = {0}, dfreq[32] = {0};
    uint32_t entry = 0;
    std::vector<uint32_t> mt(NT), jmp0(NT);
    for (uint32_t T0 = 0; T0 < n; T0 += NT) {
        const uint32_t tend = std::min<uint32_t>(NT, n - T0);
        std::vector<uint32_t> key(NT), hv(NT), hh(NT);
        std::vector<bool> v4(NT);
        for (int t = 0; t < NT; t++) {
            uint32_t p = T0 + t;
            v4[t] = level > 0 && p + 4 <= n;
            uint32_t cur = v4[t] ? u32at(buf, p) : 0;
            hh[t] = (cur * 0x9E3779B1u) >> (32 - HB);
            key[t] = v4[t] ? hh[t] : (0x80000000u | t);
            hv[t] = v4[t] ? head[hh[t]] : 0;
        }
        for (int t = 0; t < NT; t++) {
            int lane = t & 31, wbase = t - lane;
            bool highest = true;
            for (int l = lane + 1; l < 32; l++)
                if (key[wbase + l] == key[t]) highest = false;
            if (v4[t] && highest) head[hh[t]] = std::max(head[hh[t]], T0 + t + 1);
            uint32_t best = 0, p = T0 + t;
            if (v4[t]) {
                uint32_t maxl = std::min<uint32_t>(MAX_MATCH, n - p);
                int below = -1;
                for (int l = lane - 1; l >= 0; l--)
                    if (key[wbase + l] == key[t]) {
                        below = l;
                        break;
                    }
                if (below >= 0) {
                    uint32_t c = p - lane + below;
                    uint32_t L = match_len(buf, p, c, maxl);
                    if (L >= MIN_MATCH) best = (L << 16) | (p - c);
                }
                if (hv[t]) {
                    uint32_t c = hv[t] - 1;
                    if (p - c <= WSIZE) {
                        uint32_t L = match_len(buf, p, c, maxl);
                        if (L >= MIN_MATCH && L > (best >> 16)) best = (L << 16) | (p - c);
                    }
                }
            }
            mt[t] = best;
        }
        for (uint32_t t = 0; t < NT; t++) {
            uint32_t step = 1;
            if (t < tend && mt[t]) {
                step = mt[t] >> 16;
                if (level >= 2 && t + 1 < tend && (mt[t + 1] >> 16) > step) step = 1;
            }
            jmp0[t] = t < tend ? t + step : NT;
        }
        uint32_t pos = entry;
        int exitp = 0;
        while (pos < tend) {
            uint32_t nx = jmp0[pos], st = nx - pos;
            if (st >= MIN_MATCH) {
                uint32_t d = mt[pos] & 0xFFFF;
                toks.push_back(0x80000000u | (st << 16) | (d - 1));
                lfreq[len_sym(st)]++;
                dfreq[dist_sym(d)]++;
            } else {
                toks.push_back(buf[T0 + pos]);
                lfreq[buf[T0 + pos]]++;
            }
            if (nx >= tend) exitp = (int)nx - NT;
            pos = nx;
        }
        entry = exitp > 0 ? exitp : 0;
    }
    lfreq[256] = 1;
    auto sorted_of = [](const uint32_t* f, int ns, std::vector<uint16_t>& out) {
        out.clear();
        for (int s = 0; s < ns; s++)
            if (f[s]) out.push_back(s);
        std::stable_sort(out.begin(), out.end(), [&](uint16_t a, uint16_t b) { return f[a] < f[b]; });
    };
    std::vector<uint16_t> ls, ds, cs;
    sorted_of(lfreq, NLIT, ls);
    sorted_of(dfreq, NDIST, ds);
    uint32_t A[320];
    uint8_t llen[288] = {0}, dlen[32] = {0}, cllen[20] = {0};
    build_lengths(lfreq, ls.data(), ls.size(), NLIT_ALL, A, llen, MAXBITS);
    build_lengths(dfreq, ds.data(), ds.size(), NDIST, A, dlen, MAXBITS);
    int hlit = NLIT;
    while (hlit > 257 && llen[hlit - 1] == 0) hlit--;
    int hdist = NDIST;
    while (hdist > 1 && dlen[hdist - 1] == 0) hdist--;
    uint8_t rsym[NRLE], rext[NRLE];
    int nrle = rle_lengths(llen, hlit, dlen, hdist, rsym, rext);
    uint32_t clfreq[20] = {0};
    for (int k = 0; k < nrle; k++) clfreq[rsym[k]]++;
    sorted_of(clfreq, NCL, cs);
    build_lengths(clfreq, cs.data(), cs.size(), NCL, A, cllen, CLBITS);
    int hclen = NCL;
    while (hclen > 4 && cllen[cl_order(hclen - 1)] == 0) hclen--;
    uint64_t hdr = 3 + 14 + 3 * hclen;
    for (int k = 0; k < nrle; k++) hdr += cllen[rsym[k]] + cl_extra_bits(rsym[k]);
    uint64_t dyn = hdr, fix = 3;
    for (int s = 0; s < NLIT; s++) {
        uint32_t e = s > 256 ? len_extra_bits(s) : 0;
        dyn += (uint64_t)lfreq[s] * (llen[s] + e);
        fix += (uint64_t)lfreq[s] * (fixed_lit_len(s) + e);
    }
    for (int d = 0; d < NDIST; d++) {
        dyn += (uint64_t)dfreq[d] * (dlen[d] + dist_extra_bits(d));
        fix += (uint64_t)dfreq[d] * (FIXED_DIST_LEN + dist_extra_bits(d));
    }
    uint32_t nblk = n ? (n + 65534) / 65535 : 1;
    uint64_t stored = n + 5ull * nblk;
    uint64_t bdyn = (dyn + 7) / 8, bfix = (fix + 7) / 8;
    int kind = bfix <= bdyn ? 1 : 2;
    uint64_t bits = kind == 1 ? fix : dyn;
    if (stored < (bits + 7) / 8) kind = 0;
    if (kind_out) *kind_out = kind;
    std::vector<uint8_t> out;
    if (kind == 0) {
        for (uint32_t b = 0; b < nblk; b++) {
            uint32_t len = std::min<uint32_t>(65535, n - b * 65535);
            out.push_back(b + 1 == nblk ? 1 : 0);
            out.push_back(len & 255);
            out.push_back(len >> 8);
            out.push_back(~len & 255);
            out.push_back((~len >> 8) & 255);
            out.insert(out.end(), in.begin() + b * 65535, in.begin() + b * 65535 + len);
        }
        return out;
    }
    if (kind == 1) {
        for (int s = 0; s < NLIT_ALL; s++) llen[s] = fixed_lit_len(s);
        for (int d = 0; d < NDIST; d++) dlen[d] = FIXED_DIST_LEN;
    }
    uint32_t lcode[288], dcode[32], clcode[20];
    canonical_codes(llen, NLIT_ALL, lcode);
    canonical_codes(dlen, NDIST, dcode);
    Bits B;
    uint32_t pos = 0;
    auto put = [&](uint32_t v, uint32_t nb) {
        B.put(pos, v, nb);
        pos += nb;
    };
    if (kind == 1) {
        put(1 | (1 << 1), 3);
    } else {
        canonical_codes(cllen, NCL, clcode);
        put(1 | (2 << 1), 3);
        put(hlit - 257, 5);
        put(hdist - 1, 5);
        put(hclen - 4, 4);
        for (int i = 0; i < hclen; i++) put(cllen[cl_order(i)], 3);
        for (int k = 0; k < nrle; k++) {
            uint32_t c = clcode[rsym[k]];
            put(c & 0xFFFF, c >> 16);
            put(rext[k], cl_extra_bits(rsym[k]));
        }
    }
    if (pos != (kind == 1 ? 3 : hdr)) {
        fprintf(stderr, "header bits %u vs %llu\n", pos, (unsigned long long)hdr);
        exit(1);
    }
    for (uint32_t tk : toks) {
        if (tk & 0x80000000u) {
            uint32_t L = (tk >> 16) & 0x1FF, d = (tk & 0xFFFF) + 1;
            uint32_t ls_ = len_sym(L), c = lcode[ls_];
            put(c & 0xFFFF, c >> 16);
            put(len_extra_val(L), len_extra_bits(ls_));
            uint32_t ds_ = dist_sym(d), e = dcode[ds_];
            put(e & 0xFFFF, e >> 16);
            put(dist_extra_val(d), dist_extra_bits(ds_));
        } else {
            uint32_t c = lcode[tk];
            put(c & 0xFFFF, c >> 16);
        }
    }
    put(lcode[256] & 0xFFFF, lcode[256] >> 16);
    if (pos != bits) {
        fprintf(stderr, "bits %u vs %llu (kind %d)\n", pos, (unsigned long long)bits, kind);
        exit(1);
    }
    uint32_t nbytes = (pos + 7) / 8;
    out.resize(nbytes);
    for (uint32_t i = 0; i < nbytes; i++) out[i] = (B.w[i >> 2] >> (8 * (i & 3))) & 255;
    return out;
}


static std::vector<uint8_t> read_all(const char* path) {
    std::vector<uint8_t> v;
    FILE* f = fopen(path, "rb");
    if (!f) exit(2);
    static uint8_t buf[1 << 16];
    size_t r;
    while ((r = fread(buf, 1, sizeof buf, f)) > 0) v.insert(v.end(), buf, buf + r);
    fclose(f);
    return v;
}

int main(int argc, char** argv) {
    if (argc != 5) return 2;
    const std::vector<uint8_t> data = read_all(argv[1]);
    const std::vector<uint8_t> sp = read_all(argv[2]);
    const int level = atoi(argv[3]);
    FILE* out = fopen(argv[4], "wb");
    if (!out) return 2;
    for (size_t k = 0; k + 16 <= sp.size(); k += 16) {
        int64_t off, size;
        memcpy(&off, sp.data() + k, 8);
        memcpy(&size, sp.data() + k + 8, 8);
        if (off < 0 || size < 0 || (uint64_t)(off + size) > data.size()) return 3;
        std::vector<uint8_t> in(data.begin() + off, data.begin() + off + size);
        const std::vector<uint8_t> c = model(in, level);
        const uint32_t n = (uint32_t)c.size();
        fwrite(&n, 4, 1, out);
        fwrite(c.data(), 1, c.size(), out);
    }
    fclose(out);
    return 0;
}
