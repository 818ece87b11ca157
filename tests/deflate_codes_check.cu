// Host checks of the DEFLATE code construction the compressor kernel uses (deflate_codes.cuh),
// built and run by tests/test_deflate_codes_host.py with nvcc as a host program (no GPU):
//  1. the count-based lengths of the kernel (internal-node depths -> leaves per depth -> limit ->
//     length by rank) equal the serial Moffat-Katajainen + limit lengths, on random, skewed and
//     Fibonacci-like frequency tables;
//  2. every such code is complete (Kraft sum exactly 1) and within its length limit, and the
//     Huffman lengths before limiting are optimal (equal total cost to a reference Huffman build);
//  3. the per-run coding of code lengths equals rle_lengths over whole sequences;
//  4. length/distance symbols, extra bits and values agree with RFC 1951's tables.
#include <algorithm>
#include <cstdio>
#include <queue>
#include <random>
#include <vector>

#include "../cubam_b200/csrc/deflate_codes.cuh"

using namespace cb::dfl;

static int failures = 0;
#define CHECK(cond, ...)                      \
    do {                                      \
        if (!(cond)) {                        \
            if (failures++ < 10) {            \
                printf("FAIL: " __VA_ARGS__); \
                printf("\n");                 \
            }                                 \
        }                                     \
    } while (0)

static std::vector<uint16_t> sorted_of(const std::vector<uint32_t>& f) {
    std::vector<uint16_t> s;
    for (size_t i = 0; i < f.size(); i++)
        if (f[i]) s.push_back((uint16_t)i);
    std::stable_sort(s.begin(), s.end(), [&](uint16_t a, uint16_t b) { return f[a] < f[b]; });
    return s;
}

// The kernel's route (par_lengths), step by step on the host.
static void count_based(const std::vector<uint32_t>& f, uint32_t L, uint8_t* len) {
    const int nsym = (int)f.size();
    std::vector<uint16_t> sorted = sorted_of(f);
    const int m = (int)sorted.size();
    for (int s = 0; s < nsym; s++) len[s] = 0;
    if (m < 2) {
        if (m == 0) len[0] = len[1] = 1;
        else {
            len[sorted[0]] = 1;
            len[sorted[0] == 0 ? 1 : 0] = 1;
        }
        return;
    }
    std::vector<uint32_t> A(m);
    for (int i = 0; i < m; i++) A[i] = f[sorted[i]];
    mk_pass1(A.data(), m);
    const int ni = m - 1, root = m - 2;
    std::vector<uint32_t> anc(ni), dep(ni), anc2(ni), dep2(ni);
    for (int i = 0; i < ni; i++) {
        anc[i] = i == root ? i : A[i];
        dep[i] = i == root ? 0 : 1;
    }
    for (int r = 0; r < 9; r++) {
        for (int i = 0; i < ni; i++) {
            dep2[i] = dep[i] + dep[anc[i]];
            anc2[i] = anc[anc[i]];
        }
        anc.swap(anc2);
        dep.swap(dep2);
    }
    std::vector<uint32_t> c(m + 2, 0);
    int maxd = 0;
    for (int i = 0; i < ni; i++) {
        c[dep[i]]++;
        maxd = std::max<int>(maxd, (int)dep[i]);
    }
    uint32_t cum[16];
    lengths_from_depths(c.data(), maxd, L, cum);
    for (int i = 0; i < m; i++) len[sorted[i]] = (uint8_t)length_of_rank((uint32_t)(m - 1 - i), cum);
}

static uint64_t huffman_cost(const std::vector<uint32_t>& f) {  // optimal total bits (no length limit)
    std::priority_queue<uint64_t, std::vector<uint64_t>, std::greater<uint64_t>> q;
    for (uint32_t x : f)
        if (x) q.push(x);
    if (q.size() < 2) return q.empty() ? 0 : q.top();
    uint64_t cost = 0;
    while (q.size() > 1) {
        uint64_t a = q.top();
        q.pop();
        uint64_t b = q.top();
        q.pop();
        cost += a + b;
        q.push(a + b);
    }
    return cost;
}

int main() {
    std::mt19937_64 rng(11);
    static const uint32_t fib[] = {1,    1,    2,    3,    5,    8,     13,    21,    34,    55,    89,   144,
                                   233,  377,  610,  987,  1597, 2584,  4181,  6765,  10946, 17711, 28657};
    int limited = 0;
    for (int trial = 0; trial < 60000; trial++) {
        const int nsym = trial % 3 == 0 ? 19 : trial % 3 == 1 ? 30 : 286;
        const uint32_t L = nsym == 19 ? CLBITS : MAXBITS;
        std::vector<uint32_t> f(nsym, 0);
        const int mode = (int)(rng() % 5);
        for (int s = 0; s < nsym; s++) {
            if (rng() % 3 == 0) continue;
            if (mode == 0) f[s] = 1 + rng() % 10;
            else if (mode == 1) f[s] = 1 + rng() % 100000;
            else if (mode == 2) f[s] = 1u << (rng() % 20);
            else if (mode == 3) f[s] = fib[rng() % 23];
            else f[s] = (rng() % 7 == 0) ? 5000 + rng() % 50000 : 1 + rng() % 3;
        }
        std::vector<uint16_t> sorted = sorted_of(f);
        std::vector<uint32_t> A(nsym + 2);
        uint8_t serial[288], counted[288];
        build_lengths(f.data(), sorted.data(), (int)sorted.size(), nsym, A.data(), serial, L);
        count_based(f, L, counted);
        bool same = true;
        for (int s = 0; s < nsym; s++) same &= serial[s] == counted[s];
        CHECK(same, "count-based lengths differ (trial %d, %d symbols, mode %d)", trial, nsym, mode);
        // complete and limited
        uint64_t kraft = 0, cost = 0;
        uint32_t maxlen = 0;
        for (int s = 0; s < nsym; s++) {
            if (!counted[s]) continue;
            kraft += 1ull << (15 - counted[s]);
            maxlen = std::max<uint32_t>(maxlen, counted[s]);
            cost += (uint64_t)f[s] * counted[s];
        }
        CHECK(kraft == (1ull << 15), "code not complete (trial %d)", trial);
        CHECK(maxlen <= L, "length %u over %u (trial %d)", maxlen, L, trial);
        // optimal when the limit did not bind
        if (sorted.size() >= 2) {
            std::vector<uint32_t> B(sorted.size());
            for (size_t i = 0; i < sorted.size(); i++) B[i] = f[sorted[i]];
            mk_lengths(B.data(), (int)B.size());
            if (B[0] <= L) CHECK(cost == huffman_cost(f), "not minimum-redundancy (trial %d)", trial);
            else limited++;
        }
    }
    // run-length coding
    for (int trial = 0; trial < 30000; trial++) {
        const int hlit = 257 + (int)(rng() % 30), hdist = 1 + (int)(rng() % 30);
        uint8_t lit[288], dist[32];
        const int mode = (int)(rng() % 3);
        for (int i = 0; i < hlit; i++)
            lit[i] = mode == 0 ? rng() % 16 : (rng() % 4 == 0 ? rng() % 16 : (mode == 1 ? 0 : 8));
        for (int i = 0; i < hdist; i++) dist[i] = rng() % 3 == 0 ? 0 : 5;
        uint8_t s1[NRLE], e1[NRLE], s2[NRLE], e2[NRLE];
        const int n1 = rle_lengths(lit, hlit, dist, hdist, s1, e1);
        int n2 = 0;
        const int T = hlit + hdist;
        auto at = [&](int i) { return i < hlit ? lit[i] : dist[i - hlit]; };
        for (int i = 0; i < T;) {
            int r = 1;
            while (i + r < T && at(i + r) == at(i)) r++;
            n2 += rle_run(at(i), r, s2 + n2, e2 + n2);
            i += r;
        }
        bool same = n1 == n2 && n1 <= NRLE;
        for (int k = 0; same && k < n1; k++) same = s1[k] == s2[k] && e1[k] == e2[k];
        CHECK(same, "run coding differs (trial %d)", trial);
        // the symbols expand back to the lengths
        std::vector<uint8_t> back;
        for (int k = 0; k < n1; k++) {
            if (s1[k] < 16) back.push_back(s1[k]);
            else if (s1[k] == 16) back.insert(back.end(), 3 + e1[k], back.back());
            else back.insert(back.end(), (s1[k] == 17 ? 3 : 11) + e1[k], 0);
        }
        bool round = (int)back.size() == T;
        for (int i = 0; round && i < T; i++) round = back[i] == at(i);
        CHECK(round, "run coding does not expand back (trial %d)", trial);
    }
    // RFC 1951 3.2.5 tables
    static const uint16_t lbase[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                       31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
    static const uint8_t lext[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
    static const uint16_t dbase[30] = {1,    2,    3,    4,    5,    7,    9,    13,    17,    25,
                                       33,   49,   65,   97,   129,  193,  257,  385,   513,   769,
                                       1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
    for (uint32_t len = 3; len <= 258; len++) {
        const uint32_t s = len_sym(len), k = s - 257;
        CHECK(k < 29 && lbase[k] <= len && len - lbase[k] < (1u << lext[k]) && len_extra_bits(s) == lext[k] &&
                  len_extra_val(len) == len - lbase[k],
              "length %u", len);
    }
    for (uint32_t d = 1; d <= 32768; d++) {
        const uint32_t s = dist_sym(d);
        const uint32_t e = s < 30 ? dist_extra_bits(s) : 99;
        CHECK(s < 30 && dbase[s] <= d && d - dbase[s] < (1u << e) && dist_extra_val(d) == d - dbase[s], "distance %u", d);
    }
    printf("%d failures (%d limited codes)\n", failures, limited);
    return failures != 0;
}
