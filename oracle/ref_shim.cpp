// Host build of the reference's reader kernels: TEST INFRASTRUCTURE ONLY.
//
// cubam keeps its CUDA kernels as a C++ string (src/cubam/_kernels.py:7-622).
// oracle/build_ref.py extracts that string, unchanged, into oracle/_ref/ref_kernels.inc
// (git-ignored, never committed), and this file compiles it for the CPU: the CUDA
// qualifiers become plain C++ and every thread of a launch runs one after the other.
// Warp intrinsics are given their single-lane meaning, which is exact for the
// kernels called here: warp_append (src/cubam/_kernels.py:19-31) then appends each
// passing offset on its own, and the callers sort the offsets anyway
// (src/cubam/_kernels.py:662-673).  crc32_spans needs a real warp and is not called.
//
// Entry point: ref_launch(name, n_threads, args), args as cuLaunchKernel passes
// them (an array of pointers to the argument values).

#include <cstdint>
#include <cstring>
#include <string>
#include <string_view>

struct Dim3Host { unsigned int x, y, z; };
static thread_local Dim3Host threadIdx, blockIdx, blockDim;

#define __global__
#define __device__
#define __forceinline__ inline
#define __shared__ static

static inline void __syncthreads() {}
static inline unsigned int __ballot_sync(unsigned int, bool r) { return r ? (1u << (threadIdx.x & 31)) : 0u; }
static inline int __ffs(unsigned int x) { return x ? __builtin_ctz(x) + 1 : 0; }
static inline int __popc(unsigned int x) { return __builtin_popcount(x); }
static inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
    unsigned long long o = *p;
    *p = o + v;
    return o;
}
template <class T> static inline T __shfl_sync(unsigned int, T v, int) { return v; }
template <class T> static inline T __shfl_xor_sync(unsigned int, T v, int) { return v; }
static inline unsigned int __float_as_uint(float f) {
    unsigned int u;
    std::memcpy(&u, &f, 4);
    return u;
}

#include "ref_kernels.inc"

namespace {

template <class T> inline T A(void** a, int i) { return *reinterpret_cast<T*>(a[i]); }

template <class F> void run(long long n_threads, F&& f) {
    blockDim = {256, 1, 1};
    long long blocks = (n_threads + 255) / 256;
    for (long long b = 0; b < blocks; b++) {
        blockIdx = {static_cast<unsigned int>(b), 0, 0};
        for (unsigned int t = 0; t < 256; t++) {
            threadIdx = {t, 0, 0};
            f();
        }
    }
}

typedef const unsigned char* cu8p;
typedef unsigned char* u8p;
typedef const long long* ci64p;
typedef long long* i64p;
typedef long long i64;

}  // namespace

extern "C" int ref_launch(const char* name, long long n_threads, void** a) {
    std::string_view k(name);
    if (k == "copy_spans") {
        run(n_threads, [&] { copy_spans(A<cu8p>(a, 0), A<u8p>(a, 1), A<ci64p>(a, 2), A<ci64p>(a, 3), A<ci64p>(a, 4), A<i64>(a, 5)); });
    } else if (k == "bgzf_candidates") {
        run(n_threads, [&] {
            bgzf_candidates(A<cu8p>(a, 0), A<i64>(a, 1), A<i64p>(a, 2), A<unsigned long long>(a, 3),
                            A<unsigned long long*>(a, 4));
        });
    } else if (k == "bgzf_sizes") {
        run(n_threads, [&] { bgzf_sizes(A<cu8p>(a, 0), A<ci64p>(a, 1), A<i64>(a, 2), A<i64p>(a, 3), A<i64p>(a, 4)); });
    } else if (k == "record_candidates") {
        run(n_threads, [&] {
            record_candidates(A<cu8p>(a, 0), A<i64>(a, 1), A<int>(a, 2), A<i64p>(a, 3), A<unsigned long long>(a, 4),
                              A<unsigned long long*>(a, 5));
        });
    } else if (k == "record_ends") {
        run(n_threads, [&] { record_ends(A<cu8p>(a, 0), A<ci64p>(a, 1), A<i64>(a, 2), A<i64p>(a, 3)); });
    } else if (k == "decode_fixed") {
        run(n_threads, [&] {
            decode_fixed(A<cu8p>(a, 0), A<ci64p>(a, 1), A<i64>(a, 2), A<int*>(a, 3), A<int*>(a, 4), A<int*>(a, 5),
                         A<unsigned char*>(a, 6), A<unsigned short*>(a, 7), A<int*>(a, 8), A<int*>(a, 9),
                         A<int*>(a, 10), A<int*>(a, 11), A<unsigned short*>(a, 12), A<unsigned short*>(a, 13));
        });
    } else if (k == "name_hash") {
        run(n_threads, [&] { name_hash(A<cu8p>(a, 0), A<ci64p>(a, 1), A<i64>(a, 2), A<unsigned long long*>(a, 3)); });
    } else if (k == "find_tag") {
        run(n_threads, [&] {
            find_tag(A<cu8p>(a, 0), A<ci64p>(a, 1), A<i64>(a, 2), A<unsigned char>(a, 3), A<unsigned char>(a, 4),
                     A<unsigned char*>(a, 5), A<i64p>(a, 6), A<int*>(a, 7), A<i64p>(a, 8));
        });
    } else if (k == "aligned_len") {
        run(n_threads, [&] { aligned_len(A<cu8p>(a, 0), A<ci64p>(a, 1), A<i64>(a, 2), A<int*>(a, 3)); });
    } else if (k == "blocks") {
        run(n_threads, [&] {
            blocks(A<cu8p>(a, 0), A<ci64p>(a, 1), A<i64>(a, 2), A<int>(a, 3), A<int>(a, 4), A<ci64p>(a, 5),
                   A<int*>(a, 6), A<i64p>(a, 7), A<int*>(a, 8), A<int*>(a, 9));
        });
    } else if (k == "base_at") {
        run(n_threads, [&] {
            base_at(A<cu8p>(a, 0), A<ci64p>(a, 1), A<ci64p>(a, 2), A<const int*>(a, 3), A<i64>(a, 4),
                    A<signed char*>(a, 5));
        });
    } else if (k == "hash_spans") {
        run(n_threads, [&] {
            hash_spans(A<cu8p>(a, 0), A<ci64p>(a, 1), A<const int*>(a, 2), A<i64>(a, 3), A<unsigned long long*>(a, 4));
        });
    } else if (k == "pack_acgt") {
        run(n_threads, [&] {
            pack_acgt(A<cu8p>(a, 0), A<ci64p>(a, 1), A<const int*>(a, 2), A<i64>(a, 3), A<unsigned long long*>(a, 4),
                      A<unsigned char*>(a, 5));
        });
    } else if (k == "unpack_acgt") {
        run(n_threads, [&] {
            unpack_acgt(A<const unsigned long long*>(a, 0), A<ci64p>(a, 1), A<i64>(a, 2), A<unsigned char*>(a, 3));
        });
    } else {
        return 1;
    }
    return 0;
}
