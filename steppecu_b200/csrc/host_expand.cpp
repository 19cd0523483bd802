// steppecu_b200/csrc/host_expand.cpp
//
// Host side of the host-output path's vpair transfer (stpf2_abi.cu: contract_segments): the
// upper 128 x 128 tiles of each P x P count slab arrive packed as 16-bit (or 32-bit)
// integers in counts_pack.cu's order, and are widened here to FP64 into both halves of the
// exactly symmetric, column-major slab (element (i, j) at i + P * j): tile (ti, tj) to rows
// ti*128.. x columns tj*128.., and off the diagonal its transpose as well.
//
// With AVX2, 32-byte aligned slabs and P % 4 == 0, four counts are widened per instruction
// and written with streaming stores (no read-for-ownership of the lines being written);
// otherwise element by element.
#include <immintrin.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace stpf2 {

namespace {

// Widening of packed counts (counts_pack.cu): 4 counts at a time with AVX2.
template <class In>
__attribute__((target("avx2"))) inline __m256d widen4(const In* p) {
    if constexpr (sizeof(In) == 2) {
        const __m128i x = _mm_loadl_epi64(reinterpret_cast<const __m128i*>(p));
        return _mm256_cvtepi32_pd(_mm_cvtepu16_epi32(x));
    } else {
        // Counts stay below 2^31 (SNPs of one block), so the signed conversion is exact.
        return _mm256_cvtepi32_pd(_mm_loadu_si128(reinterpret_cast<const __m128i*>(p)));
    }
}

// One run of n counts to n doubles at dst (32-byte aligned, n % 4 == 0), streaming.
template <class In>
__attribute__((target("avx2"))) void widen_run_avx2(const In* src, double* dst, int64_t n) {
    for (int64_t k = 0; k < n; k += 4) _mm256_stream_pd(dst + k, widen4(src + k));
}

template <class In>
void widen_run_scalar(const In* src, double* dst, int64_t n) {
    for (int64_t k = 0; k < n; ++k) dst[k] = static_cast<double>(src[k]);
}

template <class In>
void expand_slab(const In* tiles, double* S, int64_t P, bool avx2) {
    constexpr int64_t T = 128;
    const int64_t nt = (P + T - 1) / T;
    std::vector<In> tr(static_cast<size_t>(T * T));  // one tile, transposed
    int64_t u = 0;
    for (int64_t ti = 0; ti < nt; ++ti)
        for (int64_t tj = ti; tj < nt; ++tj, ++u) {
            const In* t = tiles + u * T * T;
            const int64_t nr = std::min(T, P - ti * T), nc = std::min(T, P - tj * T);
            // (i, j): column tj*T + c, rows ti*T.. of the slab = the tile's column c.
            for (int64_t c = 0; c < nc; ++c) {
                double* dst = S + ti * T + P * (tj * T + c);
#if defined(__x86_64__)
                if (avx2) {
                    widen_run_avx2(t + c * T, dst, nr);
                    continue;
                }
#endif
                widen_run_scalar(t + c * T, dst, nr);
            }
            if (ti == tj) continue;
            // (j, i): column ti*T + r, rows tj*T.. = the tile's row r.
            for (int64_t c = 0; c < nc; ++c)
                for (int64_t r = 0; r < nr; ++r) tr[static_cast<size_t>(r * T + c)] = t[c * T + r];
            for (int64_t r = 0; r < nr; ++r) {
                double* dst = S + tj * T + P * (ti * T + r);
#if defined(__x86_64__)
                if (avx2) {
                    widen_run_avx2(tr.data() + r * T, dst, nc);
                    continue;
                }
#endif
                widen_run_scalar(tr.data() + r * T, dst, nc);
            }
        }
}

}  // namespace

void expand_counts(const void* packed, bool wide, double* S, int64_t P) {
    bool avx2 = false;
#if defined(__x86_64__)
    static const bool has_avx2 = __builtin_cpu_supports("avx2");
    avx2 = has_avx2 && P % 4 == 0 && reinterpret_cast<uintptr_t>(S) % 32 == 0;
#endif
    if (wide) expand_slab(static_cast<const uint32_t*>(packed), S, P, avx2);
    else expand_slab(static_cast<const uint16_t*>(packed), S, P, avx2);
#if defined(__x86_64__)
    if (avx2) _mm_sfence();
#endif
}

}  // namespace stpf2
