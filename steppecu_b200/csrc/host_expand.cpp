// steppecu_b200/csrc/host_expand.cpp
//
// Host side of the host-output path (stpf2_abi.cu: contract_segments). Every P x P slab is
// exactly symmetric and column-major (element (i, j) at i + P * j), so only its upper
// 128 x 128 tiles (row tile <= column tile, diagonal tiles whole) cross PCIe:
// - f2: the upper tiles land in place and mirror_lower_tiles fills the rest by
//   transposition (rows past each band x the band's columns are the transpose of the block
//   right of the band's diagonal tile);
// - vpair: the upper tiles arrive packed as 16-bit (or 32-bit) counts in counts_pack.cu's
//   order, and expand_counts widens them to FP64 into both halves: tile (ti, tj) to rows
//   ti*128.. x columns tj*128.., and off the diagonal its transpose as well.
//
// With AVX2, 32-byte aligned slabs and P % 4 == 0, both use 4-wide vector code with
// streaming stores (no read-for-ownership of the lines being written: 4 x 4 register
// transposes, 4 counts widened per instruction); otherwise element by element.
#include <immintrin.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace stpf2 {

namespace {

void mirror_scalar(double* S, int64_t P, int64_t T) {
    for (int64_t r0 = 0; r0 < P; r0 += T) {
        const int64_t r1 = std::min(P, r0 + T);
        for (int64_t i0 = r1; i0 < P; i0 += 32)
            for (int64_t j0 = r0; j0 < r1; j0 += 32) {
                const int64_t i1 = std::min(P, i0 + 32), j1 = std::min(r1, j0 + 32);
                for (int64_t j = j0; j < j1; ++j)
                    for (int64_t i = i0; i < i1; ++i) S[i + P * j] = S[j + P * i];
            }
    }
}

#if defined(__x86_64__)
// Requires P % 4 == 0, T % 4 == 0 and S 32-byte aligned: every range below is then a
// multiple of 4 and every destination S[i + P * j] with i % 4 == 0 is 32-byte aligned.
__attribute__((target("avx2"))) void mirror_avx2(double* S, int64_t P, int64_t T) {
    for (int64_t r0 = 0; r0 < P; r0 += T) {
        const int64_t r1 = std::min(P, r0 + T);
        for (int64_t i0 = r1; i0 < P; i0 += 32)
            for (int64_t j0 = r0; j0 < r1; j0 += 32) {
                const int64_t i1 = std::min(P, i0 + 32), j1 = std::min(r1, j0 + 32);
                for (int64_t j = j0; j < j1; j += 4)
                    for (int64_t i = i0; i < i1; i += 4) {
                        // rows j..j+3 of columns i..i+3 (contiguous in the column)
                        const __m256d a0 = _mm256_loadu_pd(S + j + P * (i + 0));
                        const __m256d a1 = _mm256_loadu_pd(S + j + P * (i + 1));
                        const __m256d a2 = _mm256_loadu_pd(S + j + P * (i + 2));
                        const __m256d a3 = _mm256_loadu_pd(S + j + P * (i + 3));
                        const __m256d t0 = _mm256_unpacklo_pd(a0, a1), t1 = _mm256_unpackhi_pd(a0, a1);
                        const __m256d t2 = _mm256_unpacklo_pd(a2, a3), t3 = _mm256_unpackhi_pd(a2, a3);
                        // column j + m, rows i..i+3
                        _mm256_stream_pd(S + i + P * (j + 0), _mm256_permute2f128_pd(t0, t2, 0x20));
                        _mm256_stream_pd(S + i + P * (j + 1), _mm256_permute2f128_pd(t1, t3, 0x20));
                        _mm256_stream_pd(S + i + P * (j + 2), _mm256_permute2f128_pd(t0, t2, 0x31));
                        _mm256_stream_pd(S + i + P * (j + 3), _mm256_permute2f128_pd(t1, t3, 0x31));
                    }
            }
    }
    _mm_sfence();
}
#endif

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

void mirror_lower_tiles(double* S, int64_t P, int64_t T) {
#if defined(__x86_64__)
    static const bool avx2 = __builtin_cpu_supports("avx2");
    if (avx2 && P % 4 == 0 && T % 4 == 0 && reinterpret_cast<uintptr_t>(S) % 32 == 0) {
        mirror_avx2(S, P, T);
        return;
    }
#endif
    mirror_scalar(S, P, T);
}

}  // namespace stpf2
