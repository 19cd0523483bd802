// steppecu_b200/csrc/host_mirror.cpp
//
// Host side of the band download (stp_f2_extract_blocks with host output): every P x P f2 /
// vpair slab is exactly symmetric, so only its upper row bands cross PCIe and the host fills
// the lower tiles by transposition. Column-major slab: element (i, j) at i + P * j. Band t
// holds rows [t*T, t*T + T) x columns [t*T, P); below each band's diagonal tile, rows past
// the band x the band's columns are the transpose of the block right of that tile.
//
// With AVX2, 32-byte aligned slabs and P % 4 == 0, 4 x 4 blocks are transposed in registers
// and written with streaming stores (no read-for-ownership of the lines being written);
// otherwise 32 x 32 scalar sub-blocks.
#include <immintrin.h>

#include <algorithm>
#include <cstdint>

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

}  // namespace

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
