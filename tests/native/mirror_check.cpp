// Checker for steppecu_b200/csrc/host_mirror.cpp, built and run by tests/test_host_mirror.py.
//
// For each P (and a 32-byte aligned and a misaligned slab, so that both the AVX2 path and the
// scalar path run where the CPU has AVX2), it builds a symmetric P x P column-major slab,
// keeps only the upper row bands of T = 128 rows (what the band download copies), fills the
// rest with -1, calls mirror_lower_tiles and compares the result with the full slab bit for
// bit. Prints "ok" and exits 0, or names the first failing case and exits 1.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace stpf2 {
void mirror_lower_tiles(double* S, int64_t P, int64_t T);
}

int main() {
    const int64_t T = 128;
    const int64_t sizes[] = {1, 3, 4, 8, 100, 127, 128, 129, 132, 300, 1000, 1001};
    uint64_t state = 20261203;
    auto next = [&state]() {
        state = state * 6364136223846793005ull + 1442695040888963407ull;
        return static_cast<double>(state >> 11) * 0x1.0p-53;
    };
    for (int64_t P : sizes) {
        for (int off = 0; off < 2; ++off) {
            std::vector<double> buf(static_cast<size_t>(P * P + 8));
            const uintptr_t base = (reinterpret_cast<uintptr_t>(buf.data()) + 31) & ~uintptr_t(31);
            double* S = reinterpret_cast<double*>(base) + off;
            std::vector<double> full(static_cast<size_t>(P * P));
            for (int64_t j = 0; j < P; ++j)
                for (int64_t i = 0; i <= j; ++i) {
                    const double v = next();
                    full[i + P * j] = v;
                    full[j + P * i] = v;
                }
            for (int64_t k = 0; k < P * P; ++k) S[k] = -1.0;
            for (int64_t r0 = 0; r0 < P; r0 += T)
                for (int64_t j = r0; j < P; ++j)
                    for (int64_t i = r0; i < r0 + T && i < P; ++i) S[i + P * j] = full[i + P * j];
            stpf2::mirror_lower_tiles(S, P, T);
            if (std::memcmp(S, full.data(), static_cast<size_t>(P * P) * sizeof(double)) != 0) {
                std::printf("mismatch P=%lld offset=%d\n", static_cast<long long>(P), off);
                return 1;
            }
        }
    }
    std::printf("ok\n");
    return 0;
}
