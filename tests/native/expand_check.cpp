// Checker for steppecu_b200/csrc/host_expand.cpp, built and run by tests/test_host_expand.py.
//
// mirror_lower_tiles: for each P (and a 32-byte aligned and a misaligned slab), a symmetric
// P x P column-major slab is kept only in its upper 128 x 128 tiles (what the download
// copies), the rest set to -1; the mirror must restore the full slab bit for bit.
//
// expand_counts: for each P, both count widths and a 32-byte aligned and a misaligned slab (so that both the
// AVX2 path and the element path run where the CPU has AVX2), it draws a symmetric P x P
// integer slab, packs its upper 128 x 128 tiles the way counts_pack.cu does (upper tile u in
// row-major order of ti <= tj, then column c, then row r; zero past the last population),
// calls expand_counts on a slab pre-filled with -1 and compares the result with the full
// slab bit for bit. Prints "ok" and exits 0, or names the first failing case and exits 1.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace stpf2 {
void expand_counts(const void* packed, bool wide, double* S, int64_t P);
void mirror_lower_tiles(double* S, int64_t P, int64_t T);
}

template <class T>
static std::vector<T> pack(const std::vector<double>& full, int64_t P) {
    const int64_t B = 128, nt = (P + B - 1) / B;
    std::vector<T> out(static_cast<size_t>(nt * (nt + 1) / 2 * B * B), 0);
    int64_t u = 0;
    for (int64_t ti = 0; ti < nt; ++ti)
        for (int64_t tj = ti; tj < nt; ++tj, ++u)
            for (int64_t c = 0; c < B; ++c)
                for (int64_t r = 0; r < B; ++r) {
                    const int64_t i = ti * B + r, j = tj * B + c;
                    if (i < P && j < P) out[static_cast<size_t>(u * B * B + c * B + r)] = static_cast<T>(full[i + P * j]);
                }
    return out;
}

int main() {
    const int64_t sizes[] = {1, 3, 4, 8, 100, 127, 128, 129, 132, 300, 1000, 1001};
    uint64_t state = 20261203;
    auto next = [&state](uint64_t range) {
        state = state * 6364136223846793005ull + 1442695040888963407ull;
        return static_cast<double>((state >> 20) % range);
    };
    for (int64_t P : sizes)
        for (int wide = 0; wide < 2; ++wide) {
            std::vector<double> full(static_cast<size_t>(P * P));
            const uint64_t range = wide ? 3000000000ull : 65536ull;  // up to the width's limit
            for (int64_t j = 0; j < P; ++j)
                for (int64_t i = 0; i <= j; ++i) full[i + P * j] = full[j + P * i] = next(wide ? (1ull << 31) - 1 : range);
            const std::vector<uint16_t> p16 = pack<uint16_t>(full, P);
            const std::vector<uint32_t> p32 = pack<uint32_t>(full, P);
            for (int off = 0; off < 2; ++off) {
                std::vector<double> buf(static_cast<size_t>(P * P + 8));
                const uintptr_t base = (reinterpret_cast<uintptr_t>(buf.data()) + 31) & ~uintptr_t(31);
                double* S = reinterpret_cast<double*>(base) + off;
                for (int64_t k = 0; k < P * P; ++k) S[k] = -1.0;
                stpf2::expand_counts(wide ? static_cast<const void*>(p32.data()) : static_cast<const void*>(p16.data()),
                                     wide != 0, S, P);
                if (std::memcmp(S, full.data(), static_cast<size_t>(P * P) * sizeof(double)) != 0) {
                    std::printf("mismatch P=%lld wide=%d offset=%d\n", static_cast<long long>(P), wide, off);
                    return 1;
                }
            }
        }
    for (int64_t P : sizes)
        for (int off = 0; off < 2; ++off) {
            std::vector<double> buf(static_cast<size_t>(P * P + 8));
            const uintptr_t base = (reinterpret_cast<uintptr_t>(buf.data()) + 31) & ~uintptr_t(31);
            double* S = reinterpret_cast<double*>(base) + off;
            std::vector<double> full(static_cast<size_t>(P * P));
            for (int64_t j = 0; j < P; ++j)
                for (int64_t i = 0; i <= j; ++i) full[i + P * j] = full[j + P * i] = next(1ull << 40) * 0x1.0p-40;
            for (int64_t k = 0; k < P * P; ++k) S[k] = -1.0;
            for (int64_t r0 = 0; r0 < P; r0 += 128)
                for (int64_t j = r0; j < P; ++j)
                    for (int64_t i = r0; i < r0 + 128 && i < P; ++i) S[i + P * j] = full[i + P * j];
            stpf2::mirror_lower_tiles(S, P, 128);
            if (std::memcmp(S, full.data(), static_cast<size_t>(P * P) * sizeof(double)) != 0) {
                std::printf("mirror mismatch P=%lld offset=%d\n", static_cast<long long>(P), off);
                return 1;
            }
        }
    std::printf("ok\n");
    return 0;
}
