// steppecu_b200/csrc/counts_pack.cu
//
// Host-output path, vpair side: the both-present counts of a run of P x P slabs are small
// integers (at most the block's SNP count), so only their upper 128 x 128 tiles (row tile
// <= column tile, diagonal tiles whole) cross PCIe, packed as 16-bit counts (32-bit when a
// block has 65,536 SNPs or more); the host widens them to FP64 and writes both halves of
// each exactly symmetric slab (host_expand.cpp: expand_counts). The f2 slabs themselves
// cross whole.
//
// Packed order: slab, upper tile u (ti = 0.., tj = ti..T-1), column c of the tile, row r:
// element (slab * n_ut + u) * 16384 + c * 128 + r, zero past the last population.
#include <algorithm>

#include "stpf2_internal.cuh"

namespace stpf2 {

namespace {

constexpr int kT = 128;

// The upper tile with index u of a T x T tile grid: ti, tj with ti <= tj, rows first.
__device__ __forceinline__ void upper_tile(int u, int T, int& ti, int& tj) {
    int t = 0;
    while (u >= T - t) {
        u -= T - t;
        ++t;
    }
    ti = t;
    tj = t + u;
}

template <class Out>
__global__ void __launch_bounds__(kT) pack_counts_kernel(const double* __restrict__ vp, int64_t P, int T,
                                                          Out* __restrict__ out) {
    const int u = blockIdx.x;
    const int64_t s = blockIdx.y;
    const int n_ut = T * (T + 1) / 2;
    int ti, tj;
    upper_tile(u, T, ti, tj);
    const int r = threadIdx.x;
    const int64_t i = static_cast<int64_t>(ti) * kT + r;
    const double* src = vp + s * P * P + i;
    Out* dst = out + (s * n_ut + u) * static_cast<int64_t>(kT * kT) + r;
    const int64_t j0 = static_cast<int64_t>(tj) * kT;
#pragma unroll 4
    for (int c = 0; c < kT; ++c) {
        const int64_t j = j0 + c;
        const double v = (i < P && j < P) ? __ldg(src + P * j) : 0.0;
        dst[c * kT] = static_cast<Out>(v);
    }
}

}  // namespace

size_t packed_counts_bytes(int P, int64_t nb, bool wide) {
    const int64_t T = (P + kT - 1) / kT;
    return static_cast<size_t>(nb) * static_cast<size_t>(T * (T + 1) / 2) * kT * kT * (wide ? 4u : 2u);
}

void launch_pack_counts(Ctx& c, const double* vp, int P, int64_t nb, bool wide, void* out, cudaStream_t s) {
    if (P <= 0 || nb <= 0) return;
    const int T = (P + kT - 1) / kT;
    const int64_t tile_elems = static_cast<int64_t>(T * (T + 1) / 2) * kT * kT;
    for (int64_t s0 = 0; s0 < nb; s0 += 65535) {  // grid.y limit
        const dim3 grid(static_cast<unsigned>(T * (T + 1) / 2), static_cast<unsigned>(std::min<int64_t>(65535, nb - s0)));
        const double* src = vp + s0 * static_cast<int64_t>(P) * P;
        if (wide) pack_counts_kernel<uint32_t><<<grid, kT, 0, s>>>(src, P, T, static_cast<uint32_t*>(out) + s0 * tile_elems);
        else pack_counts_kernel<uint16_t><<<grid, kT, 0, s>>>(src, P, T, static_cast<uint16_t*>(out) + s0 * tile_elems);
        STPF2_CUDA(cudaGetLastError());
        c.launches++;
    }
}

}  // namespace stpf2
