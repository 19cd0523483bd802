// steppecu_b200/csrc/noalloc.cu
//
// The allocation-free variant of the count decode behind stp_decode_counts: ploidy
// detection, the canonical transpose and the per-population count fold, with every
// intermediate (the caller's selection copied in, selection descriptors, file-row map,
// tile table, column map, column centres, canonical quads, an error flag) carved out of
// one file-scope static device array instead of cudaMalloc'd buffers. Its address is
// taken once per device with cudaGetSymbolAddress. The reference has no counterpart: its
// backends allocate per call.
//
// What must start at a fixed value is set by the call itself with cudaMemsetAsync: the
// file-row map (-1 = not selected) and the error flag (0). Everything else in the scratch
// is written before it is read within the same call. The scratch is shared by every call
// on a device, so calls whose work overlaps in time (other host threads, other streams)
// race on it and must be serialised by the caller.
#include <algorithm>
#include <exception>
#include <mutex>
#include <string>

#include "stpf2_internal.cuh"

namespace stpf2 {

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

size_t round256(size_t x) { return (x + 255) & ~size_t(255); }

// Selection descriptors (file row, ploidy) and the file-row -> selected-index map. A row
// selected twice raises the error flag (the plan path rejects it on the host).
__global__ void noalloc_select_kernel(const int64_t* __restrict__ sel_rows, int64_t n_sel,
                                      const int32_t* __restrict__ ploidy_in, int mode_ploidy,
                                      uint32_t* __restrict__ desc, int32_t* __restrict__ pos, int* err) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n_sel) return;
    const int64_t row = sel_rows[g];
    int pl = ploidy_in ? ploidy_in[g] : mode_ploidy;
    if (pl != 1 && pl != 2) pl = 0;  // a bad ploidy contributes nothing (decode_af.hpp:58-65)
    desc[g] = (static_cast<uint32_t>(row >> 2) << 5) | (static_cast<uint32_t>(6 - 2 * (row & 3)) << 2) |
              static_cast<uint32_t>(pl);
    if (atomicCAS(pos + row, -1, static_cast<int32_t>(g)) != -1) atomicExch(err, 1);
}

// Contiguous column space (no block padding): tile t holds SNPs 32t .. 32t+31.
__global__ void noalloc_layout_kernel(int64_t n_snp, int64_t n_tiles, TileInfo* __restrict__ tiles,
                                      int32_t* __restrict__ col_snp, const int64_t* __restrict__ po64,
                                      int32_t* __restrict__ po32, int P) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n_tiles * kTileK) col_snp[k] = k < n_snp ? static_cast<int32_t>(k) : -1;
    if (k < n_tiles) {
        const int64_t rem = n_snp - k * kTileK;
        tiles[k] = TileInfo{static_cast<int32_t>(k * kTileK), static_cast<int32_t>(rem < kTileK ? rem : kTileK)};
    }
    if (k <= P) po32[k] = static_cast<int32_t>(po64[k]);
}

// An error thrown after work was queued must not return while that work still writes the
// caller's outputs and the shared scratch: wait for the stream first.
struct SyncOnError {
    cudaStream_t s;
    ~SyncOnError() {
        if (std::uncaught_exceptions() > 0) cudaStreamSynchronize(s);
    }
};

void* scratch_base(int device) {
    if (device < 0 || device >= kMaxDevices) fail(STP_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        STPF2_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_ptr[device] = p;
    }
    return g_scratch_ptr[device];
}

}  // namespace

size_t noalloc_scratch_bytes(int64_t n_snp, int64_t n_ind, int64_t n_sel, int P, bool copy_ploidy) {
    const int64_t n_tiles = (n_snp + kTileK - 1) / kTileK;
    const int64_t n_quads = (n_tiles + 3) / 4;
    const int64_t n_sel_pad = (n_sel + 3) / 4 * 4;
    const int64_t n_ind16 = (n_ind + 15) / 16 * 16;
    size_t b = 0;
    b += round256(static_cast<size_t>(n_sel) * 8);                      // sel_rows
    b += round256(static_cast<size_t>(P + 1) * 8);                      // pop_offsets (int64)
    b += copy_ploidy ? round256(static_cast<size_t>(n_sel) * 4) : 0;   // sample ploidy
    b += round256(static_cast<size_t>(n_sel_pad) * 4);                  // descriptors
    b += round256(static_cast<size_t>(n_ind16) * 4);                    // file-row map
    b += round256(static_cast<size_t>(P + 1) * 4);                      // pop_offsets (int32)
    b += round256(static_cast<size_t>(n_tiles) * sizeof(TileInfo));    // tiles
    b += round256(static_cast<size_t>(n_tiles) * kTileK * 4);           // column -> SNP
    b += round256(static_cast<size_t>(n_tiles) * kTileK * 8);           // column centres
    b += round256(static_cast<size_t>(n_quads) * n_sel_pad * 32);       // canonical quads
    b += 256;                                                            // error flag
    return b;
}

void noalloc_decode_counts(Ctx& c, const uint8_t* d_records, uint64_t pitch, int64_t n_snp, int64_t n_ind,
                           const int64_t* sel_rows, int64_t n_sel, const int64_t* pop_offsets, int P,
                           const int32_t* sample_ploidy, int mode_ploidy, bool detect, int32_t* d_ac2,
                           int32_t* d_n, cudaStream_t s) {
    const size_t need = noalloc_scratch_bytes(n_snp, n_ind, n_sel, P, sample_ploidy != nullptr);
    if (need > kNoAllocScratchBytes)
        fail(STP_INVALID_ARGUMENT, "no-alloc decode: this request needs " + std::to_string(need) +
                                       " bytes of scratch; the static scratch holds " +
                                       std::to_string(kNoAllocScratchBytes) +
                                       " (about n_sel * n_snp / 4 bytes of canonical genotypes + 12 bytes per SNP)");
    uint8_t* base = static_cast<uint8_t*>(scratch_base(c.device));
    const int64_t n_tiles = (n_snp + kTileK - 1) / kTileK;
    const int64_t n_quads = (n_tiles + 3) / 4;
    const int64_t n_sel_pad = (n_sel + 3) / 4 * 4;
    const int64_t n_ind16 = (n_ind + 15) / 16 * 16;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        uint8_t* p = base + off;
        off += round256(bytes);
        return p;
    };
    auto* d_sel_rows = reinterpret_cast<int64_t*>(take(static_cast<size_t>(n_sel) * 8));
    auto* d_po64 = reinterpret_cast<int64_t*>(take(static_cast<size_t>(P + 1) * 8));
    int32_t* d_pl = sample_ploidy ? reinterpret_cast<int32_t*>(take(static_cast<size_t>(n_sel) * 4)) : nullptr;
    auto* d_desc = reinterpret_cast<uint32_t*>(take(static_cast<size_t>(n_sel_pad) * 4));
    auto* d_pos = reinterpret_cast<int32_t*>(take(static_cast<size_t>(n_ind16) * 4));
    auto* d_po32 = reinterpret_cast<int32_t*>(take(static_cast<size_t>(P + 1) * 4));
    auto* d_tiles = reinterpret_cast<TileInfo*>(take(static_cast<size_t>(n_tiles) * sizeof(TileInfo)));
    auto* d_col_snp = reinterpret_cast<int32_t*>(take(static_cast<size_t>(n_tiles) * kTileK * 4));
    auto* d_center = reinterpret_cast<double*>(take(static_cast<size_t>(n_tiles) * kTileK * 8));
    auto* d_canon = reinterpret_cast<uint64_t*>(take(static_cast<size_t>(n_quads) * n_sel_pad * 32));
    auto* d_err = reinterpret_cast<int*>(take(256));

    SyncOnError sync_on_error{s};
    STPF2_CUDA(cudaMemcpyAsync(d_sel_rows, sel_rows, static_cast<size_t>(n_sel) * 8, cudaMemcpyHostToDevice, s));
    STPF2_CUDA(cudaMemcpyAsync(d_po64, pop_offsets, static_cast<size_t>(P + 1) * 8, cudaMemcpyHostToDevice, s));
    if (d_pl)
        STPF2_CUDA(cudaMemcpyAsync(d_pl, sample_ploidy, static_cast<size_t>(n_sel) * 4, cudaMemcpyHostToDevice, s));
    STPF2_CUDA(cudaMemsetAsync(d_pos, 0xFF, static_cast<size_t>(n_ind16) * 4, s));  // -1: not selected
    STPF2_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s));
    if (n_sel > 0) {
        noalloc_select_kernel<<<static_cast<unsigned>((n_sel + 255) / 256), 256, 0, s>>>(
            d_sel_rows, n_sel, d_pl, mode_ploidy, d_desc, d_pos, d_err);
        STPF2_CUDA(cudaGetLastError());
        c.launches++;
    }
    const int64_t layout_n = std::max<int64_t>(n_tiles * kTileK, P + 1);
    noalloc_layout_kernel<<<static_cast<unsigned>((layout_n + 255) / 256), 256, 0, s>>>(
        n_snp, n_tiles, d_tiles, d_col_snp, d_po64, d_po32, P);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
    if (detect) launch_detect_ploidy_words(c, d_records, pitch, n_snp, n_ind, d_pos, d_desc, s);
    launch_transpose_pa(c, d_records, pitch, n_ind, d_tiles, n_tiles, d_pos, n_sel_pad, d_canon, d_center, s);
    CanonDecodeArgs a;
    a.canon = d_canon;
    a.n_tiles = n_tiles;
    a.n_sel = n_sel_pad;
    a.sel = d_desc;
    a.pop_off = d_po32;
    a.P = P;
    a.center = d_center;
    a.col_snp = d_col_snp;
    a.op.planes = nullptr;  // counts only
    a.cnt_ac2 = d_ac2;
    a.cnt_n = d_n;
    launch_decode_canon(c, a, s);
    int h_err = 0;
    STPF2_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    STPF2_CUDA(cudaStreamSynchronize(s));
    if (h_err) fail(STP_INVALID_ARGUMENT, "a sample is selected more than once");
}

}  // namespace stpf2
