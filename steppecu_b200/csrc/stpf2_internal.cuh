// steppecu_b200/csrc/stpf2_internal.cuh
//
// Shared internals of libstpf2.so: error plumbing, the context, the block layout that
// maps jackknife blocks onto padded operand columns, and the launch wrappers each .cu
// file exports to the C-ABI layer (stpf2_abi.cu).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <memory>
#include <vector>

#include "../../include/stpf2.h"

namespace stpf2 {

// ---- errors --------------------------------------------------------------------------

// Carries a status code through C++ code paths; the C-ABI layer turns it into the
// return value plus the thread's last-error message.
struct Error : std::runtime_error {
    stp_status status;
    Error(stp_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] inline void fail(stp_status s, const std::string& m) { throw Error(s, m); }

inline void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    // A failed call also leaves its (non-sticky) error as the thread's last error: clear it,
    // so the next launch check of this or a later call reports only its own launch.
    (void)cudaGetLastError();
    const stp_status s = (e == cudaErrorMemoryAllocation) ? STP_DEVICE_OOM : STP_CUDA_ERROR;
    fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define STPF2_CUDA(call) ::stpf2::cuda_check((call), #call)

// ---- device buffers -------------------------------------------------------------------

// Owning device allocation (RAII). Sizes in bytes.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); ptr = o.ptr; bytes = o.bytes; o.ptr = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() { if (ptr) cudaFree(ptr); ptr = nullptr; bytes = 0; }
    // Grows (never shrinks) to at least n bytes; contents are not preserved.
    void reserve(size_t n) {
        if (n <= bytes) return;
        release();
        if (n == 0) return;
        STPF2_CUDA(cudaMalloc(&ptr, n));
        bytes = n;
    }
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Grow-only pinned host memory, for packing many small tables into one upload. Reserving
// more drops the contents; the caller makes sure no copy from it is still in flight.
struct PinnedBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf() { if (ptr) cudaFreeHost(ptr); }
    void reserve(size_t n) {
        if (n <= bytes) return;
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
        STPF2_CUDA(cudaMallocHost(&ptr, n));
        bytes = n;
    }
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Offsets of buffers packed into one allocation (each start 256-byte aligned).
struct Packing {
    size_t end = 0;
    size_t add(size_t bytes) {
        const size_t o = end;
        end = (end + bytes + 255) & ~size_t(255);
        return o;
    }
};

// ---- context --------------------------------------------------------------------------

// Bounded-wait settings of the fixed-point contraction. timeout_ns bounds every device-side
// wait; withhold_stage >= 0 makes the f2 kernel's producer stop before that stage (a test
// hook: the issuer's wait then runs out and the call reports STP_DEVICE_TIMEOUT).
// Row classes of an operand tile side: class k holds 8k+1 .. 8k+8 valid populations (of
// the tile's 128 rows). kDefaultPartialFeed: the classes whose stage copies carry only
// their valid 8-row groups (the measured choice, steppecu_b200/tile_classes.json).
constexpr uint32_t kDefaultPartialFeed = 0xBFFFu;  // measured on B200: all but 113-120 rows

struct FxTuning {
    unsigned long long timeout_ns = 4000000000ull;
    long long withhold_stage = -1;
    uint32_t partial_feed = kDefaultPartialFeed;  // bit k: row class k copies valid rows only
};

struct Ctx {
    int device = 0;
    FxTuning fx_tuning;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    std::atomic<uint64_t> launches{0};
    cudaStream_t h2d = nullptr, d2h = nullptr;  // copy streams of the pipelined host-buffer path
    static constexpr int kSideStreams = 4;
    cudaStream_t side[kSideStreams] = {};  // grouped batches: the requests' image emissions run concurrently
    // Grow-only scratch reused across calls of the host-buffer entry points, so repeated
    // extractions do not pay cudaMalloc each time.
    DevBuf ws_records, ws_f2, ws_vpair, ws_misc, ws_canon, ws_center;
    // Grouped batches: operand images; the shared canonical copy and its tables; the batch
    // populations' counts and every request's tables; the contraction's work lists; and
    // the pinned staging of the tables.
    DevBuf ws_batch, ws_union, ws_tables, ws_items;
    DevBuf ws_fstat;  // stp_fstats scratch
    DevBuf ws_vpc;    // grouped fixed-point batches: compact vpair tiles
    DevBuf ws_fxtab;  // grouped fixed-point batches: the term table of the union's counts
    PinnedBuf pin_union, pin_tables, pin_items;
    PinnedBuf pin_stage;  // streamed extraction: the two-segment staging ring of f2 / vpair slabs
    DevBuf ws_counts;      // host-output path: packed vpair tiles of two segments
    PinnedBuf pin_counts;  // their host staging (every segment, or a two-segment ring with a sink)
    // Completion time of each request of the last stp_f2_extract_batch call, in ms from the
    // start of its group's device work (NaN for requests that ran on their own).
    std::vector<double> last_batch_ms;
    // The plan of the last one-shot extraction with its request, reused by the next call
    // with an identical request (stpf2_abi.cu: PlanCache).
    std::shared_ptr<void> plan_cache;
};

// ---- block layout ---------------------------------------------------------------------

// Column padding of every block in the operand planes: a block's first column is a
// multiple of kColAlign so tensor-core tiles start on aligned addresses, and its tail up
// to the next multiple stays zero (zero operands contribute nothing to any sum).
constexpr int kColAlign = 64;

struct BlockInfo {  // device-visible, one per jackknife block
    int64_t col;      // first padded column
    int32_t k;        // SNPs in the block
    int32_t b;        // block id (slab index of the output)
    int32_t grp = 0;  // request of a batch (index into the GroupInfo table)
    int32_t pad_ = 0;
};

// One request of a grouped contraction: its operand images and its output slabs.
struct GroupInfo {
    const uint8_t* images;  // (row tile t, chunk c) at (t * n_ck + c) * kImageBytes (FX: kFxImageBytes)
    double* f2;             // [P x P x n_block]
    double* vpair;
    int64_t n_ck;
    int32_t P;
    int32_t pad_;
    const uint8_t* mplanes;  // FX: the request's M tiles
};

struct BlockLayout {
    int n_block = 0;
    int64_t n_snp = 0;
    int64_t ld = 0;  // padded column count = row pitch of every operand plane
    std::vector<int64_t> snp_begin;
    std::vector<BlockInfo> blocks;
    std::vector<int32_t> snp_col;  // padded column of every SNP
};

// Validates a contiguous non-decreasing partition (core::block_ranges,
// src/core/domain/block_partition_rule.hpp:56-96) and builds the padded column map.
// with_snp_col = false skips the per-SNP column map (only the Q/V/N feeder reads it).
BlockLayout make_block_layout(const int32_t* block_id, int64_t n_snp, int n_block, bool with_snp_col = true);

// Work item of the contraction: tile pair (ti <= tj) of one block.
struct WorkItem {
    int32_t blk;  // index into BlockInfo array
    int16_t ti, tj;
};

// Tile pairs of every block, costliest (largest k) first.
std::vector<WorkItem> make_work_items(const BlockLayout& L, int P, int tile);

// The fixed-point vpair kernel counts two items in one unit when the second is the next
// column tile of the first's row tile in the same block (one MMA on the stacked B tiles).
__host__ __device__ inline bool vpair_pairs_with(const WorkItem& x, const WorkItem& y) {
    return y.blk == x.blk && y.ti == x.ti && y.tj == x.tj + 1;
}
// Its units over an item list: the index of each unit's first item, greedily left to right
// (item k takes item k + 1 when vpair_pairs_with holds), the rule the kernel re-applies.
std::vector<int32_t> make_vpair_units(const std::vector<WorkItem>& items);

// ---- operand planes --------------------------------------------------------------------

// Operand formats the decode/feeder kernels emit, one per contraction arithmetic.
enum class OpFmt : int { F32 = 0, BF16 = 1, F16 = 2, FX = 3 };

inline OpFmt fmt_of(int precision) {
    switch (precision) {
        case STP_PREC_FP32_SIMT: return OpFmt::F32;
        case STP_PREC_SPLIT_BF16: return OpFmt::BF16;
        case STP_PREC_SPLIT_F16: return OpFmt::F16;
        case STP_PREC_SPLIT_F16_FINE: return OpFmt::F16;
        case STP_PREC_FIXED_I8: return OpFmt::FX;
    }
    fail(STP_INVALID_ARGUMENT, "unknown precision mode " + std::to_string(precision));
}

// Where decode/feeder write. For F32: planes = [Pt f32][Ah f32] (2 planes) + m_u8, plane
// p, row i, column c at planes + (p * P + i) * ld + c. For BF16/F16: 16-bit [Pt_hi][Pt_lo]
// [Ah_hi][Ah_lo][M] and int8 M, tiled into operand images (below).
// Pt = m*(q - c_s), Ah = m*((q - c_s)^2 - h)/2, h = q(1-q)/max(n-1,1), m = [n > 0];
// then num(i,j) = 2 * sum_s (Ah_i M_j + M_i Ah_j - Pt_i Pt_j).
//
// The 16-bit planes and the int8 M plane are TILED for the tensor cores: populations in
// row tiles of 128, columns in chunks of 32, and every (row tile, chunk) stored as ONE
// contiguous 44 KiB operand image holding exactly what the MMAs read from shared memory:
// the five 16-bit tiles [Pt_hi][Pt_lo][Ah_hi][Ah_lo][M] (128 rows x 64 bytes each, 64-byte
// swizzle: 16-byte chunk index XOR (row / 2) % 4), then the int8 M tile (128 rows x 32
// bytes, 32-byte swizzle: chunk XOR (row / 4) % 2). Image (row tile t, chunk c) sits at
// planes + (t * n_ck + c) * kImageBytes, so one side of a pipeline stage is a single bulk
// copy. Rows past P stay zero. The FP32 planes of the SIMT contraction stay row-major.
struct OperandPlanes {
    OpFmt fmt = OpFmt::F32;
    int P = 0;
    int64_t ld = 0;
    void* planes = nullptr;
    uint8_t* m_u8 = nullptr;  // FP32 form only: row-major int8 M
    uint8_t* mplanes = nullptr;  // FX only: the M tiles, (row tile, chunk) 4 KiB each
    // FX only, optional: the digit words (fx_digits of X, of -A) of every count pair a
    // population can reach, entry n * fx_table_ld + a2 (fx_table_kernel), read by the emit
    // instead of computing the terms; null: computed per element.
    const uint2* fx_table = nullptr;
    int32_t fx_table_ld = 0;
    double scale_inv = 1.0;  // numerator scale undo (F16 planes are pre-scaled)
    int n_rt = 0;            // tiled: row tiles of 128 populations
    int64_t n_ck = 0;        // tiled: column chunks of 32
};

constexpr int kTileRows = 128;
constexpr int kTileK = 32;
constexpr int64_t kTile16Bytes = kTileRows * kTileK * 2;  // one 16-bit tile image
constexpr int64_t kTile8Bytes = kTileRows * kTileK;       // one int8 tile image
constexpr int64_t kImageBytes = 5 * kTile16Bytes + kTile8Bytes;  // one operand image (44 KiB)

// Byte offset of element (row r < 128, column k < 32) inside a 16-bit / int8 tile image.
__host__ __device__ inline uint32_t tile16_offset(int r, int k) {
    return static_cast<uint32_t>(r * 64 + ((((k >> 3) ^ (r >> 1)) & 3) << 4) + (k & 7) * 2);
}
__host__ __device__ inline uint32_t tile8_offset(int r, int k) {
    return static_cast<uint32_t>(r * 32 + ((((k >> 4) ^ (r >> 2)) & 1) << 4) + (k & 15));
}

constexpr int kF16PtShift = 7;  // F16: Pt scaled by 2^7, Ah by 2^14 (num by 2^14)

// FX (fixed point, exact integer accumulation): one image per (row tile, chunk) of eight
// int8 tiles [X0][X1][X2][X3][E3][E4][E5][E6] (128 rows x 32 bytes each, the 32-byte
// swizzle of tile8_offset), where X0..X3 are the balanced base-256 digits of X =
// round((q - 1/2) * kFxScale), least significant first, and E3..E6 those of -A with A =
// round((x^2 - h) * kFxAScale); the images of all row tiles first, then one M tile per
// (row tile, chunk), M = kFxM * [n > 0], at mplanes + (t * n_ck + c) * 4 KiB (the f2
// contraction stages it as a ninth plane after the image; the vpair contraction reads the
// M tiles of consecutive chunks in one copy and counts 64 * 64 per both-present SNP).
// kFxScale = 127 * 2^25 keeps |X| <= 127 * 2^24 (|x| <= 1/2) and kFxAScale = kFxScale^2 /
// 2^31 keeps |A| < 2^31 (|a| <= 1/4).
constexpr int kFxPlanes = 9;                                      // staged: the image and M
constexpr int64_t kFxImageBytes = (kFxPlanes - 1) * kTile8Bytes;  // 32 KiB in memory
constexpr double kFxScale = 127.0 * 33554432.0;     // 127 * 2^25
constexpr double kFxAScale = 16129.0 * 524288.0;    // kFxScale^2 / 2^31 = 127^2 * 2^19
constexpr double kFxRoundMagic = 6755399441055744.0;  // 1.5 * 2^52
constexpr int kFxM = 64;
// f2 numerator from W = sum_w V_w 2^(8(w-3)) (the four int32 accumulators): num = -2^25 W /
// kFxScale^2 = -W / (16129 * 2^25).
constexpr double kFxNumScale = -1.0 / (16129.0 * 33554432.0);

size_t operand_plane_bytes(OpFmt f, int P, int64_t ld);
void bind_operand_planes(OperandPlanes& op, OpFmt f, int P, int64_t ld, void* base);

// ---- launch wrappers (defined in the .cu files) ----------------------------------------

// Selected-sample descriptor: byte offset in the record << 5 | code shift << 2 | ploidy
// (0 = contributes nothing).
inline uint32_t pack_sel(int64_t row, int ploidy) {
    const uint32_t byte = static_cast<uint32_t>(row >> 2);
    const uint32_t shift = static_cast<uint32_t>(6 - 2 * (row & 3));
    return (byte << 5) | (shift << 2) | static_cast<uint32_t>(ploidy & 3);
}

// One 32-column tile of the padded column space: the SNP of its first column and how many
// of its columns hold SNPs (the rest are block padding).
struct TileInfo {
    int32_t snp0;
    int32_t nvalid;
};

struct CanonDecodeArgs {
    const uint64_t* canon = nullptr;   // [quads][n_sel][4] 8-byte canonical tile words
    int64_t n_tiles = 0, n_sel = 0;
    const uint32_t* sel = nullptr;     // [n_sel] descriptors (ploidy in the low bits)
    const int32_t* pop_off = nullptr;  // [P+1]
    int P = 0;
    const double* center = nullptr;    // [ld] per-column centre (a multiple of 1/256)
    const double* rec_n = nullptr;     // [n_max+1] 1/n (0 at n = 0)
    const double* rec_nm1 = nullptr;   // [n_max+1] 1/max(n-1, 1)
    const int32_t* col_snp = nullptr;  // [ld] SNP of each column, -1 for padding
    int64_t col_base = 0;              // padded column of tile 0 (a range of the column space)
    OperandPlanes op;                  // planes == nullptr: counts only
    int32_t* cnt_ac2 = nullptr;        // optional [P x n_snp] column-major counts
    int32_t* cnt_n = nullptr;
    // Shared-canonical mode (umap != nullptr), for a batch over one panel: canon holds a
    // set of canonical samples (n_sel = its padded count) in the same tiles as this
    // decode, and selected sample g is canonical sample umap[g]; centres come per SNP from
    // center_snp through col_snp (center unused).
    const int32_t* umap = nullptr;
    const double* center_snp = nullptr;
    // Optional packed counts (ac2 | n << 16), population-major: population i, SNP s at
    // cnt_packed[i * cnt_ld + s].
    uint32_t* cnt_packed = nullptr;
    int64_t cnt_ld = 0;
    // Optional fold order: within each group of 64 populations, the order in which the fold
    // warps take them (local indices, largest population first), so that a warp's eight
    // populations have similar sample counts; null keeps the natural order.
    const int32_t* fold_order = nullptr;
};

// Ploidy detection over 4-byte record words (records and pitch 4-byte aligned); pos maps
// file rows to selected indices (-1: not selected), each row selected once.
void launch_detect_ploidy_words(Ctx& c, const uint8_t* records, uint64_t pitch, int64_t n_snp, int64_t n_ind,
                                const int32_t* pos, uint32_t* sel, cudaStream_t s);
void launch_detect_ploidy_pa(Ctx& c, const uint8_t* records, uint64_t pitch, int64_t n_snp,
                             uint32_t* sel, int64_t n_sel, cudaStream_t s);
// row_map (optional): record row of every SNP index the tiles name (a kept-SNP compaction).
void launch_transpose_pa(Ctx& c, const uint8_t* records, uint64_t pitch, int64_t n_ind, const TileInfo* tiles,
                         int64_t n_tiles, const int32_t* pos, int64_t n_sel, uint64_t* canon, double* center,
                         cudaStream_t s, const int32_t* row_map = nullptr);
// Canonical individual-major tile -> SNP-major records (pitch >= ceil(n_ind / 4)).
void launch_canonical_to_records(Ctx& c, const uint8_t* packed, uint64_t bpr, int64_t n_snp, int64_t n_ind,
                                 uint8_t* records, uint64_t pitch, cudaStream_t s);
// extract-f2's per-SNP keep mask (filters.cu): from packed pop-major counts (ac2 | n << 16,
// population i, SNP s at cnt[i * ld + s]) or from FP64 q / n [P x M] (i + P * s). out4
// (optional, device [4 * M]): pooled ref AF, pooled minor AF, missing fraction, pooled
// allele count per SNP.
void launch_keep_mask_counts(Ctx& c, const uint32_t* cnt, int64_t ld, int P, int64_t M, const char* ref,
                             const char* alt, const int32_t* chrom, const stp_snp_filter& f, double total_indiv,
                             uint8_t* keep, double* out4, cudaStream_t s);
void launch_keep_mask_qn(Ctx& c, const double* Q, const double* N, int P, int64_t M, const char* ref, const char* alt,
                         const int32_t* chrom, const stp_snp_filter& f, double total_indiv, uint8_t* keep,
                         double* out4, cudaStream_t s);
// FP64 [P x M] -> [P x n_kept]: column s goes to column dst_col[s] (-1: dropped).
void launch_compact_columns(Ctx& c, const double* in, int P, int64_t M, const int64_t* dst_col, double* out,
                            cudaStream_t s);
void launch_decode_canon(Ctx& c, const CanonDecodeArgs& a, cudaStream_t s);
void launch_decode_canonical(Ctx& c, const uint8_t* packed, uint64_t bpr, int64_t n_snp,
                             int64_t n_ind, const int32_t* pop_off, int P, const int32_t* ploidy,
                             double* q, double* v, double* n, cudaStream_t s);
void launch_detect_ploidy_canonical(Ctx& c, const uint8_t* packed, uint64_t bpr, int64_t n_snp,
                                    int64_t n_ind, int32_t* ploidy, cudaStream_t s);
void launch_feed_qvn(Ctx& c, const double* Q, const double* V, const double* N, int P,
                     int64_t M, const int32_t* snp_col, const OperandPlanes& op, cudaStream_t s);

void launch_f2_simt(Ctx& c, const WorkItem* items, int n_items, const BlockInfo* blocks,
                    const OperandPlanes& op, double* f2, double* vpair, cudaStream_t s);

// tcgen05 contraction; returns false if the device cannot run it.
struct UmmaPlan;
// One request of a grouped contraction (a batch over one panel): its block layout and its
// images / outputs.
struct GroupSpec {
    const BlockLayout* L = nullptr;
    GroupInfo info{};
};
// Contracts every request of a batch in one persistent launch over all their (block, tile
// pair) items, requests in ascending order of work. stamps (optional) receives each
// request's completion time (%globaltimer, ns). Synchronises s; timeouts raise.
void launch_f2_umma_grouped(Ctx& c, OpFmt fmt, double scale_inv, int chunk_stages, const std::vector<GroupSpec>& groups,
                            cudaStream_t s, std::vector<unsigned long long>* stamps);
// %globaltimer of the device when the stream reaches this point, written to *dst.
void launch_timestamp(Ctx& c, unsigned long long* dst, cudaStream_t s);
// The column -> SNP map (ld entries, -1 for padding) and the 32-column tile table (ld / 32)
// of a block layout, built on the device from its blocks and their first SNPs.
void launch_layout_tables(Ctx& c, const BlockInfo* blocks, const int64_t* snp_begin, int n_block, int64_t ld,
                          int32_t* col_snp, TileInfo* tiles, cudaStream_t s);
// Operand images of one request (P populations, n_tiles padded tiles) from packed
// per-population counts: population i reads counts row upop[i], column c SNP col_snp[c].
// counts: rows of cnt_ld words over n_snp SNPs; rows 16-byte aligned with cnt_ld >= n_snp + 4
// let eight consecutive SNPs load as three 16-byte vectors.
void launch_emit_counts(Ctx& c, const uint32_t* counts, int64_t cnt_ld, int64_t n_snp, const int32_t* upop, int P, int64_t n_tiles,
                        const int32_t* col_snp, const double* center_snp, const double* rec_n, const double* rec_nm1,
                        const OperandPlanes& op, cudaStream_t s);
// Entries of desc marked 3 (ploidy to be detected) take the ploidy bits of union sample
// umap[g] (a batch's shared ploidy pass).
void launch_copy_union_ploidy(Ctx& c, uint32_t* desc, const int32_t* umap, int64_t n_sel, const uint32_t* desc_u,
                              cudaStream_t s);

// The fixed-point contraction (f2_fx.cu): vpair_fx_kernel then f2_fx_kernel over the same
// items. vpc holds fx_vpc_bytes(n_items); counters two ints; groups non-null for a batch.
struct FxLaunch {
    const uint8_t* images = nullptr;
    const uint8_t* mplanes = nullptr;
    int64_t n_ck = 0;
    const WorkItem* items = nullptr;
    int n_items = 0;
    const int32_t* units = nullptr;  // vpair units: first items, as indices past unit_base
    int n_units = 0;
    int unit_base = 0;
    const BlockInfo* blocks = nullptr;
    int P = 0;
    double* f2 = nullptr;
    double* vpair = nullptr;
    int32_t* vpc = nullptr;
    const double* rcp = nullptr;
    int rcp_max = 0;
    int* err = nullptr;
    int* counters = nullptr;
    int b_base = 0;
    const GroupInfo* groups = nullptr;
    int* grp_done = nullptr;
    unsigned long long* grp_ns = nullptr;
    const int* grp_items = nullptr;
};
size_t fx_vpc_bytes(int n_items);
// Shared-memory attributes of the fixed-point kernels (the current device); call before the
// first launch, outside stream capture.
void fx_prepare();
void launch_fx(Ctx& c, const FxLaunch& L, cudaStream_t s);

// chunk_stages: 32-SNP stages per FP32 TMEM chunk (1 or 2).
UmmaPlan* umma_plan_create(Ctx& c, const OperandPlanes& op, const BlockLayout& L, int chunk_stages);
// 32-SNP stages per FP32 chunk for a tensor-core precision mode.
inline int chunk_stages_of(int precision) { return precision == STP_PREC_SPLIT_F16_FINE ? 1 : 2; }
void umma_plan_destroy(UmmaPlan* p);
// per_block: one launch per jackknife block instead of one persistent launch over all
// blocks (the comparison form of the grouped schedule).
void launch_f2_umma(Ctx& c, UmmaPlan* p, double* f2, double* vpair, cudaStream_t s, bool per_block = false);
// The tile pairs of blocks [b0, b1) only, in one launch.
// Blocks [b0, b1) only; rebase: f2 / vpair point at block b0's slab (a buffer of b1 - b0
// slabs) instead of the whole tensor.
void launch_f2_umma_blocks(Ctx& c, UmmaPlan* p, int b0, int b1, double* f2, double* vpair, cudaStream_t s,
                           bool rebase = false);
// After a stream sync: raises STP_DEVICE_TIMEOUT if the kernel's bounded waits expired.
void umma_check(UmmaPlan* p);
int umma_tile();

void launch_survivors(Ctx& c, const double* vpair, int P, int nb, int32_t* keep, cudaStream_t s);
void launch_fstat_assemble(Ctx& c, const double* f2, int P, const int32_t* surv, int ns, int kind,
                           const int32_t* idx, int64_t n_stat, int64_t m, int64_t nr, double* x, cudaStream_t s);
void launch_jackknife(Ctx& c, const double* x, const int32_t* block_sizes, int64_t m, int nb,
                      double* est, double* var, cudaStream_t s);

// Host-output transfer (counts_pack.cu, host_expand.cpp): the upper 128 x 128 tiles of nb
// count slabs packed as 16-bit (wide: 32-bit) integers, and their widening on the host into
// both halves of one P x P FP64 slab.
size_t packed_counts_bytes(int P, int64_t nb, bool wide);
// The fixed-point term table of OperandPlanes::fx_table for called-allele counts 0..n_max
// (decode.cu); fx_table_entries: its size, 0 when it would exceed the cap (then the emit
// computes the terms).
int64_t fx_table_entries(int64_t n_max);
void launch_fx_table(Ctx& c, const double* rec_n, const double* rec_nm1, int64_t n_max, uint2* out, cudaStream_t s);
void launch_pack_counts(Ctx& c, const double* vp, int P, int64_t nb, bool wide, void* out, cudaStream_t s);
void expand_counts(const void* packed, bool wide, double* S, int64_t P);
// Fills the lower tiles of a symmetric P x P column-major slab whose upper T x T tiles are in
// place (host_expand.cpp).
void mirror_lower_tiles(double* S, int64_t P, int64_t T);

// Allocation-free count decode (noalloc.cu): every intermediate lives in one static
// device array of kNoAllocScratchBytes.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
size_t noalloc_scratch_bytes(int64_t n_snp, int64_t n_ind, int64_t n_sel, int P, bool copy_ploidy);
void noalloc_decode_counts(Ctx& c, const uint8_t* d_records, uint64_t pitch, int64_t n_snp, int64_t n_ind,
                           const int64_t* sel_rows, int64_t n_sel, const int64_t* pop_offsets, int P,
                           const int32_t* sample_ploidy, int mode_ploidy, bool detect, int32_t* d_ac2,
                           int32_t* d_n, cudaStream_t s);

}  // namespace stpf2
