// steppecu_b200/csrc/f2_umma.cu
//
// The tensor-core f2 contraction for sm_100a: one persistent, warp-specialised kernel
// over every (jackknife block, 128x128 population tile pair ti <= tj) work item.
//
//   warp 0      producer: per 32-SNP stage, bulk-copies the pre-swizzled operand image of
//               the row tile and of the column tile (one side on diagonal tiles): 44 KiB
//               each, the 5 split planes (Pt_hi, Pt_lo, Ah_hi, Ah_lo, M as 16-bit) and the
//               int8 M plane in one contiguous copy; no tensor maps, no multicast.
//   warp 1      TMEM owner + single-thread tcgen05.mma issuer. Per 16-SNP K step, seven
//               kind::f16 MMAs accumulate num/2 = sum(Ah_i M_j + M_i Ah_j - Pt_i Pt_j) over
//               the hi/lo splits (the -Pt Pt products use the descriptor's A-negate bit)
//               into one FP32 TMEM buffer per chunk (64 SNPs = two stages; 32 SNPs in the
//               fine mode); one kind::i8 MMA per stage
//               accumulates the exact both-present count M M^T into an int32 TMEM buffer.
//   warps 2-17  epilogue, four warps per TMEM lane quarter, 32 tile columns each: drains
//               the FP32 chunks two at a time into FP64 registers (one round-to-nearest FP32
//               add of the two chunk sums, then one FP32 -> FP64 conversion and FP64 add);
//               at the end of the block, reads vpair, forms f2 = num / vpair in FP64 (0 when
//               vpair = 0, f2_estimator.hpp:42-46) and stores (i,j) and (j,i) of the block's
//               slab.
//
// TMEM (512 columns): a ring of three FP32 numerator chunk buffers at [0,128), [128,256),
// [256,384) (the MMAs fill the third while a pair drains) and the int32 vpair of the
// current tile at [384,512) (the issuer waits for the previous tile's vpair to be read
// before the tile's first i8 MMA). Every wait is bounded (a few seconds); on expiry the
// kernel raises an error flag the host turns into STP_DEVICE_TIMEOUT, lets its copies and
// MMAs finish, frees TMEM and returns.
#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>
#include <vector>

#include "stpf2_internal.cuh"
#include "umma_ptx.cuh"

namespace stpf2 {

namespace {

constexpr int kTile = 128;
constexpr int kStageK = 32;        // SNP columns per pipeline stage
constexpr int kStages = 2;
constexpr int kNumBufs = 3;        // FP32 chunk buffers in TMEM
constexpr uint32_t kVpCol = kNumBufs * 128u;
constexpr int kPlanes = 5;
constexpr uint32_t kTile16 = kTile * kStageK * 2;                 // 8 KiB
constexpr uint32_t kTile8 = kTile * kStageK;                      // 4 KiB
constexpr uint32_t kSideBytes = kPlanes * kTile16 + kTile8;       // 44 KiB
constexpr uint32_t kStageBytes = 2 * kSideBytes;                  // 88 KiB
static_assert(kSideBytes == kImageBytes, "a stage side is one operand image");
constexpr int kEpiWarps = 16;
constexpr int kEpiWarp0 = 2;                        // epilogue = warps 2..17
constexpr int kThreads = 32 * (kEpiWarp0 + kEpiWarps);  // 576
constexpr int kCols = 4 * kTile / kEpiWarps;        // tile columns per epilogue thread (32)
// 18 warps put five warps on two SM sub-partitions, so at most 16384 / (5 * 32) = 102
// registers per thread (96 in allocation steps); 32 FP64 accumulators per thread fit.
// Four epilogue warps per TMEM lane quarter keep enough tensor-memory loads in flight.
constexpr uint32_t kTmemCols = 512;
// Per-epilogue-warp staging tile for the transposed stores (f2, then vpair): 32 rows x 8
// columns, rows padded to 9 doubles (fewer bank conflicts).
constexpr int kStagePitch = 9;
constexpr int kStageDoubles = 32 * kStagePitch;
constexpr uint32_t kCtlBytes = 256;

struct UmmaArgs {
    const uint8_t* images;    // operand images, (row tile, chunk) at (t * n_ck + c) * kSideBytes
    int64_t n_ck;             // column chunks per row tile
    const WorkItem* items;
    int n_items;
    const BlockInfo* blocks;
    int P;
    double* f2;
    double* vpair;
    double num_scale;  // 2 * plane scale undo
    const double* rcp; // rcp[k] = 1/k for k = 0..rcp_max (rcp[0] = 0): vpair never exceeds the block size
    int rcp_max;
    int* err;
    int* next_item;    // work-item counter, zero at launch
    int b_base;        // block id whose slab starts the output buffers (0: the whole tensor)
    uint32_t idesc_pp, idesc_am, idesc_i8;
    // Grouped launch (a batch of requests): per-request images and outputs, indexed by
    // BlockInfo::grp; null for one request (images, n_ck, P, f2, vpair above). Optional
    // completion stamps: grp_done counts finished (item, epilogue warp) pairs per request,
    // and the last one writes %globaltimer to grp_ns.
    const GroupInfo* groups;
    int* grp_done;
    unsigned long long* grp_ns;
    const int* grp_items;
};

constexpr int kItemRing = 4;  // work items handed from the producer to the other roles

struct SmemCtl {
    unsigned long long item_full[kItemRing], item_empty[kItemRing];
    int item_idx[kItemRing];
    unsigned long long full[kStages], empty[kStages];
    unsigned long long acc_full[kNumBufs], acc_empty[kNumBufs];
    unsigned long long vp_full, vp_empty;
    unsigned long long drain;
    uint32_t tmem_base;
    volatile int abort;
};

// ---- PTX wrappers (umma_ptx.cuh) ---------------------------------------------------------

using namespace ptx;

// Bounded wait honouring this CTA's abort flag.
__device__ __forceinline__ bool wait_bounded(unsigned long long* b, uint32_t parity, SmemCtl* ctl, int* err,
                                          bool honour_abort = true) {
    return ptx::wait_bounded(b, parity, &ctl->abort, err, kTimeoutNs, honour_abort);
}

// ---- roles -------------------------------------------------------------------------------

__device__ __forceinline__ int stages_of(int k) { return (k + kStageK - 1) / kStageK; }
inline int stages_of_host(int k) { return (k + kStageK - 1) / kStageK; }

// Work items are handed out dynamically, in list order (costliest block first, a block's
// tile pairs together): the producer takes the next item from a global counter and
// publishes its index to the issuer and the epilogue warps through a small ring, so the
// CTAs stay within a window of consecutive items and a block's operand images are reused
// from L2 by all of its tile pairs. Index -1 ends the work.
__device__ __forceinline__ int take_item(const UmmaArgs& a, SmemCtl* ctl, uint32_t gi, bool& ok) {
    const int slot = static_cast<int>(gi % kItemRing);
    ok = wait_bounded(&ctl->item_empty[slot], ((gi / kItemRing) & 1u) ^ 1u, ctl, a.err);
    if (!ok) return -1;
    int it = atomicAdd(a.next_item, 1);
    if (it >= a.n_items) it = -1;
    *reinterpret_cast<volatile int*>(&ctl->item_idx[slot]) = it;
    mbar_arrive(&ctl->item_full[slot]);
    return it;
}

// Consumer side (one thread): the gi-th item index, or -1 when the work ends or on abort.
__device__ __forceinline__ int read_item(const UmmaArgs& a, SmemCtl* ctl, uint32_t gi) {
    const int slot = static_cast<int>(gi % kItemRing);
    if (!wait_bounded(&ctl->item_full[slot], (gi / kItemRing) & 1u, ctl, a.err)) return -2;
    const int it = *reinterpret_cast<volatile int*>(&ctl->item_idx[slot]);
    mbar_arrive(&ctl->item_empty[slot]);
    return it;
}

template <bool kGrouped>
__device__ void producer(const UmmaArgs& a, uint8_t* smem, SmemCtl* ctl) {
    uint32_t g = 0;
    for (uint32_t gi = 0;; ++gi) {
        bool ok = true;
        const int it = take_item(a, ctl, gi, ok);
        if (!ok) goto abort;
        if (it < 0) break;
        const WorkItem w = a.items[it];
        const BlockInfo bi = a.blocks[w.blk];
        const int nst = stages_of(bi.k);
        const bool diag = w.ti == w.tj;
        const uint8_t* images = a.images;
        int64_t n_ck = a.n_ck;
        if constexpr (kGrouped) {
            images = a.groups[bi.grp].images;
            n_ck = a.groups[bi.grp].n_ck;
        }
        for (int st = 0; st < nst; ++st, ++g) {
            const int slot = static_cast<int>(g % kStages);
            const uint32_t ph = (g / kStages) & 1u;
            if (!wait_bounded(&ctl->empty[slot], ph ^ 1u, ctl, a.err)) goto abort;
            {
                uint8_t* sb = smem + slot * kStageBytes;
                mbar_expect_tx(&ctl->full[slot], diag ? kSideBytes : kStageBytes);
                const int64_t chunk = bi.col / kStageK + st;
                const int64_t ta = static_cast<int64_t>(w.ti) * n_ck + chunk;
                bulk_load(sb, images + ta * kSideBytes, kSideBytes, &ctl->full[slot]);
                if (!diag) {
                    const int64_t tb = static_cast<int64_t>(w.tj) * n_ck + chunk;
                    bulk_load(sb + kSideBytes, images + tb * kSideBytes, kSideBytes, &ctl->full[slot]);
                }
            }
        }
    }
    return;
abort:
    // Let the copies already issued land before the CTA's shared memory goes away.
    for (uint32_t k = (g >= kStages ? g - kStages : 0); k < g; ++k)
        wait_bounded(&ctl->full[k % kStages], (k / kStages) & 1u, ctl, a.err, false);
}

template <int kChunkStages>
__device__ void mma_issuer(const UmmaArgs& a, uint8_t* smem, SmemCtl* ctl, uint32_t tmem) {
    uint32_t g = 0, cs = 0, is = 0;
    for (uint32_t gi = 0;; ++gi) {
        const int it = read_item(a, ctl, gi);
        if (it < 0) break;
        const WorkItem w = a.items[it];
        const BlockInfo bi = a.blocks[w.blk];
        const int nst = stages_of(bi.k);
        if (nst == 0) continue;
        const bool diag = w.ti == w.tj;
        {
            const uint32_t d_vp = tmem + kVpCol;
            for (int st = 0; st < nst; ++st, ++g) {
                const int sc = st % kChunkStages;  // stage within the chunk
                const int nb = static_cast<int>(cs % kNumBufs);
                if (sc == 0) {
                    if (!wait_bounded(&ctl->acc_empty[nb], ((cs / kNumBufs) & 1u) ^ 1u, ctl, a.err)) goto done;
                    tc_fence_after();
                }
                const uint32_t d_num = tmem + static_cast<uint32_t>(nb) * 128u;
                const int slot = static_cast<int>(g % kStages);
                if (!wait_bounded(&ctl->full[slot], (g / kStages) & 1u, ctl, a.err)) goto done;
                tc_fence_after();
                const uint32_t sa = smem_u32(smem + slot * kStageBytes);
                const uint32_t sb = diag ? sa : sa + kSideBytes;
#pragma unroll
                for (int k = 0; k < kStageK / 16; ++k) {
                    const uint32_t ko = static_cast<uint32_t>(k) * 32u;  // 16 elements x 2 bytes
                    const uint64_t aPh = smem_desc(sa + 0 * kTile16 + ko, 512, 4);
                    const uint64_t aPl = smem_desc(sa + 1 * kTile16 + ko, 512, 4);
                    const uint64_t aAh = smem_desc(sa + 2 * kTile16 + ko, 512, 4);
                    const uint64_t aAl = smem_desc(sa + 3 * kTile16 + ko, 512, 4);
                    const uint64_t aM = smem_desc(sa + 4 * kTile16 + ko, 512, 4);
                    const uint64_t bPh = smem_desc(sb + 0 * kTile16 + ko, 512, 4);
                    const uint64_t bPl = smem_desc(sb + 1 * kTile16 + ko, 512, 4);
                    const uint64_t bAh = smem_desc(sb + 2 * kTile16 + ko, 512, 4);
                    const uint64_t bAl = smem_desc(sb + 3 * kTile16 + ko, 512, 4);
                    const uint64_t bM = smem_desc(sb + 4 * kTile16 + ko, 512, 4);
                    const uint32_t first = (sc == 0 && k == 0) ? 0u : 1u;
                    // Large terms first and interleaved in sign, the lo corrections last.
                    mma_f16(d_num, aAh, bM, a.idesc_am, first);
                    mma_f16(d_num, aPh, bPh, a.idesc_pp, 1u);
                    mma_f16(d_num, aM, bAh, a.idesc_am, 1u);
                    mma_f16(d_num, aPh, bPl, a.idesc_pp, 1u);
                    mma_f16(d_num, aPl, bPh, a.idesc_pp, 1u);
                    mma_f16(d_num, aAl, bM, a.idesc_am, 1u);
                    mma_f16(d_num, aM, bAl, a.idesc_am, 1u);
                }
                if (st == 0) {  // the previous tile's vpair has been read
                    if (!wait_bounded(&ctl->vp_empty, (is & 1u) ^ 1u, ctl, a.err)) goto done;
                    tc_fence_after();
                }
                mma_i8(d_vp, smem_desc(sa + kPlanes * kTile16, 256, 6), smem_desc(sb + kPlanes * kTile16, 256, 6),
                       a.idesc_i8, st > 0 ? 1u : 0u);
                mma_commit(&ctl->empty[slot]);
                if (sc == kChunkStages - 1 || st == nst - 1) {
                    mma_commit(&ctl->acc_full[nb]);
                    ++cs;
                }
            }
            mma_commit(&ctl->vp_full);
            ++is;
        }
    }
done:
    // Every MMA this thread issued completes before TMEM is released.
    mma_commit(&ctl->drain);
    wait_bounded(&ctl->drain, 0u, ctl, a.err, false);
}

// The output side of a work item for this epilogue thread (row r of the tile, column
// part h): its request's P and slabs, the slab offset, the thread's row i and first column
// j0, and the first row i0 of its warp.
struct ItemOut {
    double* f2;
    double* vp;
    int64_t slab;
    int P, i, j0, i0, grp;
    bool diag;
};

template <bool kGrouped>
__device__ __forceinline__ ItemOut item_out(const UmmaArgs& a, int it, int r, int h) {
    const WorkItem w = a.items[it];
    const BlockInfo bi = a.blocks[w.blk];
    ItemOut o;
    o.grp = bi.grp;
    o.P = a.P;
    o.f2 = a.f2;
    o.vp = a.vpair;
    if constexpr (kGrouped) {
        const GroupInfo& gr = a.groups[bi.grp];
        o.P = gr.P;
        o.f2 = gr.f2;
        o.vp = gr.vpair;
    }
    o.diag = w.ti == w.tj;
    o.i = w.ti * kTile + r;
    o.i0 = w.ti * kTile + (r & ~31);
    o.j0 = w.tj * kTile + h * kCols;
    o.slab = static_cast<int64_t>(o.P) * o.P * (bi.b - a.b_base);
    return o;
}

// Completion stamp of a grouped launch: the last (item, epilogue warp) of a request records
// the time.
template <bool kGrouped>
__device__ __forceinline__ void stamp(const UmmaArgs& a, int grp, int lane) {
    if (!kGrouped || !a.grp_done) return;
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        const int d = atomicAdd(a.grp_done + grp, 1);
        if (d == a.grp_items[grp] * kEpiWarps - 1) a.grp_ns[grp] = globaltimer();
    }
}

template <int kChunkStages, bool kGrouped>
__device__ void epilogue(const UmmaArgs& a, SmemCtl* ctl, uint32_t tmem, int warp, int lane, double* stage) {
    const int e = warp - kEpiWarp0;
    const int q = warp & 3;                 // TMEM lane quarter this warp may access
    const int h = e >> 2;                   // column part of the tile (kCols columns)
    const int r = q * 32 + lane;            // tile row (TMEM lane)
    const uint32_t lane_addr = static_cast<uint32_t>(q * 32) << 16;
    const uint32_t col_addr = static_cast<uint32_t>(h * kCols);
    uint32_t cs = 0, is = 0;
    double acc[kCols];  // FP64 running numerator per column
    for (uint32_t gi = 0;; ++gi) {
        int it = 0;
        if (lane == 0) it = read_item(a, ctl, gi);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it < 0) return;
        // Only the stage count lives through the drain; the output side of the item is
        // read again at its end (fewer registers held across the chunk loop).
        const int nst = stages_of(a.blocks[a.items[it].blk].k);
        if (nst == 0) {  // an empty block id: zeros (cpu_backend.cpp:234)
            const ItemOut o = item_out<kGrouped>(a, it, r, h);
            if (o.i < o.P)
                for (int c = 0; c < kCols; ++c) {
                    const int j = o.j0 + c;
                    if (j >= o.P || (o.diag && j < o.i)) continue;
                    o.f2[o.slab + o.i + static_cast<int64_t>(o.P) * j] = 0.0;
                    o.vp[o.slab + o.i + static_cast<int64_t>(o.P) * j] = 0.0;
                    o.f2[o.slab + j + static_cast<int64_t>(o.P) * o.i] = 0.0;
                    o.vp[o.slab + j + static_cast<int64_t>(o.P) * o.i] = 0.0;
                }
            stamp<kGrouped>(a, o.grp, lane);
            continue;
        }
#pragma unroll
        for (int c = 0; c < kCols; ++c) acc[c] = 0.0;
        const int nch = (nst + kChunkStages - 1) / kChunkStages;
        for (int ch = 0; ch < nch; ch += 2) {
            const bool pair = ch + 1 < nch;
            const int nb0 = static_cast<int>(cs % kNumBufs), nb1 = static_cast<int>((cs + 1) % kNumBufs);
            bool ok = true;
            if (lane == 0) {
                ok = wait_bounded(&ctl->acc_full[nb0], (cs / kNumBufs) & 1u, ctl, a.err);
                if (ok && pair) ok = wait_bounded(&ctl->acc_full[nb1], ((cs + 1) / kNumBufs) & 1u, ctl, a.err);
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) return;
            tc_fence_after();
            const uint32_t b0 = tmem + lane_addr + static_cast<uint32_t>(nb0) * 128u + col_addr;
            // A lone last chunk reads its buffer twice and adds zero (exact).
            const uint32_t b1 = pair ? tmem + lane_addr + static_cast<uint32_t>(nb1) * 128u + col_addr : b0;
            const float w1 = pair ? 1.0f : 0.0f;
#pragma unroll
            for (int q8 = 0; q8 < kCols / 8; ++q8) {
                uint32_t v0[8], v1[8];
                tmem_ld8(b0 + static_cast<uint32_t>(q8) * 8u, v0);
                tmem_ld8(b1 + static_cast<uint32_t>(q8) * 8u, v1);
                tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    acc[q8 * 8 + c] += static_cast<double>(__fmaf_rn(w1, __uint_as_float(v1[c]), __uint_as_float(v0[c])));
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&ctl->acc_empty[nb0]);
                if (pair) mbar_arrive(&ctl->acc_empty[nb1]);
            }
            cs += pair ? 2u : 1u;
        }
        {
            bool ok = true;
            if (lane == 0) ok = wait_bounded(&ctl->vp_full, is & 1u, ctl, a.err);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) return;
        }
        tc_fence_after();
        const uint32_t vbase = tmem + lane_addr + kVpCol + col_addr;
        // Output: (i, j) straight from registers (32 consecutive i per store: full sectors);
        // (j, i) through this warp's staging tile, so each store covers 4 rows x 8
        // consecutive j (64-byte segments) instead of 32 scattered 8-byte pieces.
        const ItemOut o = item_out<kGrouped>(a, it, r, h);
        const int P = o.P, i = o.i, i0 = o.i0, j0 = o.j0;
        const bool diag = o.diag;
        const int64_t row_i = o.slab + i;                              // (i, j) at row_i + P*j
        const int64_t row_j0 = o.slab + static_cast<int64_t>(P) * i0;  // (j, i0 + rr) at row_j0 + P*rr + j
#pragma unroll
        for (int q8 = 0; q8 < kCols / 8; ++q8) {
            uint32_t v[8];
            tmem_ld8(vbase + static_cast<uint32_t>(q8) * 8u, v);
            tmem_wait_ld();
            if (q8 == kCols / 8 - 1) {
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&ctl->vp_empty);
            }
            double fv[8], vv[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int col = q8 * 8 + c;
                const int j = j0 + col;
                // vpair is an exact count <= the block size: convert it with the 2^52 trick
                // (an FP64 add) and divide through the 1/k table (within 2 ulp of num / vp).
                const int32_t vpi = static_cast<int32_t>(v[c]);
                const int32_t vk = vpi < a.rcp_max ? vpi : a.rcp_max;
                vv[c] = __hiloint2double(0x43300000, vpi) - 4503599627370496.0;
                fv[c] = vk > 0 ? acc[col] * a.num_scale * __ldg(a.rcp + vk) : 0.0;
                if (i < P && j < P && !(diag && j < i)) {
                    const int64_t ij = row_i + static_cast<int64_t>(P) * j;
                    __stcs(o.f2 + ij, fv[c]);  // output is never re-read: evict-first
                    __stcs(o.vp + ij, vv[c]);
                }
            }
            const int jj = j0 + q8 * 8 + (lane & 7);
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                double* out = part == 0 ? o.f2 : o.vp;
#pragma unroll
                for (int c = 0; c < 8; ++c) stage[lane * kStagePitch + c] = part == 0 ? fv[c] : vv[c];
                __syncwarp();
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int rr = 4 * k + (lane >> 3);
                    if (i0 + rr < P && jj < P && !(diag && jj <= i0 + rr))
                        __stcs(out + row_j0 + static_cast<int64_t>(P) * rr + jj, stage[rr * kStagePitch + (lane & 7)]);
                }
                __syncwarp();
            }
        }
        stamp<kGrouped>(a, o.grp, lane);
        ++is;
    }
}

// kChunkStages: pipeline stages of 32 SNPs accumulated into one FP32 TMEM chunk before the
// epilogue moves it to FP64 (1: 32-SNP chunks, 2: 64-SNP chunks; longer chunks halve the
// epilogue's conversions and lengthen the FP32 sums).
template <int kChunkStages, bool kGrouped>
__global__ void __maxnreg__(96)
f2_umma_kernel(const __grid_constant__ UmmaArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    SmemCtl* ctl = reinterpret_cast<SmemCtl*>(smem + kStages * kStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kItemRing; ++s) {
            mbar_init(&ctl->item_full[s], 1);
            mbar_init(&ctl->item_empty[s], 1 + kEpiWarps);  // the issuer and every epilogue warp
        }
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        for (int b = 0; b < kNumBufs; ++b) {
            mbar_init(&ctl->acc_full[b], 1);
            mbar_init(&ctl->acc_empty[b], kEpiWarps);
        }
        mbar_init(&ctl->vp_full, 1);
        mbar_init(&ctl->vp_empty, kEpiWarps);
        mbar_init(&ctl->drain, 1);
        ctl->abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&ctl->tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;

    if (warp < kEpiWarp0) {
        if (warp == 0 && lane == 0) producer<kGrouped>(a, smem, ctl);
        if (warp == 1 && lane == 0) mma_issuer<kChunkStages>(a, smem, ctl, tmem);
    } else {
        epilogue<kChunkStages, kGrouped>(a, ctl, tmem, warp, lane,
                 reinterpret_cast<double*>(smem + kStages * kStageBytes + kCtlBytes) + (warp - kEpiWarp0) * kStageDoubles);
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// Instruction descriptors (kind::f16 / kind::i8): D format, A/B formats, A negate,
// K-major A and B, N >> 3 at bit 17, M >> 4 at bit 24.
uint32_t idesc_f16(bool bf16, bool negate_a) {
    const uint32_t fmt = bf16 ? 1u : 0u;
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((negate_a ? 1u : 0u) << 13) | ((kTile >> 3) << 17) |
           ((kTile >> 4) << 24);
}
uint32_t idesc_u8_s32() { return (2u << 4) | (0u << 7) | (0u << 10) | ((kTile >> 3) << 17) | ((kTile >> 4) << 24); }

constexpr size_t kSmemBytes = kStages * kStageBytes + kCtlBytes + kEpiWarps * kStageDoubles * sizeof(double) + 1024;
static_assert(sizeof(SmemCtl) <= kCtlBytes, "barrier block overflows its slot");

void set_umma_smem() {
    const int b = static_cast<int>(kSmemBytes);
    STPF2_CUDA(cudaFuncSetAttribute(f2_umma_kernel<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    STPF2_CUDA(cudaFuncSetAttribute(f2_umma_kernel<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    STPF2_CUDA(cudaFuncSetAttribute(f2_umma_kernel<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    STPF2_CUDA(cudaFuncSetAttribute(f2_umma_kernel<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
}

void launch_kernel(int chunk_stages, bool grouped, int grid, const UmmaArgs& a, cudaStream_t s) {
    if (chunk_stages == 1) {
        if (grouped) f2_umma_kernel<1, true><<<grid, kThreads, kSmemBytes, s>>>(a);
        else f2_umma_kernel<1, false><<<grid, kThreads, kSmemBytes, s>>>(a);
    } else {
        if (grouped) f2_umma_kernel<2, true><<<grid, kThreads, kSmemBytes, s>>>(a);
        else f2_umma_kernel<2, false><<<grid, kThreads, kSmemBytes, s>>>(a);
    }
}

}  // namespace

struct UmmaPlan {
    const uint8_t* images = nullptr;
    const uint8_t* mplanes = nullptr;  // FX: the M tiles
    int64_t n_ck = 0;
    DevBuf items, blocks, err, rcp, block_items, counter;
    DevBuf vpc;  // FX: compact vpair tiles, one per item of the largest launch
    DevBuf units, block_units;  // FX: vpair units of items and of block_items
    std::vector<int> block_item_off;  // per block: its tile pairs in block_items
    std::vector<int> block_unit_off;  // per block: its vpair units in block_units
    int n_items = 0;
    int n_units = 0;
    int rcp_max = 0;
    int P = 0;
    OpFmt fmt = OpFmt::BF16;
    double num_scale = 2.0;
    int chunk_stages = 2;
};

int umma_tile() { return kTile; }

UmmaPlan* umma_plan_create(Ctx& c, const OperandPlanes& op, const BlockLayout& L, int chunk_stages) {
    if (op.fmt == OpFmt::F32) fail(STP_INVALID_ARGUMENT, "tensor-core contraction needs tiled operand images");
    auto p = std::make_unique<UmmaPlan>();
    if (chunk_stages != 1 && chunk_stages != 2) fail(STP_INVALID_ARGUMENT, "chunk stages must be 1 or 2");
    p->P = op.P;
    p->fmt = op.fmt;
    p->chunk_stages = chunk_stages;
    p->num_scale = 2.0 * op.scale_inv;
    const std::vector<WorkItem> items = make_work_items(L, op.P, kTile);
    p->n_items = static_cast<int>(items.size());
    // The same items grouped by block, for the one-launch-per-block comparison form.
    std::vector<WorkItem> by_block(items);
    std::stable_sort(by_block.begin(), by_block.end(), [](const WorkItem& x, const WorkItem& y) { return x.blk < y.blk; });
    p->block_item_off.assign(L.blocks.size() + 1, 0);
    for (const WorkItem& w : by_block) p->block_item_off[static_cast<size_t>(w.blk) + 1]++;
    for (size_t b = 0; b < L.blocks.size(); ++b) p->block_item_off[b + 1] += p->block_item_off[b];
    p->block_items.reserve(std::max<size_t>(by_block.size() * sizeof(WorkItem), 16));
    STPF2_CUDA(cudaMemcpyAsync(p->block_items.ptr, by_block.data(), by_block.size() * sizeof(WorkItem),
                               cudaMemcpyHostToDevice, c.stream));
    p->items.reserve(std::max<size_t>(items.size() * sizeof(WorkItem), 16));
    p->blocks.reserve(std::max<size_t>(L.blocks.size() * sizeof(BlockInfo), 16));
    p->err.reserve(16);
    p->counter.reserve(16);
    STPF2_CUDA(cudaMemcpyAsync(p->items.ptr, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                               c.stream));
    STPF2_CUDA(cudaMemcpyAsync(p->blocks.ptr, L.blocks.data(), L.blocks.size() * sizeof(BlockInfo),
                               cudaMemcpyHostToDevice, c.stream));
    STPF2_CUDA(cudaMemsetAsync(p->err.ptr, 0, 16, c.stream));
    int max_k = 0;
    for (const BlockInfo& b : L.blocks) max_k = std::max(max_k, b.k);
    std::vector<double> rcp(static_cast<size_t>(max_k) + 1, 0.0);
    for (int k = 1; k <= max_k; ++k) rcp[k] = 1.0 / static_cast<double>(k);
    p->rcp_max = max_k;
    p->rcp.reserve(rcp.size() * sizeof(double));
    STPF2_CUDA(cudaMemcpyAsync(p->rcp.ptr, rcp.data(), rcp.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    std::vector<int32_t> units, block_units;
    if (op.fmt == OpFmt::FX) {
        units = make_vpair_units(items);
        block_units = make_vpair_units(by_block);
        p->n_units = static_cast<int>(units.size());
        // Units never span two blocks, so each block's units are a run of block_units.
        p->block_unit_off.assign(L.blocks.size() + 1, 0);
        for (int32_t u : block_units) p->block_unit_off[static_cast<size_t>(by_block[u].blk) + 1]++;
        for (size_t b = 0; b < L.blocks.size(); ++b) p->block_unit_off[b + 1] += p->block_unit_off[b];
        p->units.reserve(std::max<size_t>(units.size() * sizeof(int32_t), 16));
        p->block_units.reserve(std::max<size_t>(block_units.size() * sizeof(int32_t), 16));
        STPF2_CUDA(cudaMemcpyAsync(p->units.ptr, units.data(), units.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                   c.stream));
        STPF2_CUDA(cudaMemcpyAsync(p->block_units.ptr, block_units.data(), block_units.size() * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, c.stream));
    }
    STPF2_CUDA(cudaStreamSynchronize(c.stream));  // the host tables above go out of scope

    if (op.n_rt <= 0 || op.n_ck <= 0) fail(STP_INVALID_ARGUMENT, "tensor-core contraction needs tiled planes");
    p->images = static_cast<const uint8_t*>(op.planes);
    p->n_ck = op.n_ck;
    if (op.fmt == OpFmt::FX) {
        p->mplanes = op.mplanes;
        p->vpc.reserve(fx_vpc_bytes(p->n_items));
        fx_prepare();
    } else {
        set_umma_smem();
    }
    return p.release();
}

void umma_plan_destroy(UmmaPlan* p) { delete p; }

void launch_umma_items(Ctx& c, UmmaPlan* p, const WorkItem* items, int n_items, double* f2, double* vpair,
                       cudaStream_t s, int b_base = 0, int b0 = -1, int b1 = -1);

void launch_f2_umma(Ctx& c, UmmaPlan* p, double* f2, double* vpair, cudaStream_t s, bool per_block) {
    if (!p || p->n_items <= 0) return;
    if (per_block) {  // comparison form: one launch per jackknife block
        for (size_t b = 0; b + 1 < p->block_item_off.size(); ++b) {
            const int n = p->block_item_off[b + 1] - p->block_item_off[b];
            if (n > 0)
                launch_umma_items(c, p, p->block_items.as<WorkItem>() + p->block_item_off[b], n, f2, vpair, s, 0,
                                  static_cast<int>(b), static_cast<int>(b) + 1);
        }
        return;
    }
    launch_umma_items(c, p, p->items.as<WorkItem>(), p->n_items, f2, vpair, s);
}

void launch_f2_umma_blocks(Ctx& c, UmmaPlan* p, int b0, int b1, double* f2, double* vpair, cudaStream_t s,
                           bool rebase) {
    if (!p || b1 <= b0) return;
    const int n = p->block_item_off[static_cast<size_t>(b1)] - p->block_item_off[static_cast<size_t>(b0)];
    if (n > 0)
        launch_umma_items(c, p, p->block_items.as<WorkItem>() + p->block_item_off[static_cast<size_t>(b0)], n, f2, vpair, s,
                          rebase ? b0 : 0, b0, b1);
}

// b0 < 0: items is the whole costliest-first list; otherwise the block_items of blocks
// b0..b1-1.
void launch_umma_items(Ctx& c, UmmaPlan* p, const WorkItem* items, int n_items, double* f2, double* vpair,
                       cudaStream_t s, int b_base, int b0, int b1) {
    if (p->fmt == OpFmt::FX) {
        FxLaunch L;
        L.images = p->images;
        L.mplanes = p->mplanes;
        L.n_ck = p->n_ck;
        L.items = items;
        L.n_items = n_items;
        if (b0 < 0) {
            L.units = p->units.as<int32_t>();
            L.n_units = p->n_units;
        } else {
            const int u0 = p->block_unit_off[static_cast<size_t>(b0)], u1 = p->block_unit_off[static_cast<size_t>(b1)];
            L.units = p->block_units.as<int32_t>() + u0;
            L.n_units = u1 - u0;
            L.unit_base = p->block_item_off[static_cast<size_t>(b0)];
        }
        L.blocks = p->blocks.as<BlockInfo>();
        L.P = p->P;
        L.f2 = f2;
        L.vpair = vpair;
        L.vpc = p->vpc.as<int32_t>();
        L.rcp = p->rcp.as<double>();
        L.rcp_max = p->rcp_max;
        L.err = p->err.as<int>();
        L.counters = p->counter.as<int>();
        L.b_base = b_base;
        launch_fx(c, L, s);
        return;
    }
    UmmaArgs a{};
    a.b_base = b_base;
    a.images = p->images;
    a.n_ck = p->n_ck;
    a.items = items;
    a.n_items = n_items;
    a.next_item = p->counter.as<int>();
    STPF2_CUDA(cudaMemsetAsync(a.next_item, 0, sizeof(int), s));
    a.blocks = p->blocks.as<BlockInfo>();
    a.P = p->P;
    a.f2 = f2;
    a.vpair = vpair;
    a.num_scale = p->num_scale;
    a.rcp = p->rcp.as<double>();
    a.rcp_max = p->rcp_max;
    a.err = p->err.as<int>();
    const bool bf16 = p->fmt == OpFmt::BF16;
    a.idesc_pp = idesc_f16(bf16, true);
    a.idesc_am = idesc_f16(bf16, false);
    a.idesc_i8 = idesc_u8_s32();
    const int grid = std::min(c.sm_count, n_items);
    launch_kernel(p->chunk_stages, false, grid, a, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFuncAttributes fa{};
        cudaFuncGetAttributes(&fa, f2_umma_kernel<2, false>);
        fail(STP_CUDA_ERROR, std::string("f2_umma_kernel launch: ") + cudaGetErrorString(e) + " (regs " +
                                 std::to_string(fa.numRegs) + ", max threads " + std::to_string(fa.maxThreadsPerBlock) +
                                 ", dyn smem " + std::to_string(kSmemBytes) + ", max dyn smem " +
                                 std::to_string(fa.maxDynamicSharedSizeBytes) + ", local " +
                                 std::to_string(fa.localSizeBytes) + ")");
    }
    c.launches++;
}

void launch_f2_umma_grouped(Ctx& c, OpFmt fmt, double scale_inv, int chunk_stages, const std::vector<GroupSpec>& groups,
                            cudaStream_t s, std::vector<unsigned long long>* stamps) {
    if (fmt == OpFmt::F32) fail(STP_INVALID_ARGUMENT, "tensor-core contraction needs tiled operand images");
    if (chunk_stages != 1 && chunk_stages != 2) fail(STP_INVALID_ARGUMENT, "chunk stages must be 1 or 2");
    const int G = static_cast<int>(groups.size());
    if (stamps) stamps->assign(static_cast<size_t>(G), 0ull);
    // Requests in ascending order of work (shortest first: lower median completion), each
    // request's items costliest-first and its tile pairs together.
    std::vector<double> cost(static_cast<size_t>(G), 0.0);
    for (int g = 0; g < G; ++g) {
        const int T = (groups[g].info.P + kTile - 1) / kTile;
        for (const BlockInfo& b : groups[g].L->blocks) cost[g] += static_cast<double>(stages_of_host(b.k)) * T * (T + 1) / 2;
    }
    std::vector<int> ord(static_cast<size_t>(G));
    for (int g = 0; g < G; ++g) ord[g] = g;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return cost[x] < cost[y]; });
    std::vector<BlockInfo> blocks;
    std::vector<WorkItem> items;
    std::vector<int> n_items(static_cast<size_t>(G), 0);
    std::vector<GroupInfo> info(static_cast<size_t>(G));
    int max_k = 0;
    for (int g : ord) {
        const BlockLayout& L = *groups[g].L;
        info[g] = groups[g].info;
        const int base = static_cast<int>(blocks.size());
        for (BlockInfo b : L.blocks) {
            b.grp = g;
            blocks.push_back(b);
            max_k = std::max(max_k, b.k);
        }
        if (info[g].P <= 0) continue;
        for (WorkItem w : make_work_items(L, info[g].P, kTile)) {
            w.blk += base;
            items.push_back(w);
            n_items[g]++;
        }
    }
    if (items.empty()) return;
    if (items.size() > static_cast<size_t>(INT_MAX)) fail(STP_RUNTIME_ERROR, "too many work items in one batch");
    std::vector<double> rcp(static_cast<size_t>(max_k) + 1, 0.0);
    for (int k = 1; k <= max_k; ++k) rcp[k] = 1.0 / static_cast<double>(k);
    // Every table in one pinned staging buffer and one upload; counters cleared on device.
    Packing pk;
    const size_t o_items = pk.add(items.size() * sizeof(WorkItem));
    const size_t o_blocks = pk.add(blocks.size() * sizeof(BlockInfo));
    const size_t o_info = pk.add(info.size() * sizeof(GroupInfo));
    const size_t o_rcp = pk.add(rcp.size() * sizeof(double));
    const size_t o_nitems = pk.add(n_items.size() * sizeof(int));
    const bool fx = fmt == OpFmt::FX;
    const std::vector<int32_t> units = fx ? make_vpair_units(items) : std::vector<int32_t>();
    const size_t o_units = pk.add(units.size() * sizeof(int32_t));
    const size_t staged = pk.end;
    const size_t o_done = pk.add(static_cast<size_t>(G) * sizeof(int));
    const size_t o_ns = pk.add(static_cast<size_t>(G) * sizeof(unsigned long long));
    const size_t o_err = pk.add(16);
    const size_t o_counter = pk.add(16);
    if (fx) c.ws_vpc.reserve(fx_vpc_bytes(static_cast<int>(items.size())));
    c.pin_items.reserve(staged);
    c.ws_items.reserve(pk.end);
    uint8_t* h = c.pin_items.as<uint8_t>();
    std::memcpy(h + o_items, items.data(), items.size() * sizeof(WorkItem));
    std::memcpy(h + o_blocks, blocks.data(), blocks.size() * sizeof(BlockInfo));
    std::memcpy(h + o_info, info.data(), info.size() * sizeof(GroupInfo));
    std::memcpy(h + o_rcp, rcp.data(), rcp.size() * sizeof(double));
    std::memcpy(h + o_nitems, n_items.data(), n_items.size() * sizeof(int));
    if (!units.empty()) std::memcpy(h + o_units, units.data(), units.size() * sizeof(int32_t));
    uint8_t* d = c.ws_items.as<uint8_t>();
    STPF2_CUDA(cudaMemcpyAsync(d, h, staged, cudaMemcpyHostToDevice, s));
    STPF2_CUDA(cudaMemsetAsync(d + staged, 0, pk.end - staged, s));
    if (fx) {
        fx_prepare();
        FxLaunch L;
        L.images = info[ord[0]].images;
        L.mplanes = info[ord[0]].mplanes;
        L.n_ck = info[ord[0]].n_ck;
        L.P = info[ord[0]].P;
        L.f2 = info[ord[0]].f2;
        L.vpair = info[ord[0]].vpair;
        L.items = reinterpret_cast<const WorkItem*>(d + o_items);
        L.n_items = static_cast<int>(items.size());
        L.units = reinterpret_cast<const int32_t*>(d + o_units);
        L.n_units = static_cast<int>(units.size());
        L.blocks = reinterpret_cast<const BlockInfo*>(d + o_blocks);
        L.vpc = c.ws_vpc.as<int32_t>();
        L.rcp = reinterpret_cast<const double*>(d + o_rcp);
        L.rcp_max = max_k;
        L.err = reinterpret_cast<int*>(d + o_err);
        L.counters = reinterpret_cast<int*>(d + o_counter);
        L.groups = reinterpret_cast<const GroupInfo*>(d + o_info);
        L.grp_done = reinterpret_cast<int*>(d + o_done);
        L.grp_ns = reinterpret_cast<unsigned long long*>(d + o_ns);
        L.grp_items = reinterpret_cast<const int*>(d + o_nitems);
        launch_fx(c, L, s);
    } else {
    set_umma_smem();

    UmmaArgs a{};
    a.images = info[ord[0]].images;
    a.n_ck = info[ord[0]].n_ck;
    a.P = info[ord[0]].P;
    a.f2 = info[ord[0]].f2;
    a.vpair = info[ord[0]].vpair;
    a.items = reinterpret_cast<const WorkItem*>(d + o_items);
    a.n_items = static_cast<int>(items.size());
    a.next_item = reinterpret_cast<int*>(d + o_counter);
    a.blocks = reinterpret_cast<const BlockInfo*>(d + o_blocks);
    a.num_scale = 2.0 * scale_inv;
    a.rcp = reinterpret_cast<const double*>(d + o_rcp);
    a.rcp_max = max_k;
    a.err = reinterpret_cast<int*>(d + o_err);
    const bool bf16 = fmt == OpFmt::BF16;
    a.idesc_pp = idesc_f16(bf16, true);
    a.idesc_am = idesc_f16(bf16, false);
    a.idesc_i8 = idesc_u8_s32();
    a.groups = reinterpret_cast<const GroupInfo*>(d + o_info);
    a.grp_done = reinterpret_cast<int*>(d + o_done);
    a.grp_ns = reinterpret_cast<unsigned long long*>(d + o_ns);
    a.grp_items = reinterpret_cast<const int*>(d + o_nitems);
    const int grid = std::min(c.sm_count, a.n_items);
    launch_kernel(chunk_stages, true, grid, a, s);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
    }
    int err = 0;
    STPF2_CUDA(cudaMemcpyAsync(&err, d + o_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (stamps)
        STPF2_CUDA(cudaMemcpyAsync(stamps->data(), d + o_ns, static_cast<size_t>(G) * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, s));
    STPF2_CUDA(cudaStreamSynchronize(s));
    if (err) fail(STP_DEVICE_TIMEOUT, "grouped tensor-core contraction: a bounded device wait expired; results are invalid");
}

namespace {
__global__ void timestamp_kernel(unsigned long long* dst) { *dst = globaltimer(); }
}  // namespace

void launch_timestamp(Ctx& c, unsigned long long* dst, cudaStream_t s) {
    timestamp_kernel<<<1, 1, 0, s>>>(dst);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

// Reads (and clears) the kernel's timeout flag; call after the stream has synchronised.
void umma_check(UmmaPlan* p) {
    if (!p) return;
    int e = 0;
    STPF2_CUDA(cudaMemcpy(&e, p->err.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        STPF2_CUDA(cudaMemset(p->err.ptr, 0, sizeof(int)));
        fail(STP_DEVICE_TIMEOUT, "tensor-core contraction: a bounded device wait expired; results are invalid");
    }
}

}  // namespace stpf2
