// steppecu_b200/csrc/f2_fx.cu
//
// The fixed-point f2 contraction (STP_PREC_FIXED_I8) for sm_100a: exact integer tensor-core
// sums over 32-bit fixed-point operands, two persistent warp-specialised kernels over every
// (jackknife block, 128x128 population tile pair ti <= tj) work item.
//
// Operands (decode.cu, emit8_fx): per population and SNP, X = round((q - 1/2) S) and
// A = round((x^2 - h) S^2 / 2^31) with S = kFxScale, each as four balanced int8 digits
// (X = sum_d X_d 256^d, X_d in [-128, 127]), plus M = 64 [n > 0]; a missing population has
// X = A = M = 0. With T = (x_i - x_j)^2 - h_i - h_j = a_i + a_j - 2 x_i x_j
// (f2_estimator.hpp:29-36) the block numerator sum_s T over SNPs where both are called is
//     -2 / S^2 * sum_s [ X_i X_j - 2^24 (A_i M_j + M_i A_j) ]
// and f2_fx_kernel computes the bracket in four int32 TMEM accumulators V_3..V_6 of weight
// 256^3..256^6, exactly but for the dropped low digit products:
//     V_w += X_a(i) X_b(j)        for a + b = w        (products of weight below 256^3 are
//                                                       dropped: under 3.1 * 2^30 / S^2,
//                                                       i.e. 1.7e-10, per SNP)
//     V_w += E_w(i) M(j) + M(i) E_w(j)                  (E_3..E_6: the digits of -A)
// i.e. 18 kind::i8 products (M = N = 128, K = 32) per 32-SNP stage, all integer and exact,
// issued as 12 MMAs: where two products of one A operand go into adjacent weights from
// adjacent B planes, one MMA of N = 256 covers both.
// The epilogue forms W = sum_w V_w 256^(w-3) exactly in int64 once per tile (every 16,384
// SNPs of a longer block, the int32 bound; segments add in FP64), f2 = W * kFxNumScale /
// vpair (0 when vpair = 0, f2_estimator.hpp:42-46), and stores (i,j) and (j,i) of the
// block's slab.
//
// Error against exact arithmetic, per SNP and pair: the two roundings of x (2^-32.0 each,
// times |x| <= 1/2, twice), of a (2^-33, twice) and the dropped digit products: under
// 7e-10 on T; a block mean over K SNPs averages independent roundings (~1e-10 / sqrt(K)).
//
// vpair_fx_kernel runs first over the same items: the exact both-present counts
// m_i . m_j (kind::i8 MMAs on the M tiles, 64 m on both sides, so 4096 per SNP; two items
// of one row tile per unit where the next column tile follows; 128 SNPs per stage, a ring
// of two 256-column TMEM accumulators, at most 524,032 SNPs per accumulation) written as
// one compact int32 128x128 tile per item, which the f2 epilogue reads for its divide and
// its vpair stores. (The four f2 accumulators fill TMEM's 512 columns, so the counts
// cannot share the f2 kernel.)
//
//   f2_fx_kernel:   warp 0 producer (a 32 KiB image and a 4 KiB M copy per stage side, no
//                   tensor maps, no multicast), warp 1 TMEM owner + single-thread MMA issuer, warps 2-17
//                   epilogue (four per TMEM lane quarter, 32 tile columns each).
//   vpair_fx_kernel: warp 0 producer (16 KiB of A and of each column tile per stage),
//                   warp 1 issuer, warps 2-9 epilogue (two per lane quarter, one item each).
// Every wait is bounded (FxTuning::timeout_ns); on expiry the kernel raises an error flag
// the host turns into STP_DEVICE_TIMEOUT, lets its copies and MMAs finish, frees TMEM and
// returns.
#include <algorithm>
#include <climits>

#include "stpf2_internal.cuh"
#include "umma_ptx.cuh"

namespace stpf2 {

namespace {

using namespace ptx;

constexpr int kTile = 128;
constexpr int kStageK = 32;
constexpr int kItemRing = 4;
constexpr int kVpTileInts = kTile * kTile;  // one compact vpair tile: (row r, column c) at c * 128 + r

// ---- f2 kernel constants ----
constexpr int kStages = 3;
constexpr uint32_t kSide = static_cast<uint32_t>(kFxPlanes * kTile8Bytes);  // 36 KiB: image and M
constexpr uint32_t kStageBytes = 2 * kSide;
constexpr int kEpiWarps = 16;
constexpr int kEpiWarp0 = 2;
constexpr int kThreads = 32 * (kEpiWarp0 + kEpiWarps);  // 576
constexpr int kCols = 4 * kTile / kEpiWarps;            // 32 tile columns per epilogue thread
constexpr int kSegStages = 512;  // 16,384 SNPs: |V_3| < 81,920 per SNP stays below 2^31
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kCtlBytes = 256;

// ---- vpair kernel constants ----
constexpr int kVpChunks = 4;  // 32-SNP chunks per stage
constexpr uint32_t kVpASide = kVpChunks * static_cast<uint32_t>(kTile8Bytes);  // 16 KiB
constexpr uint32_t kVpStageBytes = 3 * kVpASide;  // A, then the two column tiles
constexpr int kVpStages = 4;
constexpr int kVpAcc = 2;  // TMEM ring of 256-column accumulators
constexpr uint32_t kVpAccCols = 2 * kTile;
constexpr int kVpEpiWarps = 8;
constexpr int kVpThreads = 32 * (2 + kVpEpiWarps);  // 320
// 32-SNP chunks per accumulation: M = 64 on both sides adds 4096 per both-present SNP, so
// an int32 accumulator holds 524,032 SNPs (a whole number of stages).
constexpr int kVpPartChunks = 16376;
static_assert(4096ll * 32 * kVpPartChunks < (1ll << 31) && kVpPartChunks % kVpChunks == 0, "vpair part");
static_assert(kVpStages >= kStages && kVpAcc * kVpAccCols <= 512, "barrier and TMEM slots");

struct FxArgs {
    const uint8_t* images;   // (row tile t, chunk c) image at (t * n_ck + c) * kFxImageBytes
    const uint8_t* mplanes;  // (row tile t, chunk c) M tile at (t * n_ck + c) * 4 KiB
    int64_t n_ck;
    const WorkItem* items;
    int n_items;
    const BlockInfo* blocks;
    int P;
    double* f2;
    double* vpair;
    int32_t* vpc;  // compact vpair tiles, item it at vpc + it * kVpTileInts
    const double* rcp;  // rcp[k] = 1/k, k = 0..rcp_max (rcp[0] = 0)
    int rcp_max;
    int* err;
    int* next_item;  // work-item (f2) or unit (vpair) counter, zero at launch
    const int32_t* units;  // vpair units: first item of each, as an index past unit_base
    int n_units;
    int unit_base;
    int b_base;      // block id whose slab starts the output buffers
    uint32_t idesc;
    unsigned long long timeout_ns;
    long long withhold;  // test hook: the producer stops before its stage of this index (-1: never)
    uint32_t partial_feed;  // bit k: a side with 8k+1 .. 8k+8 valid rows copies those rows only
    const GroupInfo* groups;  // grouped launch: per-request images / outputs (null for one request)
    int* grp_done;
    unsigned long long* grp_ns;
    const int* grp_items;
};

struct FxCtl {
    unsigned long long item_full[kItemRing], item_empty[kItemRing];
    int item_idx[kItemRing];
    unsigned long long full[kVpStages], empty[kVpStages];  // f2 kernel uses the first kStages
    unsigned long long acc_full[kVpAcc], acc_empty[kVpAcc];  // f2 kernel uses slot 0 only
    unsigned long long drain;
    uint32_t tmem_base;
    volatile int abort;
};
static_assert(sizeof(FxCtl) <= kCtlBytes, "barrier block overflows its slot");

__device__ __forceinline__ bool waitb(unsigned long long* b, uint32_t parity, FxCtl* ctl, const FxArgs& a,
                                      bool honour_abort = true) {
    return wait_bounded(b, parity, &ctl->abort, a.err, a.timeout_ns, honour_abort);
}

__device__ __forceinline__ int stages_of(int k, int per) { return (k + per - 1) / per; }

// The MMA width of a tile pair: the column tile's populations rounded up to the N step of
// 16 (at most 128). Columns past the last population are never stored, so a short last
// column tile costs only its own columns of tensor work.
template <bool kGrouped>
__device__ __forceinline__ uint32_t idesc_for(const FxArgs& a, const WorkItem& w, const BlockInfo& bi) {
    const int P = kGrouped ? a.groups[bi.grp].P : a.P;
    const int cols = min(kTile, P - w.tj * kTile);
    const uint32_t n = static_cast<uint32_t>((cols + 15) & ~15);
    return (a.idesc & ~(0x3Fu << 17)) | ((n >> 3) << 17);
}

// Work items in list order from a global counter (costliest block first, a block's tile
// pairs together), handed from the producer to the other roles through a small ring.
__device__ __forceinline__ int take_item(const FxArgs& a, FxCtl* ctl, uint32_t gi, bool& ok) {
    const int slot = static_cast<int>(gi % kItemRing);
    ok = waitb(&ctl->item_empty[slot], ((gi / kItemRing) & 1u) ^ 1u, ctl, a);
    if (!ok) return -1;
    int it = atomicAdd(a.next_item, 1);
    if (it >= a.n_items) it = -1;
    *reinterpret_cast<volatile int*>(&ctl->item_idx[slot]) = it;
    mbar_arrive(&ctl->item_full[slot]);
    return it;
}

__device__ __forceinline__ int read_item(const FxArgs& a, FxCtl* ctl, uint32_t gi) {
    const int slot = static_cast<int>(gi % kItemRing);
    if (!waitb(&ctl->item_full[slot], (gi / kItemRing) & 1u, ctl, a)) return -2;
    const int it = *reinterpret_cast<volatile int*>(&ctl->item_idx[slot]);
    mbar_arrive(&ctl->item_empty[slot]);
    return it;
}

__device__ __forceinline__ void init_ring(FxCtl* ctl, int consumers) {
    for (int s = 0; s < kItemRing; ++s) {
        mbar_init(&ctl->item_full[s], 1);
        mbar_init(&ctl->item_empty[s], consumers);
    }
}

// ============================== f2 kernel ================================================

// 8-row groups a stage copies of an operand side with `rows` valid populations: all 16
// (the whole tile in one copy per region), or only the groups holding valid rows when the
// side's row class is marked for partial copies. Rows past the valid ones are never read
// into a stored result: A rows past them make accumulator rows past P, B rows make columns
// past P, and the epilogue stores neither, so whatever the stage slot held there is harmless.
__device__ __forceinline__ uint32_t feed_groups(const FxArgs& a, int rows) {
    const int cls = (rows + 7) / 8 - 1;  // 0..15
    return ((a.partial_feed >> cls) & 1u) ? static_cast<uint32_t>(cls + 1) : 16u;
}

// One stage side: image planes 0..7 and the M tile (plane 8), `g` 8-row groups of each.
__device__ __forceinline__ uint32_t side_bytes(uint32_t g) { return g == 16 ? kSide : 9u * g * 256u; }

__device__ __forceinline__ void copy_side(uint8_t* dst, const uint8_t* img, const uint8_t* mt, uint32_t g,
                                          unsigned long long* bar) {
    constexpr uint32_t kImg = static_cast<uint32_t>(kFxImageBytes), kM = static_cast<uint32_t>(kTile8Bytes);
    if (g == 16) {
        bulk_load(dst, img, kImg, bar);      // planes 0..7
        bulk_load(dst + kImg, mt, kM, bar);  // plane 8
        return;
    }
    const uint32_t b = g * 256u;
#pragma unroll 1
    for (int pl = 0; pl < 8; ++pl) bulk_load(dst + pl * kM, img + pl * kM, b, bar);
    bulk_load(dst + kImg, mt, b, bar);
}

template <bool kGrouped>
__device__ void fx_producer(const FxArgs& a, uint8_t* smem, FxCtl* ctl) {
    uint32_t g = 0;
    for (uint32_t gi = 0;; ++gi) {
        bool ok = true;
        const int it = take_item(a, ctl, gi, ok);
        if (!ok) goto abort;
        if (it < 0) break;
        {
            const WorkItem w = a.items[it];
            const BlockInfo bi = a.blocks[w.blk];
            const int nst = stages_of(bi.k, kStageK);
            const bool diag = w.ti == w.tj;
            const uint8_t* images = a.images;
            const uint8_t* mplanes = a.mplanes;
            int64_t n_ck = a.n_ck;
            if constexpr (kGrouped) {
                images = a.groups[bi.grp].images;
                mplanes = a.groups[bi.grp].mplanes;
                n_ck = a.groups[bi.grp].n_ck;
            }
            const int P = kGrouped ? a.groups[bi.grp].P : a.P;
            const uint32_t gA = feed_groups(a, min(kTile, P - w.ti * kTile));
            const uint32_t gB = feed_groups(a, min(kTile, P - w.tj * kTile));
            const uint32_t bytes = diag ? side_bytes(gA) : side_bytes(gA) + side_bytes(gB);
            for (int st = 0; st < nst; ++st, ++g) {
                if (static_cast<long long>(g) == a.withhold) return;  // test hook: stop feeding
                const int slot = static_cast<int>(g % kStages);
                if (!waitb(&ctl->empty[slot], ((g / kStages) & 1u) ^ 1u, ctl, a)) goto abort;
                uint8_t* sb = smem + slot * kStageBytes;
                mbar_expect_tx(&ctl->full[slot], bytes);
                const int64_t ci = static_cast<int64_t>(w.ti) * n_ck + bi.col / kStageK + st;
                copy_side(sb, images + ci * kFxImageBytes, mplanes + ci * kTile8Bytes, gA, &ctl->full[slot]);
                if (!diag) {
                    const int64_t cj = static_cast<int64_t>(w.tj) * n_ck + bi.col / kStageK + st;
                    copy_side(sb + kSide, images + cj * kFxImageBytes, mplanes + cj * kTile8Bytes, gB, &ctl->full[slot]);
                }
            }
        }
    }
    return;
abort:
    // Let the copies already issued land before the CTA's shared memory goes away.
    for (uint32_t k = (g >= kStages ? g - kStages : 0); k < g; ++k)
        waitb(&ctl->full[k % kStages], (k / kStages) & 1u, ctl, a, false);
}

template <bool kGrouped>
__device__ void fx_issuer(const FxArgs& a, uint8_t* smem, FxCtl* ctl, uint32_t tmem) {
    uint32_t g = 0, cs = 0;
    const uint32_t V3 = tmem, V4 = tmem + 128u, V5 = tmem + 256u, V6 = tmem + 384u;
    for (uint32_t gi = 0;; ++gi) {
        const int it = read_item(a, ctl, gi);
        if (it < 0) break;
        const WorkItem w = a.items[it];
        const BlockInfo bi = a.blocks[w.blk];
        const int nst = stages_of(bi.k, kStageK);
        const uint32_t id = idesc_for<kGrouped>(a, w, bi);
        // The same shape with N = 128 + n: two adjacent B planes into two adjacent weights.
        const uint32_t id2 = (id & ~(0x3Fu << 17)) | ((((id >> 17) & 0x3Fu) + 16u) << 17);
        const bool diag = w.ti == w.tj;
        for (int st = 0; st < nst; ++st, ++g) {
            const int sseg = st % kSegStages;
            if (sseg == 0) {  // the epilogue has read the accumulators of the previous segment
                if (!waitb(&ctl->acc_empty[0], (cs & 1u) ^ 1u, ctl, a)) goto done;
                tc_fence_after();
            }
            const int slot = static_cast<int>(g % kStages);
            if (!waitb(&ctl->full[slot], (g / kStages) & 1u, ctl, a)) goto done;
            tc_fence_after();
            {
                const uint32_t sa = smem_u32(smem + slot * kStageBytes);
                const uint32_t sb = diag ? sa : sa + kSide;
                auto dA = [&](int t) { return smem_desc(sa + static_cast<uint32_t>(t) * 4096u, 256, 6); };
                auto dB = [&](int t) { return smem_desc(sb + static_cast<uint32_t>(t) * 4096u, 256, 6); };
                const uint32_t f = sseg == 0 ? 0u : 1u;  // the first stage of a segment overwrites
                using C = CollectorA;
                // Planes are 4 KiB apart and V_3..V_6 128 TMEM columns apart, so an MMA of
                // N = 128 + n on two adjacent B planes fills two adjacent weights at once
                // (columns 0..n-1 from the first plane, 128.. from the second): 12 MMAs per
                // stage for the 18 digit products, A kept in the collector buffer across the
                // two MMAs that share it (X3, X2 and M: nine A reads per stage).
                mma_i8_c<C::kFill>(V3, dA(3), dB(0), id2, f);     // X3 [X0;X1] -> V3,V4
                mma_i8_c<C::kLastUse>(V5, dA(3), dB(2), id2, f);  // X3 [X2;X3] -> V5,V6
                mma_i8_c<C::kFill>(V3, dA(2), dB(1), id, 1u);     // X2 X1      -> V3
                mma_i8_c<C::kLastUse>(V4, dA(2), dB(2), id2, 1u); // X2 [X2;X3] -> V4,V5
                mma_i8(V3, dA(1), dB(2), id2, 1u);                // X1 [X2;X3] -> V3,V4
                mma_i8(V3, dA(0), dB(3), id, 1u);                 // X0 X3      -> V3
                // M(i) E_w(j) on the stacked E planes, and E_w(i) M(j): tiles 4..7 are
                // E_3..E_6, tile 8 is M.
                mma_i8_c<C::kFill>(V3, dA(8), dB(4), id2, 1u);     // M [E3;E4] -> V3,V4
                mma_i8_c<C::kLastUse>(V5, dA(8), dB(6), id2, 1u);  // M [E5;E6] -> V5,V6
                mma_i8(V3, dA(4), dB(8), id, 1u);
                mma_i8(V4, dA(5), dB(8), id, 1u);
                mma_i8(V5, dA(6), dB(8), id, 1u);
                mma_i8(V6, dA(7), dB(8), id, 1u);
            }
            mma_commit(&ctl->empty[slot]);
            if (sseg == kSegStages - 1 || st == nst - 1) {
                mma_commit(&ctl->acc_full[0]);
                ++cs;
            }
        }
    }
done:
    // Every MMA this thread issued completes before TMEM is released.
    mma_commit(&ctl->drain);
    waitb(&ctl->drain, 0u, ctl, a, false);
}

struct ItemOut {
    double* f2;
    double* vp;
    int64_t slab;
    int P, i, j0, i0, grp;
    bool diag;
};

template <bool kGrouped>
__device__ __forceinline__ ItemOut item_out(const FxArgs& a, int it, int r, int h, int cols) {
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
    o.j0 = w.tj * kTile + h * cols;
    o.slab = static_cast<int64_t>(o.P) * o.P * (bi.b - a.b_base);
    return o;
}

template <bool kGrouped>
__device__ __forceinline__ void stamp(const FxArgs& a, int grp, int lane) {
    if (!kGrouped || !a.grp_done) return;
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        const int d = atomicAdd(a.grp_done + grp, 1);
        if (d == a.grp_items[grp] * kEpiWarps - 1) a.grp_ns[grp] = globaltimer();
    }
}

// int64 -> FP64 without a conversion instruction: each 32-bit half is placed in the
// mantissa of 2^52 (2^52 + 2^31 for the signed high half) by its bit pattern and the bias
// subtracted exactly; hi * 2^32 + lo then rounds once (a correctly rounded conversion).
__device__ __forceinline__ double i64_to_f64(int64_t w) {
    const int lo = static_cast<int>(static_cast<uint32_t>(w));
    const int hi = static_cast<int>(static_cast<uint32_t>(static_cast<uint64_t>(w) >> 32) ^ 0x80000000u);
    const double dl = __hiloint2double(0x43300000, lo) - 4503599627370496.0;  // 2^52
    const double dh = __hiloint2double(0x43300000, hi) - 4503601774854144.0;  // 2^52 + 2^31
    return fma(dh, 4294967296.0, dl);
}

__device__ __forceinline__ void st_cs_v2(double* p, double x, double y) {
    asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(x), "d"(y) : "memory");
}

__device__ __forceinline__ void st_cs_v4(double* p, double x, double y, double z, double w) {
    asm volatile("st.global.cs.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(x), "d"(y), "d"(z), "d"(w) : "memory");
}

// Eight consecutive doubles v[0..7] to p, where p's element offset is kP modulo 4 (the run
// starts kP elements past a 32-byte boundary): scalar and 16-byte stores up to the boundary,
// then 32-byte stores, then the tail. Each 32-byte store fills one sector.
template <int kP>
__device__ __forceinline__ void store_run8(double* p, const double (&v)[8]) {
    constexpr int head = (4 - kP) & 3;  // elements before the first 32-byte boundary
    int k = 0;
    if constexpr (head & 1) { __stcs(p, v[0]); k = 1; }
    if constexpr (head & 2) { st_cs_v2(p + k, v[k], v[k + 1]); k += 2; }
    st_cs_v4(p + k, v[k], v[k + 1], v[k + 2], v[k + 3]);
    if constexpr (head == 0) st_cs_v4(p + 4, v[4], v[5], v[6], v[7]);
    else {
        k += 4;
        if constexpr (((8 - head - 4) & 2) != 0) { st_cs_v2(p + k, v[k], v[k + 1]); k += 2; }
        if constexpr (((8 - head - 4) & 1) != 0) __stcs(p + k, v[k]);
    }
}

__device__ __forceinline__ void store_run8(double* p, const double (&v)[8]) {
    switch (static_cast<int>((reinterpret_cast<uintptr_t>(p) >> 3) & 3u)) {
        case 0: store_run8<0>(p, v); break;
        case 1: store_run8<1>(p, v); break;
        case 2: store_run8<2>(p, v); break;
        default: store_run8<3>(p, v); break;
    }
}

template <bool kGrouped>
__device__ void fx_epilogue(const FxArgs& a, FxCtl* ctl, uint32_t tmem, int warp, int lane) {
    const int e = warp - kEpiWarp0;
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int h = e >> 2;    // column part of the tile
    const int r = q * 32 + lane;
    const uint32_t lane_addr = static_cast<uint32_t>(q * 32) << 16;
    const uint32_t col_addr = static_cast<uint32_t>(h * kCols);
    uint32_t cs = 0;
    double acc[kCols];  // W of this thread's row and columns
    for (uint32_t gi = 0;; ++gi) {
        int it = 0;
        if (lane == 0) it = read_item(a, ctl, gi);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it < 0) return;
        const int nst = stages_of(a.blocks[a.items[it].blk].k, kStageK);
        if (nst == 0) {  // an empty block id: zeros (cpu_backend.cpp:234)
            const ItemOut o = item_out<kGrouped>(a, it, r, h, kCols);
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
        // This thread's counts: column c of its part at vpt + c * 128 (+ lane). Pull the
        // warp's 32 lines into L2 while the MMAs run.
        const int32_t* vpt = a.vpc + static_cast<int64_t>(it) * kVpTileInts + (h * kCols) * kTile + q * 32;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(vpt + lane * kTile));
#pragma unroll
        for (int c = 0; c < kCols; ++c) acc[c] = 0.0;
        const int nseg = (nst + kSegStages - 1) / kSegStages;
        for (int sg = 0; sg < nseg; ++sg) {
            bool ok = true;
            if (lane == 0) ok = waitb(&ctl->acc_full[0], cs & 1u, ctl, a);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) return;
            tc_fence_after();
#pragma unroll
            for (int g8 = 0; g8 < kCols / 8; ++g8) {
                // Columns g8*8.. of V_3..V_6, one wait for the four loads.
                uint32_t v[4][8];
#pragma unroll
                for (int w = 0; w < 4; ++w)
                    tmem_ld8(tmem + lane_addr + static_cast<uint32_t>(w) * 128u + col_addr + static_cast<uint32_t>(g8) * 8u,
                             v[w]);
                tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    // W of the segment, exact in int64 (|W| < 2^56), then one rounding to FP64.
                    const int64_t w = static_cast<int64_t>(static_cast<int32_t>(v[0][c])) +
                                      (static_cast<int64_t>(static_cast<int32_t>(v[1][c])) << 8) +
                                      (static_cast<int64_t>(static_cast<int32_t>(v[2][c])) << 16) +
                                      (static_cast<int64_t>(static_cast<int32_t>(v[3][c])) << 24);
                    acc[g8 * 8 + c] += i64_to_f64(w);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl->acc_empty[0]);
            ++cs;
        }
        // Output: (i, j) straight from registers (32 consecutive i per store: full sectors);
        // (j, i) from the same registers, as this row's run of 8 consecutive j per column
        // group (32-byte stores where the run allows; per element at the tile's diagonal
        // and right edge).
        const ItemOut o = item_out<kGrouped>(a, it, r, h, kCols);
        const int P = o.P, i = o.i, j0 = o.j0;
        const bool diag = o.diag;
        const int64_t row_i = o.slab + i;
        const int64_t col_i = o.slab + static_cast<int64_t>(P) * i;
#pragma unroll
        for (int q8 = 0; q8 < kCols / 8; ++q8) {
            int32_t vpi[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) vpi[c] = __ldg(vpt + (q8 * 8 + c) * kTile + lane);
            double f8[8], v8[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int col = q8 * 8 + c;
                const int j = j0 + col;
                const int32_t vk = vpi[c] < a.rcp_max ? vpi[c] : a.rcp_max;
                f8[c] = vk > 0 ? acc[col] * kFxNumScale * __ldg(a.rcp + vk) : 0.0;
                v8[c] = static_cast<double>(vpi[c]);
                if (i < P && j < P && !(diag && j < i)) {
                    const int64_t ij = row_i + static_cast<int64_t>(P) * j;
                    __stcs(o.f2 + ij, f8[c]);
                    __stcs(o.vp + ij, v8[c]);
                }
            }
            const int jr = j0 + q8 * 8;  // the run's first j
            if (i < P && jr + 7 < P && !(diag && jr <= i)) {
                store_run8(o.f2 + col_i + jr, f8);
                store_run8(o.vp + col_i + jr, v8);
            } else if (i < P) {
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int j = jr + c;
                    if (j < P && !(diag && j <= i)) {
                        __stcs(o.f2 + col_i + j, f8[c]);
                        __stcs(o.vp + col_i + j, v8[c]);
                    }
                }
            }
            // Keep the next group's count loads after this group's stores (they would
            // otherwise all be hoisted, and held, at once).
            asm volatile("" ::: "memory");
        }
        stamp<kGrouped>(a, o.grp, lane);
    }
}

template <bool kGrouped>
// 18 warps put five on two SM sub-partitions: at most 96 registers per thread.
__global__ void __maxnreg__(96)
f2_fx_kernel(const __grid_constant__ FxArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    FxCtl* ctl = reinterpret_cast<FxCtl*>(smem + kStages * kStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        init_ring(ctl, 1 + kEpiWarps);  // the issuer and every epilogue warp
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        mbar_init(&ctl->acc_full[0], 1);
        mbar_init(&ctl->acc_empty[0], kEpiWarps);
        mbar_init(&ctl->drain, 1);
        ctl->abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(&ctl->tmem_base, kTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;
    if (warp < kEpiWarp0) {
        if (warp == 0 && lane == 0) fx_producer<kGrouped>(a, smem, ctl);
        if (warp == 1 && lane == 0) fx_issuer<kGrouped>(a, smem, ctl, tmem);
    } else {
        fx_epilogue<kGrouped>(a, ctl, tmem, warp, lane);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, kTmemCols);
}

constexpr size_t kFxSmemBytes = kStages * kStageBytes + kCtlBytes + 1024;

// ============================== vpair kernel ==============================================
//
// A unit is one work item, or two when the second is the next column tile of the first's
// row (vpair_pairs_with): the A tile is copied once for both, and per 32-SNP chunk two MMAs
// share it from the collector buffer, one per column tile, into the two 128-column halves
// of one accumulator. A stage holds A, then the first column tile's chunks, then the
// second's, each region one bulk copy of consecutive chunks (a partial side: one copy of
// its valid 8-row groups per chunk). A diagonal unit reads A from the first B region. A
// paired unit's row tile and first column tile are whole (a later column tile exists), so
// only its second column tile can be a partial side.

// The unit's second item, or -1.
__device__ __forceinline__ int vp_second(const FxArgs& a, int it) {
    return it + 1 < a.n_items && vpair_pairs_with(a.items[it], a.items[it + 1]) ? it + 1 : -1;
}

// Units in list order from the vpair counter, the next one claimed while this one streams
// (u_next: the claim made one unit earlier); the ring carries the unit's first item.
__device__ __forceinline__ int take_unit(const FxArgs& a, FxCtl* ctl, uint32_t gi, int& u_next, bool& ok) {
    const int slot = static_cast<int>(gi % kItemRing);
    ok = waitb(&ctl->item_empty[slot], ((gi / kItemRing) & 1u) ^ 1u, ctl, a);
    if (!ok) return -1;
    const int u = u_next;
    const int it = u < a.n_units ? __ldg(a.units + u) - a.unit_base : -1;
    *reinterpret_cast<volatile int*>(&ctl->item_idx[slot]) = it;
    mbar_arrive(&ctl->item_full[slot]);
    if (it >= 0) u_next = atomicAdd(a.next_item, 1);
    return it;
}

// MMA shape for column tile t: its populations rounded up to 16.
template <bool kGrouped>
__device__ __forceinline__ uint32_t vp_idesc(const FxArgs& a, const BlockInfo& bi, int t) {
    const int P = kGrouped ? a.groups[bi.grp].P : a.P;
    const int cols = min(kTile, P - t * kTile);
    const uint32_t n = static_cast<uint32_t>((cols + 15) & ~15);
    return (a.idesc & ~(0x3Fu << 17)) | ((n >> 3) << 17);
}

// Bytes per chunk of a region with g valid 8-row groups (0: a region not copied).
__device__ __forceinline__ uint32_t chunk_bytes(uint32_t g) { return g == 16 ? 4096u : g * 256u; }

// n consecutive 4 KiB chunks of one M tile into a stage region: one copy when whole, the
// valid groups of each chunk when partial, nothing when g = 0.
__device__ __forceinline__ void vp_copy_region(uint8_t* dst, const uint8_t* src, uint32_t g, int n,
                                               unsigned long long* bar) {
    if (g == 16) bulk_load(dst, src, static_cast<uint32_t>(n) * 4096u, bar);
    else
        for (int j = 0; j < n && g != 0; ++j) bulk_load(dst + j * 4096, src + j * 4096, g * 256u, bar);
}

template <bool kGrouped>
__device__ void vp_producer(const FxArgs& a, uint8_t* smem, FxCtl* ctl) {
    uint32_t g = 0;
    int u_next = atomicAdd(a.next_item, 1);
    for (uint32_t gi = 0;; ++gi) {
        bool ok = true;
        const int it = take_unit(a, ctl, gi, u_next, ok);
        if (!ok) goto abort;
        if (it < 0) break;
        {
            const WorkItem w = a.items[it];
            const bool pair = vp_second(a, it) >= 0;
            const BlockInfo bi = a.blocks[w.blk];
            const int nch = stages_of(bi.k, kStageK);
            const bool diag = w.ti == w.tj;
            const uint8_t* mt = a.mplanes;
            int64_t n_ck = a.n_ck;
            if constexpr (kGrouped) {
                mt = a.groups[bi.grp].mplanes;
                n_ck = a.groups[bi.grp].n_ck;
            }
            // Per chunk: the valid 8-row groups of a partial side (feed_groups), else 4 KiB.
            const int P = kGrouped ? a.groups[bi.grp].P : a.P;
            const uint32_t gA = diag ? 0u : feed_groups(a, min(kTile, P - w.ti * kTile));
            const uint32_t gB = feed_groups(a, min(kTile, P - w.tj * kTile));
            const uint32_t gF = pair ? feed_groups(a, min(kTile, P - (w.tj + 1) * kTile)) : 0u;
            for (int c0 = 0; c0 < nch; c0 += kVpChunks, ++g) {
                const int n = min(kVpChunks, nch - c0);
                const int slot = static_cast<int>(g % kVpStages);
                if (!waitb(&ctl->empty[slot], ((g / kVpStages) & 1u) ^ 1u, ctl, a)) goto abort;
                uint8_t* sa = smem + slot * kVpStageBytes;
                unsigned long long* bar = &ctl->full[slot];
                mbar_expect_tx(bar, static_cast<uint32_t>(n) * (chunk_bytes(gA) + chunk_bytes(gB) + chunk_bytes(gF)));
                const int64_t chunk = bi.col / kStageK + c0;
                const uint8_t* si = mt + (static_cast<int64_t>(w.ti) * n_ck + chunk) * kTile8Bytes;
                const uint8_t* sj = mt + (static_cast<int64_t>(w.tj) * n_ck + chunk) * kTile8Bytes;
                vp_copy_region(sa, si, gA, n, bar);
                vp_copy_region(sa + kVpASide, sj, gB, n, bar);
                vp_copy_region(sa + 2 * kVpASide, sj + n_ck * kTile8Bytes, gF, n, bar);
            }
        }
    }
    return;
abort:
    for (uint32_t k = (g >= kVpStages ? g - kVpStages : 0); k < g; ++k)
        waitb(&ctl->full[k % kVpStages], (k / kVpStages) & 1u, ctl, a, false);
}

template <bool kGrouped>
__device__ void vp_issuer(const FxArgs& a, uint8_t* smem, FxCtl* ctl, uint32_t tmem) {
    uint32_t g = 0, n_acc = 0;
    for (uint32_t gi = 0;; ++gi) {
        const int it = read_item(a, ctl, gi);
        if (it < 0) break;
        const WorkItem w = a.items[it];
        const BlockInfo bi = a.blocks[w.blk];
        const int nch = stages_of(bi.k, kStageK);
        if (nch == 0) continue;
        const bool pair = vp_second(a, it) >= 0;
        const uint32_t id = vp_idesc<kGrouped>(a, bi, w.tj);
        const uint32_t idf = pair ? vp_idesc<kGrouped>(a, bi, w.tj + 1) : 0u;
        const bool diag = w.ti == w.tj;
        // One accumulator per part of at most kVpPartChunks chunks (the int32 bound).
        for (int p0 = 0; p0 < nch; p0 += kVpPartChunks) {
            const int p1 = min(nch, p0 + kVpPartChunks);
            const int b = static_cast<int>(n_acc % kVpAcc);
            if (!waitb(&ctl->acc_empty[b], ((n_acc / kVpAcc) & 1u) ^ 1u, ctl, a)) goto done;
            tc_fence_after();
            const uint32_t d = tmem + static_cast<uint32_t>(b) * kVpAccCols;
            for (int c0 = p0; c0 < p1; c0 += kVpChunks, ++g) {
                const int slot = static_cast<int>(g % kVpStages);
                if (!waitb(&ctl->full[slot], (g / kVpStages) & 1u, ctl, a)) goto done;
                tc_fence_after();
                const uint32_t sa = smem_u32(smem + slot * kVpStageBytes);
                const uint32_t sb = sa + kVpASide;
                const int n = min(kVpChunks, nch - c0);
                for (int j = 0; j < n; ++j) {
                    const uint32_t bj = sb + static_cast<uint32_t>(j) * 4096u;
                    const uint64_t dA = smem_desc(diag ? bj : sa + static_cast<uint32_t>(j) * 4096u, 256, 6);
                    const uint32_t f = (c0 + j) > p0 ? 1u : 0u;
                    if (pair) {
                        mma_i8_c<CollectorA::kFill>(d, dA, smem_desc(bj, 256, 6), id, f);
                        mma_i8_c<CollectorA::kLastUse>(d + kTile, dA, smem_desc(bj + kVpASide, 256, 6), idf, f);
                    } else {
                        mma_i8(d, dA, smem_desc(bj, 256, 6), id, f);
                    }
                }
                mma_commit(&ctl->empty[slot]);
            }
            mma_commit(&ctl->acc_full[b]);
            ++n_acc;
        }
    }
done:
    mma_commit(&ctl->drain);
    waitb(&ctl->drain, 0u, ctl, a, false);
}

// Warp (quarter q, half h): TMEM lanes 32q.., columns 128h.. of the accumulator, i.e. the
// unit's item h (a single unit's h = 1 warps only take part in the barriers).
__device__ void vp_epilogue(const FxArgs& a, FxCtl* ctl, uint32_t tmem, int warp, int lane) {
    const int q = warp & 3;
    const int h = (warp - 2) >> 2;
    const uint32_t lane_addr = static_cast<uint32_t>(q * 32) << 16;
    uint32_t n_acc = 0;
    for (uint32_t gi = 0;; ++gi) {
        int it = 0;
        if (lane == 0) it = read_item(a, ctl, gi);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it < 0) return;
        const int nch = stages_of(a.blocks[a.items[it].blk].k, kStageK);
        if (nch == 0) continue;  // the f2 kernel writes zeros
        const int mine = h == 0 ? it : vp_second(a, it);
        int32_t* dst = a.vpc + static_cast<int64_t>(mine) * kVpTileInts + q * 32 + lane;
        for (int p0 = 0; p0 < nch; p0 += kVpPartChunks) {
            const int b = static_cast<int>(n_acc % kVpAcc);
            bool ok = true;
            if (lane == 0) ok = waitb(&ctl->acc_full[b], (n_acc / kVpAcc) & 1u, ctl, a);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) return;
            tc_fence_after();
            if (mine >= 0) {
#pragma unroll 1
                for (int c32 = 0; c32 < kTile / 32; ++c32) {
                    uint32_t v[32];
                    tmem_ld32(tmem + lane_addr + static_cast<uint32_t>(b) * kVpAccCols +
                                  static_cast<uint32_t>(h * kTile + c32 * 32),
                              v);
                    tmem_wait_ld();
                    // M = 64 on both sides: each both-present SNP adds 4096.
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        const int32_t cnt = static_cast<int32_t>(v[c]) >> 12;
                        int32_t* o = dst + (c32 * 32 + c) * kTile;
                        *o = p0 == 0 ? cnt : *o + cnt;
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl->acc_empty[b]);
            ++n_acc;
        }
    }
}

template <bool kGrouped>
__global__ void __launch_bounds__(kVpThreads, 1) vpair_fx_kernel(const __grid_constant__ FxArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    FxCtl* ctl = reinterpret_cast<FxCtl*>(smem + kVpStages * kVpStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        init_ring(ctl, 1 + kVpEpiWarps);
        for (int s = 0; s < kVpStages; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        for (int b = 0; b < kVpAcc; ++b) {
            mbar_init(&ctl->acc_full[b], 1);
            mbar_init(&ctl->acc_empty[b], kVpEpiWarps);
        }
        mbar_init(&ctl->drain, 1);
        ctl->abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(&ctl->tmem_base, kTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;
    if (warp < 2) {
        if (warp == 0 && lane == 0) vp_producer<kGrouped>(a, smem, ctl);
        if (warp == 1 && lane == 0) vp_issuer<kGrouped>(a, smem, ctl, tmem);
    } else {
        vp_epilogue(a, ctl, tmem, warp, lane);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, kTmemCols);
}

constexpr size_t kVpSmemBytes = kVpStages * kVpStageBytes + kCtlBytes + 1024;

// kind::i8 instruction descriptor: D = s32, A = B = s8, K-major A and B, N >> 3 at bit
// 17, M >> 4 at bit 24.
uint32_t idesc_s8_s32() { return (2u << 4) | (1u << 7) | (1u << 10) | ((kTile >> 3) << 17) | ((kTile >> 4) << 24); }

void set_fx_smem() {
    const int b = static_cast<int>(kFxSmemBytes), v = static_cast<int>(kVpSmemBytes);
    STPF2_CUDA(cudaFuncSetAttribute(f2_fx_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    STPF2_CUDA(cudaFuncSetAttribute(f2_fx_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    STPF2_CUDA(cudaFuncSetAttribute(vpair_fx_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, v));
    STPF2_CUDA(cudaFuncSetAttribute(vpair_fx_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, v));
}

}  // namespace

size_t fx_vpc_bytes(int n_items) { return static_cast<size_t>(std::max(n_items, 1)) * kVpTileInts * sizeof(int32_t); }

void fx_prepare() { set_fx_smem(); }

void launch_fx(Ctx& c, const FxLaunch& L, cudaStream_t s) {
    if (L.n_items <= 0) return;
    FxArgs a{};
    a.images = L.images;
    a.mplanes = L.mplanes;
    a.n_ck = L.n_ck;
    a.items = L.items;
    a.n_items = L.n_items;
    a.units = L.units;
    a.n_units = L.n_units;
    a.unit_base = L.unit_base;
    a.blocks = L.blocks;
    a.P = L.P;
    a.f2 = L.f2;
    a.vpair = L.vpair;
    a.vpc = L.vpc;
    a.rcp = L.rcp;
    a.rcp_max = L.rcp_max;
    a.err = L.err;
    a.b_base = L.b_base;
    a.idesc = idesc_s8_s32();
    a.timeout_ns = c.fx_tuning.timeout_ns;
    a.withhold = -1;
    a.partial_feed = c.fx_tuning.partial_feed;
    a.groups = L.groups;
    a.grp_done = L.grp_done;
    a.grp_ns = L.grp_ns;
    a.grp_items = L.grp_items;
    if (!L.units || L.n_units <= 0) fail(STP_RUNTIME_ERROR, "fixed-point contraction without vpair units");
    const int grid = std::min(c.sm_count, L.n_items);
    // Two work counters: vpair units, then f2 items.
    STPF2_CUDA(cudaMemsetAsync(L.counters, 0, 2 * sizeof(int), s));
    a.next_item = L.counters;
    const int vp_grid = std::min(c.sm_count, L.n_units);
    if (L.groups) vpair_fx_kernel<true><<<vp_grid, kVpThreads, kVpSmemBytes, s>>>(a);
    else vpair_fx_kernel<false><<<vp_grid, kVpThreads, kVpSmemBytes, s>>>(a);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
    a.next_item = L.counters + 1;
    a.withhold = c.fx_tuning.withhold_stage;  // test hook: starves the f2 kernel's issuer
    if (L.groups) f2_fx_kernel<true><<<grid, kThreads, kFxSmemBytes, s>>>(a);
    else f2_fx_kernel<false><<<grid, kThreads, kFxSmemBytes, s>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFuncAttributes fa{};
        cudaFuncGetAttributes(&fa, f2_fx_kernel<false>);
        fail(STP_CUDA_ERROR, std::string("f2_fx_kernel launch: ") + cudaGetErrorString(e) + " (regs " +
                                 std::to_string(fa.numRegs) + ", dyn smem " + std::to_string(kFxSmemBytes) + ", local " +
                                 std::to_string(fa.localSizeBytes) + ")");
    }
    c.launches++;
}

}  // namespace stpf2
