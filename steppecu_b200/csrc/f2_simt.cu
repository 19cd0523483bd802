// steppecu_b200/csrc/f2_simt.cu
//
// The plain FP32 SIMT contraction (no tensor cores): the comparison form of the f2
// extraction. For every (block, 64x64 tile pair ti <= tj) one CTA accumulates, over the
// block's SNP columns,
//     acc(i,j)   = sum_s (Ah_i M_j + M_i Ah_j - Pt_i Pt_j)     (FP32, drained to FP64 every
//                                                              16 SNPs)
//     vpair(i,j) = sum_s M_i M_j                                (exact: integers < 2^24)
// and writes f2 = 2*acc/vpair (0 when vpair = 0) and vpair into both (i,j) and (j,i) of
// the block's slab: the per-block work of compute_f2_blocks (cpu_backend.cpp:217-264;
// f2_estimator.hpp:38-46 for the numerator and the divide).
#include "stpf2_internal.cuh"

namespace stpf2 {

namespace {

constexpr int kT = 64;        // tile edge (populations)
constexpr int kKc = 16;       // SNP columns per shared-memory chunk
constexpr int kThreads = 256; // 16 x 16 threads, 4 x 4 outputs each
constexpr int kPad = 4;

struct SimtOps {
    const float* pt;
    const float* ah;
    const uint8_t* m;
    int64_t ld;
    int P;
};

__global__ void __launch_bounds__(kThreads)
f2_simt_kernel(const WorkItem* __restrict__ items, const BlockInfo* __restrict__ blocks,
               SimtOps op, double* __restrict__ f2, double* __restrict__ vpair) {
    __shared__ __align__(16) float sP[2][kKc][kT + kPad];
    __shared__ __align__(16) float sA[2][kKc][kT + kPad];
    __shared__ __align__(16) float sM[2][kKc][kT + kPad];

    const WorkItem it = items[blockIdx.x];
    const BlockInfo bi = blocks[it.blk];
    const int P = op.P;
    const int row0[2] = {it.ti * kT, it.tj * kT};
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;

    double dacc[4][4];
    float vp[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            dacc[r][c] = 0.0;
            vp[r][c] = 0.0f;
        }

    const int kpad = (bi.k + kKc - 1) / kKc * kKc;
    for (int k0 = 0; k0 < kpad; k0 += kKc) {
        // Stage Pt/Ah (float4 loads along SNPs) and M (16 bytes per load) for both sides.
        for (int side = 0; side < 2; ++side) {
            for (int c = threadIdx.x; c < kT * kKc / 4; c += kThreads) {
                const int r = c / (kKc / 4), k4 = c % (kKc / 4);
                const int row = row0[side] + r;
                float4 p = make_float4(0.f, 0.f, 0.f, 0.f), a = p;
                if (row < P) {
                    const int64_t o = static_cast<int64_t>(row) * op.ld + bi.col + k0 + k4 * 4;
                    p = __ldg(reinterpret_cast<const float4*>(op.pt + o));
                    a = __ldg(reinterpret_cast<const float4*>(op.ah + o));
                }
                sP[side][k4 * 4 + 0][r] = p.x; sP[side][k4 * 4 + 1][r] = p.y;
                sP[side][k4 * 4 + 2][r] = p.z; sP[side][k4 * 4 + 3][r] = p.w;
                sA[side][k4 * 4 + 0][r] = a.x; sA[side][k4 * 4 + 1][r] = a.y;
                sA[side][k4 * 4 + 2][r] = a.z; sA[side][k4 * 4 + 3][r] = a.w;
            }
            for (int c = threadIdx.x; c < kT * kKc / 16; c += kThreads) {
                const int r = c / (kKc / 16), k16 = c % (kKc / 16);
                const int row = row0[side] + r;
                uint4 mv = make_uint4(0u, 0u, 0u, 0u);
                if (row < P)
                    mv = __ldg(reinterpret_cast<const uint4*>(op.m + static_cast<int64_t>(row) * op.ld +
                                                             bi.col + k0 + k16 * 16));
                const uint32_t w[4] = {mv.x, mv.y, mv.z, mv.w};
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    sM[side][k16 * 16 + q][r] = static_cast<float>((w[q >> 2] >> ((q & 3) * 8)) & 0xffu);
            }
        }
        __syncthreads();

        float acc[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[r][c] = 0.0f;

#pragma unroll 4
        for (int k = 0; k < kKc; ++k) {
            const float4 ap = *reinterpret_cast<const float4*>(&sP[0][k][ty * 4]);
            const float4 aa = *reinterpret_cast<const float4*>(&sA[0][k][ty * 4]);
            const float4 am = *reinterpret_cast<const float4*>(&sM[0][k][ty * 4]);
            const float4 bp = *reinterpret_cast<const float4*>(&sP[1][k][tx * 4]);
            const float4 ba = *reinterpret_cast<const float4*>(&sA[1][k][tx * 4]);
            const float4 bm = *reinterpret_cast<const float4*>(&sM[1][k][tx * 4]);
            const float AP[4] = {ap.x, ap.y, ap.z, ap.w}, AA[4] = {aa.x, aa.y, aa.z, aa.w};
            const float AM[4] = {am.x, am.y, am.z, am.w}, BP[4] = {bp.x, bp.y, bp.z, bp.w};
            const float BA[4] = {ba.x, ba.y, ba.z, ba.w}, BM[4] = {bm.x, bm.y, bm.z, bm.w};
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    acc[r][c] = fmaf(AA[r], BM[c], acc[r][c]);
                    acc[r][c] = fmaf(AM[r], BA[c], acc[r][c]);
                    acc[r][c] = fmaf(-AP[r], BP[c], acc[r][c]);
                    vp[r][c] = fmaf(AM[r], BM[c], vp[r][c]);
                }
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) dacc[r][c] += static_cast<double>(acc[r][c]);
        __syncthreads();
    }

    // Epilogue: finalize_f2 (f2_estimator.hpp:42-46) into both triangles of slab b.
    const int64_t slab = static_cast<int64_t>(P) * P * bi.b;
    const bool diag = it.ti == it.tj;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i = row0[0] + ty * 4 + r;
        if (i >= P) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int j = row0[1] + tx * 4 + c;
            if (j >= P) continue;
            if (diag && i > j) continue;
            const double v = static_cast<double>(vp[r][c]);
            const double val = (v > 0.0) ? (2.0 * dacc[r][c]) / v : 0.0;
            const int64_t ij = slab + i + static_cast<int64_t>(P) * j;
            const int64_t ji = slab + j + static_cast<int64_t>(P) * i;
            f2[ij] = val;
            vpair[ij] = v;
            f2[ji] = val;
            vpair[ji] = v;
        }
    }
}

}  // namespace

void launch_f2_simt(Ctx& c, const WorkItem* items, int n_items, const BlockInfo* blocks,
                    const OperandPlanes& op, double* f2, double* vpair, cudaStream_t s) {
    if (n_items <= 0) return;
    if (op.fmt != OpFmt::F32) fail(STP_INVALID_ARGUMENT, "f2_simt: needs FP32 operand planes");
    SimtOps o;
    o.pt = static_cast<const float*>(op.planes);
    o.ah = o.pt + static_cast<int64_t>(op.P) * op.ld;
    o.m = op.m_u8;
    o.ld = op.ld;
    o.P = op.P;
    f2_simt_kernel<<<static_cast<unsigned>(n_items), kThreads, 0, s>>>(items, blocks, o, f2, vpair);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

int simt_tile() { return kT; }

}  // namespace stpf2
