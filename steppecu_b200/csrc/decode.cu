// steppecu_b200/csrc/decode.cu
//
// Genotype decode for the f2 path (sm_100a). The hot kernel, decode_pa_kernel, reads
// SNP-major PACKEDANCESTRYMAP records straight from HBM (coalesced 128-bit loads into a
// shared-memory tile of 32 records), folds every selected sample of every population into
// exact integer counts (ac2 = 2*ac, n) following decode_af.hpp:58-65, and writes the
// contraction operands for those counts directly into the block-padded planes the
// contraction kernels read. Also here: per-sample ploidy detection (detect_ploidy_kernel.cu
// :32-57), the canonical-tile decode behind ComputeBackend::decode_af (cpu_backend.cpp
// :267-319) and the Q/V/N feeder behind compute_f2_blocks(MatView...) (f2_block_kernel.cu
// :37-61 computes the same per-element terms).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "stpf2_internal.cuh"

namespace stpf2 {

namespace {

constexpr int kDecSnps = 32;       // SNP records per CTA (one per lane)
constexpr int kDecThreads = 256;   // 8 warps share the CTA's populations
constexpr int kPloidyWindow = 1000;  // decode_af.hpp:29 (kPloidyDetectSnps)

// Per-element operand terms of one (pop, SNP) from its exact counts. q matches the
// reference bit for bit: ac = ac2/2 is exact, q = ac/n (decode_af.hpp:87-97); h is
// het_correction (f2_estimator.hpp:22-27).
struct Terms {
    double pt, ah, m;
};

__device__ __forceinline__ Terms make_terms(double q, double nd, bool valid, double center) {
    Terms t{0.0, 0.0, 0.0};
    if (valid) {
        const double nm1 = nd - 1.0;
        const double denom = (nm1 > 1.0) ? nm1 : 1.0;
        const double h = q * (1.0 - q) / denom;
        const double pt = q - center;
        t.pt = pt;
        t.ah = 0.5 * (pt * pt - h);
        t.m = 1.0;
    }
    return t;
}

template <class T> __device__ __forceinline__ T to16(double x);
template <> __device__ __forceinline__ __nv_bfloat16 to16<__nv_bfloat16>(double x) {
    return __double2bfloat16(x);
}
template <> __device__ __forceinline__ __half to16<__half>(double x) { return __double2half(x); }
template <class T> __device__ __forceinline__ double from16(T x);
template <> __device__ __forceinline__ double from16<__nv_bfloat16>(__nv_bfloat16 x) {
    return static_cast<double>(__bfloat162float(x));
}
template <> __device__ __forceinline__ double from16<__half>(__half x) {
    return static_cast<double>(__half2float(x));
}

// Writes one element of every operand plane. hi = round(x), lo = round(x - hi): the pair
// carries ~2x the mantissa of one 16-bit value; the F16 planes are pre-scaled into
// half's normal range (Pt by 2^7, Ah by 2^14, so every product carries 2^14).
template <OpFmt F>
__device__ __forceinline__ void emit(const OperandPlanes& op, int i, int64_t col, const Terms& t) {
    const int64_t row = static_cast<int64_t>(i) * op.ld + col;
    const int64_t plane = static_cast<int64_t>(op.P) * op.ld;
    if constexpr (F == OpFmt::F32) {
        float* p = static_cast<float*>(op.planes);
        p[row] = static_cast<float>(t.pt);
        p[plane + row] = static_cast<float>(t.ah);
    } else {
        using T = typename std::conditional<F == OpFmt::BF16, __nv_bfloat16, __half>::type;
        const double sp = (F == OpFmt::F16) ? double(1 << kF16PtShift) : 1.0;
        const double sa = sp * sp;
        const double pt = t.pt * sp, ah = t.ah * sa;
        const T pth = to16<T>(pt);
        const T ptl = to16<T>(pt - from16<T>(pth));
        const T ahh = to16<T>(ah);
        const T ahl = to16<T>(ah - from16<T>(ahh));
        T* p = static_cast<T*>(op.planes);
        p[row] = pth;
        p[plane + row] = ptl;
        p[2 * plane + row] = ahh;
        p[3 * plane + row] = ahl;
        p[4 * plane + row] = to16<T>(t.m);
    }
    op.m_u8[row] = static_cast<uint8_t>(t.m != 0.0);
}

// Folds one packed sample descriptor (see pack_sel) against a record byte array.
__device__ __forceinline__ void fold_sel(const uint8_t* rec, uint32_t e, int& a, int& c) {
    const uint32_t byte = rec[e >> 5];
    const int code = static_cast<int>((byte >> ((e >> 2) & 7u)) & 3u);
    const int pl = static_cast<int>(e & 3u);
    // decode_af.hpp:58-65: a valid code adds code/(3-ploidy) to ac and ploidy to n;
    // carried doubled: diploid adds 2*code, pseudo-haploid adds code.
    const bool valid = (code != 3) && (pl == 1 || pl == 2);
    a += valid ? (code << (pl - 1)) : 0;
    c += valid ? pl : 0;
}

template <OpFmt F>
__global__ void __launch_bounds__(kDecThreads)
decode_pa_kernel(PaDecodeArgs a, uint32_t stride_words, int vec16) {
    extern __shared__ __align__(16) uint32_t s_rec[];
    __shared__ double s_center[kDecSnps];

    const int64_t s0 = static_cast<int64_t>(blockIdx.x) * kDecSnps;
    const int64_t rem = a.n_snp - s0;
    const int nrows = rem < kDecSnps ? static_cast<int>(rem) : kDecSnps;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = kDecThreads / 32;

    // 1. Stage this CTA's records: 128-bit loads, coalesced along each record. The
    //    shared row stride is an odd number of words so lanes that read the same byte
    //    column of 32 different records hit 32 different banks.
    if (vec16) {
        const uint32_t cpr = static_cast<uint32_t>(a.pitch / 16);
        const uint32_t total = static_cast<uint32_t>(nrows) * cpr;
        for (uint32_t c = threadIdx.x; c < total; c += kDecThreads) {
            const uint32_t r = c / cpr, k = c - r * cpr;
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(a.records + (s0 + r) * a.pitch) + k);
            uint32_t* d = s_rec + r * stride_words + k * 4;
            d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
        }
    } else {
        uint8_t* sb = reinterpret_cast<uint8_t*>(s_rec);
        const uint32_t bpr = static_cast<uint32_t>(a.pitch);
        const uint32_t total = static_cast<uint32_t>(nrows) * bpr;
        for (uint32_t c = threadIdx.x; c < total; c += kDecThreads) {
            const uint32_t r = c / bpr, k = c - r * bpr;
            sb[r * stride_words * 4 + k] = a.records[(s0 + r) * a.pitch + k];
        }
    }
    __syncthreads();

    const uint8_t* my_rec = reinterpret_cast<const uint8_t*>(s_rec) + lane * stride_words * 4;

    // 2. Per-SNP centre c_s: pooled frequency of a fixed, evenly spread subset of the
    //    selected samples, rounded to 1/256 (exact in every operand type). f2 is
    //    invariant to a per-SNP shift of all frequencies, so c_s only shrinks magnitudes.
    if (warp == 0) {
        int ca = 0, cc = 0;
        if (lane < nrows)
            for (int g = 0; g < a.n_center; ++g) fold_sel(my_rec, __ldg(a.sel + __ldg(a.center_idx + g)), ca, cc);
        s_center[lane] = (cc > 0) ? rint((0.5 * ca / cc) * 256.0) / 256.0 : 0.5;
    }
    __syncthreads();

    const int64_t s = s0 + lane;
    const bool live = lane < nrows;
    const int64_t col = live ? static_cast<int64_t>(__ldg(a.snp_col + s)) : 0;
    const double center = s_center[lane];

    // 3. Populations round-robin over warps; lane = SNP. Exact integer fold.
    for (int i = warp; i < a.P; i += nwarps) {
        const int g0 = __ldg(a.pop_off + i), g1 = __ldg(a.pop_off + i + 1);
        int ac = 0, cn = 0, ac2 = 0, cn2 = 0;
        int g = g0;
        for (; g + 1 < g1; g += 2) {
            fold_sel(my_rec, __ldg(a.sel + g), ac, cn);
            fold_sel(my_rec, __ldg(a.sel + g + 1), ac2, cn2);
        }
        if (g < g1) fold_sel(my_rec, __ldg(a.sel + g), ac, cn);
        ac += ac2;
        cn += cn2;
        if (live) {
            const double nd = static_cast<double>(cn);
            const double q = (cn > 0) ? (static_cast<double>(ac) * 0.5) / nd : 0.0;
            emit<F>(a.op, i, col, make_terms(q, nd, cn > 0, center));
            if (a.cnt_ac2) {
                a.cnt_ac2[static_cast<int64_t>(i) + static_cast<int64_t>(a.P) * s] = ac;
                a.cnt_n[static_cast<int64_t>(i) + static_cast<int64_t>(a.P) * s] = cn;
            }
        }
    }
}

// detect_ploidy_kernel.cu:32-57 on SNP-major records: sample g is diploid iff a het
// (code 1) occurs in the first min(1000, n_snp) SNPs. Writes the ploidy into the sample
// descriptor's low bits.
__global__ void detect_ploidy_pa_kernel(const uint8_t* __restrict__ records, uint64_t pitch,
                                        int64_t window, uint32_t* sel, int64_t n_sel) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n_sel) return;
    const uint32_t e = sel[g];
    const uint32_t byte = e >> 5, shift = (e >> 2) & 7u;
    int pl = 1;
    for (int64_t s = 0; s < window; ++s) {
        if (((records[s * pitch + byte] >> shift) & 3u) == 1u) {
            pl = 2;
            break;
        }
    }
    sel[g] = (e & ~3u) | static_cast<uint32_t>(pl);
}

// cpu_backend.cpp:73-95 on the canonical individual-major tile.
__global__ void detect_ploidy_canonical_kernel(const uint8_t* __restrict__ packed, uint64_t bpr,
                                               int64_t window, int64_t n_ind, int32_t* ploidy) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n_ind) return;
    const uint8_t* rec = packed + g * bpr;
    int pl = 1;
    for (int64_t s = 0; s < window; ++s) {
        if (((rec[s >> 2] >> (6 - 2 * (s & 3))) & 3) == 1) {
            pl = 2;
            break;
        }
    }
    ploidy[g] = pl;
}

// cpu_backend.cpp:267-319: q/v/n FP64 per (pop, SNP) from the canonical tile.
__global__ void decode_canonical_kernel(const uint8_t* __restrict__ packed, uint64_t bpr,
                                        int64_t n_snp, const int32_t* __restrict__ pop_off, int P,
                                        const int32_t* __restrict__ ploidy, double* q, double* v,
                                        double* n) {
    const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (s >= n_snp || i >= P) return;
    int ac2 = 0, cn = 0;
    const int shift = 6 - 2 * static_cast<int>(s & 3);
    for (int g = pop_off[i]; g < pop_off[i + 1]; ++g) {
        const int code = (packed[static_cast<int64_t>(g) * bpr + (s >> 2)] >> shift) & 3;
        const int pl = ploidy[g];
        const bool valid = code != 3 && (pl == 1 || pl == 2);
        ac2 += valid ? (code << (pl - 1)) : 0;
        cn += valid ? pl : 0;
    }
    const int64_t off = static_cast<int64_t>(i) + static_cast<int64_t>(P) * s;
    if (cn > 0) {
        const double nd = static_cast<double>(cn);
        n[off] = nd;
        q[off] = (static_cast<double>(ac2) * 0.5) / nd;
        v[off] = 1.0;
    } else {
        n[off] = 0.0;
        q[off] = 0.0;
        v[off] = 0.0;
    }
}

// Per-SNP centre for the Q/V/N feeder: mean of the valid frequencies, rounded to 1/256.
__global__ void qvn_center_kernel(const double* __restrict__ Q, const double* __restrict__ V,
                                  int P, int64_t M, double* center) {
    const int64_t s = static_cast<int64_t>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= M) return;
    double sq = 0.0, sv = 0.0;
    for (int i = lane; i < P; i += 32) {
        const int64_t o = static_cast<int64_t>(i) + static_cast<int64_t>(P) * s;
        if (V[o] != 0.0) {
            sq += Q[o];
            sv += 1.0;
        }
    }
    for (int d = 16; d > 0; d >>= 1) {
        sq += __shfl_xor_sync(0xffffffffu, sq, d);
        sv += __shfl_xor_sync(0xffffffffu, sv, d);
    }
    if (lane == 0) center[s] = (sv > 0.0) ? rint((sq / sv) * 256.0) / 256.0 : 0.5;
}

// Q/V/N -> operand planes (the per-element work of f2_feeder_kernel, f2_block_kernel.cu
// :37-61, in this build's centred split form).
template <OpFmt F>
__global__ void feed_qvn_kernel(const double* __restrict__ Q, const double* __restrict__ V,
                                const double* __restrict__ N, int P, int64_t M,
                                const int32_t* __restrict__ snp_col,
                                const double* __restrict__ center, OperandPlanes op) {
    const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (s >= M || i >= P) return;
    const int64_t o = static_cast<int64_t>(i) + static_cast<int64_t>(P) * s;
    emit<F>(op, i, snp_col[s], make_terms(Q[o], N[o], V[o] != 0.0, center[s]));
}

}  // namespace

void launch_detect_ploidy_pa(Ctx& c, const uint8_t* records, uint64_t pitch, int64_t n_snp,
                             uint32_t* sel, int64_t n_sel, cudaStream_t s) {
    if (n_sel <= 0) return;
    const int64_t window = n_snp < kPloidyWindow ? n_snp : kPloidyWindow;
    const int threads = 128;
    detect_ploidy_pa_kernel<<<static_cast<unsigned>((n_sel + threads - 1) / threads), threads, 0, s>>>(
        records, pitch, window, sel, n_sel);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

static int center_count(int64_t n_sel) { return static_cast<int>(n_sel < 256 ? n_sel : 256); }

void launch_decode_pa(Ctx& c, const PaDecodeArgs& a, cudaStream_t s) {
    if (a.n_snp <= 0 || a.P <= 0) return;
    // Word stride of one staged record, forced odd (bank-conflict-free column reads).
    uint32_t words = static_cast<uint32_t>((a.pitch + 3) / 4);
    if ((words & 1u) == 0) words += 1;
    const size_t smem = static_cast<size_t>(kDecSnps) * words * 4;
    if (smem > 200 * 1024)
        fail(STP_INVALID_ARGUMENT, "decode: genotype record of " + std::to_string(a.pitch) +
                                       " bytes exceeds the 32-record shared-memory tile");
    const int vec16 = (a.pitch % 16 == 0) && (reinterpret_cast<uintptr_t>(a.records) % 16 == 0);
    const unsigned grid = static_cast<unsigned>((a.n_snp + kDecSnps - 1) / kDecSnps);
    switch (a.op.fmt) {
        case OpFmt::F32:
            STPF2_CUDA(cudaFuncSetAttribute(decode_pa_kernel<OpFmt::F32>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            decode_pa_kernel<OpFmt::F32><<<grid, kDecThreads, smem, s>>>(a, words, vec16);
            break;
        case OpFmt::BF16:
            STPF2_CUDA(cudaFuncSetAttribute(decode_pa_kernel<OpFmt::BF16>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            decode_pa_kernel<OpFmt::BF16><<<grid, kDecThreads, smem, s>>>(a, words, vec16);
            break;
        case OpFmt::F16:
            STPF2_CUDA(cudaFuncSetAttribute(decode_pa_kernel<OpFmt::F16>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            decode_pa_kernel<OpFmt::F16><<<grid, kDecThreads, smem, s>>>(a, words, vec16);
            break;
    }
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_detect_ploidy_canonical(Ctx& c, const uint8_t* packed, uint64_t bpr, int64_t n_snp,
                                    int64_t n_ind, int32_t* ploidy, cudaStream_t s) {
    if (n_ind <= 0) return;
    const int64_t window = n_snp < kPloidyWindow ? n_snp : kPloidyWindow;
    detect_ploidy_canonical_kernel<<<static_cast<unsigned>((n_ind + 127) / 128), 128, 0, s>>>(
        packed, bpr, window, n_ind, ploidy);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_decode_canonical(Ctx& c, const uint8_t* packed, uint64_t bpr, int64_t n_snp,
                             int64_t /*n_ind*/, const int32_t* pop_off, int P, const int32_t* ploidy,
                             double* q, double* v, double* n, cudaStream_t s) {
    if (n_snp <= 0 || P <= 0) return;
    const dim3 block(32, 8);
    const dim3 grid(static_cast<unsigned>((n_snp + 31) / 32), static_cast<unsigned>((P + 7) / 8));
    decode_canonical_kernel<<<grid, block, 0, s>>>(packed, bpr, n_snp, pop_off, P, ploidy, q, v, n);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_feed_qvn(Ctx& c, const double* Q, const double* V, const double* N, int P, int64_t M,
                     const int32_t* snp_col, const OperandPlanes& op, cudaStream_t s) {
    if (P <= 0 || M <= 0) return;
    double* center = nullptr;
    STPF2_CUDA(cudaMallocAsync(&center, static_cast<size_t>(M) * sizeof(double), s));
    qvn_center_kernel<<<static_cast<unsigned>((M + 7) / 8), 256, 0, s>>>(Q, V, P, M, center);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
    const dim3 block(32, 8);
    const dim3 grid(static_cast<unsigned>((M + 31) / 32), static_cast<unsigned>((P + 7) / 8));
    switch (op.fmt) {
        case OpFmt::F32: feed_qvn_kernel<OpFmt::F32><<<grid, block, 0, s>>>(Q, V, N, P, M, snp_col, center, op); break;
        case OpFmt::BF16: feed_qvn_kernel<OpFmt::BF16><<<grid, block, 0, s>>>(Q, V, N, P, M, snp_col, center, op); break;
        case OpFmt::F16: feed_qvn_kernel<OpFmt::F16><<<grid, block, 0, s>>>(Q, V, N, P, M, snp_col, center, op); break;
    }
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
    STPF2_CUDA(cudaFreeAsync(center, s));
}

int decode_center_count(int64_t n_sel) { return center_count(n_sel); }

}  // namespace stpf2
