// steppecu_b200/csrc/jackknife.cu
//
// FP64 block jackknife over per-block values, one thread per item (pop pair): the
// block-size-weighted total, leave-one-out values, their weighted mean and the AT2
// jackknife variance of cpu_backend.cpp:2674-2720 (compute_loo_and_total) and
// :2273-2306 (jackknife_diag). The reference sums in long double; the device has no
// wider type, so every sum here is a compensated (two-sum) FP64 sum, whose error stays
// at the level of one FP64 rounding of the result.
#include "stpf2_internal.cuh"

namespace stpf2 {

namespace {

struct CSum {  // Neumaier compensated sum
    double s = 0.0, c = 0.0;
    __device__ void add(double x) {
        const double t = s + x;
        c += (fabs(s) >= fabs(x)) ? ((s - t) + x) : ((x - t) + s);
        s = t;
    }
    __device__ double value() const { return s + c; }
};

__global__ void jackknife_kernel(const double* __restrict__ x, const int32_t* __restrict__ bl,
                                 int64_t m, int nb, double n, double* est, double* var) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= m) return;
    CSum num;
    for (int b = 0; b < nb; ++b) num.add(x[k + m * b] * static_cast<double>(bl[b]));
    const double tot = num.value() / n;
    // Weighted mean of the leave-one-out values (weights 1 - bl/n).
    CSum wnum, wden, wbl;
    for (int b = 0; b < nb; ++b) {
        const double rel = static_cast<double>(bl[b]) / n;
        const double loo = (tot - x[k + m * b] * rel) / (1.0 - rel);
        const double w = 1.0 - rel;
        wnum.add(loo * w);
        wden.add(w);
        wbl.add(loo * static_cast<double>(bl[b]));
    }
    const double totline = wnum.value() / wden.value();
    CSum diff;
    for (int b = 0; b < nb; ++b) {
        const double rel = static_cast<double>(bl[b]) / n;
        const double loo = (tot - x[k + m * b] * rel) / (1.0 - rel);
        diff.add(totline - loo);
    }
    const double term1 = (diff.value() / nb) * nb;
    const double e = term1 + wbl.value() / n;
    CSum acc;
    for (int b = 0; b < nb; ++b) {
        const double bl_d = static_cast<double>(bl[b]);
        const double rel = bl_d / n;
        const double loo = (tot - x[k + m * b] * rel) / (1.0 - rel);
        const double h = n / bl_d;
        const double xtau = (e * h - loo * (h - 1.0) - totline) / sqrt(h - 1.0);
        acc.add(xtau * xtau);
    }
    est[k] = e;
    var[k] = acc.value() / nb;
}

// survivor_blocks (cpu_backend.cpp:124-151): one CTA per block; keep[b] = 0 when block b
// has a missing pair (vpair not > 0, f2_estimator.hpp:49-51) and a present one.
__global__ void survivor_kernel(const double* __restrict__ vpair, int64_t slab, int32_t* __restrict__ keep) {
    const int64_t b = blockIdx.x;
    const double* v = vpair + slab * b;
    int missing = 0, present = 0;
    // Four independent loads per thread in flight: the pass streams every slab once.
    for (int64_t e = threadIdx.x; e < slab; e += 4 * static_cast<int64_t>(blockDim.x)) {
        double x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t k = e + static_cast<int64_t>(u) * blockDim.x;
            x[u] = k < slab ? __ldg(v + k) : 0.0;  // not loaded, and not counted, past the slab
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t k = e + static_cast<int64_t>(u) * blockDim.x;
            if (k < slab) {
                const bool p = x[u] > 0.0;
                present |= p;
                missing |= !p;
            }
        }
    }
    missing = __syncthreads_or(missing);
    present = __syncthreads_or(present);
    if (threadIdx.x == 0) keep[b] = !(missing && present);
}

// assemble_f4_quartets / assemble_f3_triples / assemble_f4 (cpu_backend.cpp:2064-2216):
// x[k + m*bs] for statistic k over surviving block bs (block surv[bs]), each sum in the
// reference's operation order.
__global__ void fstat_assemble_kernel(const double* __restrict__ f2, int64_t P, const int32_t* __restrict__ surv,
                                      int ns, int kind, const int32_t* __restrict__ idx, int64_t n_stat,
                                      int64_t m, int64_t nr, double* __restrict__ x) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= m * ns) return;
    const int64_t k = t % m, bs = t / m;
    const double* f = f2 + P * P * surv[bs];
    auto at = [&](int i, int j) { return f[i + P * j]; };
    double v;
    if (kind == 0) {
        const int p1 = idx[4 * k], p2 = idx[4 * k + 1], p3 = idx[4 * k + 2], p4 = idx[4 * k + 3];
        v = 0.5 * (at(p2, p3) + at(p1, p4) - at(p1, p3) - at(p2, p4));
    } else if (kind == 1) {
        const int pc = idx[3 * k], pa = idx[3 * k + 1], pb = idx[3 * k + 2];
        v = 0.5 * (at(pc, pa) + at(pc, pb) - at(pa, pb));
    } else {
        const int64_t i = k / nr, j = k % nr;  // k = j + nr*i
        const int L0 = idx[0], R0 = idx[n_stat], Li = idx[1 + i], Rj = idx[n_stat + 1 + j];
        v = 0.5 * (at(Li, R0) + at(L0, Rj) - at(L0, R0) - at(Li, Rj));
    }
    x[t] = v;
}

}  // namespace

void launch_jackknife(Ctx& c, const double* x, const int32_t* block_sizes, int64_t m, int nb,
                      double* est, double* var, cudaStream_t s) {
    if (m <= 0 || nb <= 0) return;
    // n = sum of block sizes (exact in FP64 for any realistic SNP count).
    std::vector<int32_t> h(static_cast<size_t>(nb));
    STPF2_CUDA(cudaMemcpyAsync(h.data(), block_sizes, sizeof(int32_t) * nb, cudaMemcpyDeviceToHost, s));
    STPF2_CUDA(cudaStreamSynchronize(s));
    double n = 0.0;
    for (int32_t v : h) n += static_cast<double>(v);
    const int threads = 128;
    jackknife_kernel<<<static_cast<unsigned>((m + threads - 1) / threads), threads, 0, s>>>(
        x, block_sizes, m, nb, n, est, var);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_survivors(Ctx& c, const double* vpair, int P, int nb, int32_t* keep, cudaStream_t s) {
    if (nb <= 0) return;
    survivor_kernel<<<nb, 256, 0, s>>>(vpair, static_cast<int64_t>(P) * P, keep);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_fstat_assemble(Ctx& c, const double* f2, int P, const int32_t* surv, int ns, int kind,
                           const int32_t* idx, int64_t n_stat, int64_t m, int64_t nr, double* x, cudaStream_t s) {
    if (m <= 0 || ns <= 0) return;
    const int64_t n = m * ns;
    fstat_assemble_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(f2, P, surv, ns, kind, idx, n_stat, m, nr, x);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

}  // namespace stpf2
