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

}  // namespace stpf2
