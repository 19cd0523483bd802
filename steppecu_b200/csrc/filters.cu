// steppecu_b200/csrc/filters.cu
//
// extract-f2's per-SNP keep mask on the device (the regime-B decision of
// decode_compact_kernel.cu:39-68 in the reference): one thread per SNP reduces the
// populations in order p = 0..P-1 into the pooled summary of
// snp_summary_reduce.hpp:38-59 (q = ac / n by IEEE division, the product q * n rounded
// before it is added: no fused multiply-add, so the sum is the host's bit for bit), then
// applies keep_decision_pooled (snp_summary_reduce.hpp:64-79) and the population-coverage
// bound: drop a SNP when more than `maxmiss` of the populations have no call
// (extract_f2_core.cpp:245-259). The pooled missing-fraction test runs with its bound at 1,
// as extract-f2 sets it (cuda_backend_decode.cu:512-513), so it never drops anything.
//
// Two inputs: the packed exact counts of the SNP-major decode (population-major, ac2 | n <<
// 16), and FP64 q / n planes [P x M] (i + P * s), the layout of ComputeBackend::decode_af.
#include "stpf2_internal.cuh"

namespace stpf2 {

namespace {

// Allele-pair predicates of filter_decision.hpp:43-87, restated: A/C/G/T in either case,
// anything else is "no allele".
__device__ __forceinline__ char norm_allele(char a) {
    const char u = (a >= 'a' && a <= 'z') ? static_cast<char>(a - 0x20) : a;
    return (u == 'A' || u == 'C' || u == 'G' || u == 'T') ? u : '\0';
}
__device__ __forceinline__ char complement_of(char a) {
    switch (a) {
        case 'A': return 'T';
        case 'T': return 'A';
        case 'C': return 'G';
        case 'G': return 'C';
    }
    return '\0';
}
__device__ __forceinline__ bool purine(char a) { return a == 'A' || a == 'G'; }

struct Summary {
    double pooled_ref_count = 0.0, allele_count = 0.0, nonmissing = 0.0;
    int missing_pops = 0;
    // One population's q and n (n = 0: no call, q = 0), in population order.
    __device__ __forceinline__ void add(double q, double nd) {
        pooled_ref_count = __dadd_rn(pooled_ref_count, __dmul_rn(q, nd));
        allele_count = __dadd_rn(allele_count, nd);
        nonmissing = __dadd_rn(nonmissing, __ddiv_rn(nd, 2.0));  // called alleles / ploidy 2
        if (!(nd > 0.0)) ++missing_pops;
    }
};

__device__ __forceinline__ uint8_t decide(const Summary& sm, char ref, char alt, int chrom, const stp_snp_filter& f,
                                          int P, double total_indiv, double* out4, int64_t s, int64_t M) {
    const double ref_af = sm.allele_count > 0.0 ? __ddiv_rn(sm.pooled_ref_count, sm.allele_count) : 0.0;
    const double minor = (ref_af < 1.0 - ref_af) ? ref_af : 1.0 - ref_af;
    const double missing_frac = total_indiv > 0.0 ? 1.0 - __ddiv_rn(sm.nonmissing, total_indiv) : 1.0;
    if (out4) {
        out4[s] = ref_af;
        out4[M + s] = minor;
        out4[2 * M + s] = missing_frac;
        out4[3 * M + s] = sm.allele_count;
    }
    const char a = norm_allele(ref), b = norm_allele(alt);
    const bool multi = a == '\0' || b == '\0' || a == b;
    if (multi) return 0;
    if (f.strand_mode == STP_STRAND_DROP && a == complement_of(b)) return 0;
    if (!(minor >= f.maf_min)) return 0;
    if (!(missing_frac <= 1.0)) return 0;
    if (f.drop_monomorphic && minor == 0.0) return 0;
    if (f.transversions_only && purine(a) == purine(b)) return 0;  // a transition
    if (f.autosomes_only && !(chrom >= 1 && chrom <= 22)) return 0;
    if (f.maxmiss < 1.0 && static_cast<double>(sm.missing_pops) / static_cast<double>(P) > f.maxmiss) return 0;
    return 1;
}

__global__ void keep_mask_counts_kernel(const uint32_t* __restrict__ cnt, int64_t ld, int P, int64_t M,
                                        const char* __restrict__ ref, const char* __restrict__ alt,
                                        const int32_t* __restrict__ chrom, stp_snp_filter f, double total_indiv,
                                        uint8_t* __restrict__ keep, double* __restrict__ out4) {
    const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= M) return;
    Summary sm;
    for (int i = 0; i < P; ++i) {
        const uint32_t v = __ldg(cnt + static_cast<int64_t>(i) * ld + s);
        const uint32_t n = v >> 16;
        double q = 0.0, nd = 0.0;
        if (n > 0) {
            nd = static_cast<double>(n);
            q = __ddiv_rn(0.5 * static_cast<double>(v & 0xFFFFu), nd);  // finalize_af_counts: ac / n
        }
        sm.add(q, nd);
    }
    keep[s] = decide(sm, ref[s], alt[s], chrom[s], f, P, total_indiv, out4, s, M);
}

__global__ void keep_mask_qn_kernel(const double* __restrict__ Q, const double* __restrict__ N, int P, int64_t M,
                                    const char* __restrict__ ref, const char* __restrict__ alt,
                                    const int32_t* __restrict__ chrom, stp_snp_filter f, double total_indiv,
                                    uint8_t* __restrict__ keep, double* __restrict__ out4) {
    const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= M) return;
    Summary sm;
    for (int i = 0; i < P; ++i) {
        const int64_t o = static_cast<int64_t>(i) + static_cast<int64_t>(P) * s;
        sm.add(Q[o], N[o]);
    }
    keep[s] = decide(sm, ref[s], alt[s], chrom[s], f, P, total_indiv, out4, s, M);
}

// Compaction of FP64 [P x M] planes to the kept columns: out column keep_idx[s] <- column s.
__global__ void compact_columns_kernel(const double* __restrict__ in, int P, int64_t M,
                                       const int64_t* __restrict__ dst_col, double* __restrict__ out) {
    const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.y + threadIdx.y;
    if (s >= M) return;
    const int64_t d = dst_col[s];
    if (d < 0) return;
    for (int i = threadIdx.x; i < P; i += blockDim.x)
        out[static_cast<int64_t>(i) + static_cast<int64_t>(P) * d] = in[static_cast<int64_t>(i) + static_cast<int64_t>(P) * s];
}

}  // namespace

void launch_keep_mask_counts(Ctx& c, const uint32_t* cnt, int64_t ld, int P, int64_t M, const char* ref,
                             const char* alt, const int32_t* chrom, const stp_snp_filter& f, double total_indiv,
                             uint8_t* keep, double* out4, cudaStream_t s) {
    if (M <= 0) return;
    keep_mask_counts_kernel<<<static_cast<unsigned>((M + 255) / 256), 256, 0, s>>>(cnt, ld, P, M, ref, alt, chrom, f,
                                                                                   total_indiv, keep, out4);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_keep_mask_qn(Ctx& c, const double* Q, const double* N, int P, int64_t M, const char* ref, const char* alt,
                         const int32_t* chrom, const stp_snp_filter& f, double total_indiv, uint8_t* keep,
                         double* out4, cudaStream_t s) {
    if (M <= 0) return;
    keep_mask_qn_kernel<<<static_cast<unsigned>((M + 255) / 256), 256, 0, s>>>(Q, N, P, M, ref, alt, chrom, f,
                                                                               total_indiv, keep, out4);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_compact_columns(Ctx& c, const double* in, int P, int64_t M, const int64_t* dst_col, double* out,
                            cudaStream_t s) {
    if (M <= 0 || P <= 0) return;
    const dim3 block(32, 8);
    compact_columns_kernel<<<static_cast<unsigned>((M + 7) / 8), block, 0, s>>>(in, P, M, dst_col, out);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

}  // namespace stpf2
