// oracle/ref_shim.cpp
//
// TEST INFRASTRUCTURE ONLY. A C-ABI shim over the reference's own CpuBackend
// (src/device/cpu/cpu_backend.cpp), compiled in place from the reference sources by
// oracle/Makefile into oracle/_ref/libref_oracle.so. Tests use it to pin the C
// restatement in f2_oracle.c, and bench.py's reference arm times it as the
// reference's CPU implementation. It is never linked into the product.
//
// Each entry point forwards to the reference interface named beside it and copies the
// result into caller-owned buffers with the reference's own layouts.
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <span>
#include <vector>

#include "core/domain/block_partition_rule.hpp"
#include "device/backend.hpp"
#include "device/backend_factory.hpp"
#include "io/filter/snp_summary_reduce.hpp"

namespace {

std::unique_ptr<steppe::ComputeBackend>& backend() {
    thread_local std::unique_ptr<steppe::ComputeBackend> be = steppe::device::make_cpu_backend();
    return be;
}

}  // namespace

extern "C" {

// ComputeBackend::compute_f2_blocks (src/device/backend.hpp:687-692).
int ref_compute_f2_blocks(const double* Q, const double* V, const double* N, int P, long M,
                          const int* block_id, int n_block, double* f2, double* vpair,
                          int* block_sizes) {
    try {
        const steppe::core::MatView q{Q, P, M}, v{V, P, M}, n{N, P, M};
        const steppe::F2BlockTensor t =
            backend()->compute_f2_blocks(q, v, n, block_id, n_block, steppe::Precision::fp64());
        std::memcpy(f2, t.f2.data(), t.f2.size() * sizeof(double));
        std::memcpy(vpair, t.vpair.data(), t.vpair.size() * sizeof(double));
        for (std::size_t b = 0; b < t.block_sizes.size(); ++b) block_sizes[b] = t.block_sizes[b];
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// ComputeBackend::decode_af (src/device/backend.hpp:736) on the canonical tile.
int ref_decode_af(const std::uint8_t* packed, std::size_t bytes_per_record, std::size_t n_snp,
                  std::size_t n_ind, const std::size_t* pop_offsets, int P,
                  const int* sample_ploidy, int ploidy, int detect, double* q, double* v,
                  double* n) {
    try {
        steppe::DecodeTileView view;
        view.packed = packed;
        view.bytes_per_record = bytes_per_record;
        view.n_snp = n_snp;
        view.n_individuals = n_ind;
        view.pop_offsets = pop_offsets;
        view.n_pop = P;
        view.sample_ploidy = sample_ploidy;
        view.ploidy = ploidy;
        view.detect_ploidy_on_device = detect != 0;
        const steppe::DecodeResult r = backend()->decode_af(view);
        std::memcpy(q, r.q.data(), r.q.size() * sizeof(double));
        std::memcpy(v, r.v.data(), r.v.size() * sizeof(double));
        std::memcpy(n, r.n.data(), r.n.size() * sizeof(double));
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// ComputeBackend::detect_sample_ploidy_device (src/device/backend.hpp:765), host default.
int ref_detect_ploidy(const std::uint8_t* packed, std::size_t bytes_per_record,
                      std::size_t n_snp, std::size_t n_ind, int* ploidy) {
    try {
        steppe::DecodeTileView view;
        view.packed = packed;
        view.bytes_per_record = bytes_per_record;
        view.n_snp = n_snp;
        view.n_individuals = n_ind;
        const std::vector<int> r = backend()->detect_sample_ploidy_device(view);
        for (std::size_t g = 0; g < r.size(); ++g) ploidy[g] = r[g];
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// core::assign_blocks (src/core/domain/block_partition_rule.cpp:57-85).
int ref_assign_blocks(const int* chrom, const double* genpos, long M, double blgsize,
                      const double* physpos, double bp_window, int* block_id) {
    const std::span<const int> c(chrom, static_cast<std::size_t>(M));
    const std::span<const double> g(genpos, static_cast<std::size_t>(M));
    const std::span<const double> p =
        physpos ? std::span<const double>(physpos, static_cast<std::size_t>(M))
                : std::span<const double>{};
    const steppe::core::BlockPartition bp = steppe::core::assign_blocks(c, g, blgsize, p, bp_window);
    for (std::size_t s = 0; s < bp.block_id.size(); ++s) block_id[s] = bp.block_id[s];
    return bp.n_block;
}

// The reference's block jackknife (cpu_backend.cpp:2674-2720 and :2273-2306) reached
// through its public surface: per-item block values x[k + m*b] are placed as f2(0, k+1, b)
// of a zero-diagonal tensor, assemble_f3_triples((0, k+1, k+1)) returns exactly those
// values with their leave-one-out totals, and jackknife_diag gives the variance.
int ref_block_jackknife(const double* x, const int* block_sizes, long m, int nb, double* est,
                        double* var) {
    try {
        const int P = static_cast<int>(m) + 1;
        steppe::F2BlockTensor t;
        t.P = P;
        t.n_block = nb;
        t.block_sizes.assign(block_sizes, block_sizes + nb);
        const std::size_t slab = static_cast<std::size_t>(P) * static_cast<std::size_t>(P);
        t.f2.assign(slab * static_cast<std::size_t>(nb), 0.0);
        t.vpair.assign(slab * static_cast<std::size_t>(nb), 1.0);
        std::vector<int> triples;
        for (long k = 0; k < m; ++k) {
            for (int b = 0; b < nb; ++b) {
                const double val = x[static_cast<std::size_t>(k) + static_cast<std::size_t>(m) * b];
                const std::size_t a = static_cast<std::size_t>(k + 1);
                t.f2[0 + P * a + slab * b] = val;
                t.f2[a + 0 + slab * b] = val;
            }
            triples.push_back(0);
            triples.push_back(static_cast<int>(k + 1));
            triples.push_back(static_cast<int>(k + 1));
        }
        auto& be = backend();
        const steppe::F4Blocks f = be->assemble_f3_triples(t, triples, steppe::Precision::fp64());
        const steppe::JackknifeDiag d = be->jackknife_diag(f, f.block_sizes, steppe::Precision::fp64());
        for (long k = 0; k < m; ++k) {
            est[k] = f.x_total[static_cast<std::size_t>(k)];
            var[k] = d.var[static_cast<std::size_t>(k)];
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// The reference's f-statistic assembly and jackknife through its public surface
// (cpu_backend.cpp:2064-2216, :2273-2306), arguments as or_fstats. Returns the number of
// surviving blocks, or -1.
int ref_fstats(const double* f2, const double* vpair, const int* block_sizes, int P, int nb, int kind,
               const int* idx, long n_idx, long n_stat, double* est, double* var) {
    try {
        steppe::F2BlockTensor t;
        t.P = P;
        t.n_block = nb;
        const std::size_t n = static_cast<std::size_t>(P) * static_cast<std::size_t>(P) * static_cast<std::size_t>(nb);
        t.f2.assign(f2, f2 + n);
        t.vpair.assign(vpair, vpair + n);
        t.block_sizes.assign(block_sizes, block_sizes + nb);
        auto& be = backend();
        steppe::F4Blocks f;
        if (kind == 0) f = be->assemble_f4_quartets(t, std::span<const int>(idx, static_cast<std::size_t>(4 * n_stat)), steppe::Precision::fp64());
        else if (kind == 1) f = be->assemble_f3_triples(t, std::span<const int>(idx, static_cast<std::size_t>(3 * n_stat)), steppe::Precision::fp64());
        else f = be->assemble_f4(t, std::span<const int>(idx, static_cast<std::size_t>(n_stat)),
                                 std::span<const int>(idx + n_stat, static_cast<std::size_t>(n_idx - n_stat)),
                                 steppe::Precision::fp64());
        const steppe::JackknifeDiag d = be->jackknife_diag(f, f.block_sizes, steppe::Precision::fp64());
        const std::size_t m = static_cast<std::size_t>(f.nl) * static_cast<std::size_t>(f.nr);
        for (std::size_t k = 0; k < m; ++k) {
            est[k] = k < f.x_total.size() ? f.x_total[k] : 0.0;
            var[k] = k < d.var.size() ? d.var[k] : 0.0;
        }
        return f.n_block;
    } catch (const std::exception&) {
        return -1;
    }
}

// extract-f2's per-SNP keep mask as the reference decides it: the shared pooled summary and
// keep rule (io::filter::derive_pooled_summary_one / keep_decision_pooled,
// src/io/filter/snp_summary_reduce.hpp:38-79, ploidy 2, the pooled missing-fraction bound at
// 1 as cuda_backend_decode.cu:512-513 sets it) and the population-coverage bound of
// extract_f2_core.cpp:245-259 / decode_compact_kernel.cu:53-64, over Q / N [P x M].
// strand_mode: 0 Drop, 1 Keep, 2 Flip. summary4 (optional) [4 * M]: ref AF, minor AF,
// missing fraction, allele count.
int ref_keep_mask(const double* Q, const double* N, int P, long M, const char* ref, const char* alt, const int* chrom,
                  double maf_min, double maxmiss, int autosomes_only, int drop_monomorphic, int transversions_only,
                  int strand_mode, double total_indiv, unsigned char* keep, double* summary4) {
    steppe::FilterConfig cfg;
    cfg.maf_min = maf_min;
    cfg.geno_max_missing = 1.0;
    cfg.autosomes_only = autosomes_only != 0;
    cfg.drop_monomorphic = drop_monomorphic != 0;
    cfg.transversions_only = transversions_only != 0;
    cfg.strand_mode = strand_mode == 0 ? steppe::StrandMode::Drop
                      : strand_mode == 1 ? steppe::StrandMode::Keep : steppe::StrandMode::Flip;
    for (long s = 0; s < M; ++s) {
        const steppe::io::filter::PooledSnpSummary ps =
            steppe::io::filter::derive_pooled_summary_one(Q, N, P, s, 2.0, total_indiv);
        bool k = steppe::io::filter::keep_decision_pooled(ps, ref[s], alt[s], chrom[s], cfg, true);
        if (k && maxmiss < 1.0) {
            int miss = 0;
            for (int p = 0; p < P; ++p)
                if (N[static_cast<long>(P) * s + p] <= 0.0) ++miss;
            if (static_cast<double>(miss) / static_cast<double>(P) > maxmiss) k = false;
        }
        keep[s] = k ? 1 : 0;
        if (summary4) {
            summary4[s] = ps.pooled_ref_af;
            summary4[M + s] = ps.pooled_minor_af;
            summary4[2 * M + s] = ps.missing_frac;
            summary4[3 * M + s] = ps.pooled_allele_count;
        }
    }
    return 0;
}

}  // extern "C"
