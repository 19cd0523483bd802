/* oracle/f2_oracle.h
 *
 * TEST INFRASTRUCTURE ONLY. A plain-C, single-threaded restatement of the reference's
 * CPU f2 block-tensor extraction (Steppe's CpuBackend), used as the checker by tests/,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg. Nothing in the product
 * path (libstpf2.so, the C++ host pipeline, the Python package) links or calls it.
 *
 * Every function cites the reference file:line whose behaviour it restates. Layouts
 * follow the reference:
 *   - Q/V/N and counts are column-major [P x M]: element (i, s) at i + P*s
 *     (src/core/internal/views.hpp:14-24);
 *   - f2/vpair are [P x P x B]: element (i, j, b) at i + P*j + P*P*b
 *     (include/steppe/fstats.hpp:52-58);
 *   - packed genotypes carry four 2-bit codes per byte, MSB-first, code 3 = missing
 *     (src/core/internal/decode_af.hpp:20-43).
 */
#ifndef STPF2_ORACLE_H
#define STPF2_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* decode_af.hpp:38-43 — 2-bit code k (mod 4) of a packed byte, MSB-first. */
int or_genotype_code(uint8_t byte, int k);

/* cpu_backend.cpp:73-95 — per-sample ploidy on the individual-major canonical tile:
 * 2 (diploid) if a het (code 1) occurs within the first min(1000, n_snp) SNPs of the
 * sample's record, else 1 (pseudo-haploid). */
void or_detect_ploidy_canonical(const uint8_t* packed, size_t bytes_per_record,
                                size_t n_snp, size_t n_ind, int32_t* ploidy);

/* The same rule read straight from PACKEDANCESTRYMAP SNP-major records (one record of
 * bytes_per_record bytes per SNP, individuals in file order). sel_rows[g] is the file
 * row of selected individual g; the canonical tile the reference scans is the transpose
 * of these records (transpose_canonical_kernel.cu:40-74), so the result is identical. */
void or_detect_ploidy_pa(const uint8_t* records, size_t bytes_per_record, size_t n_snp,
                         const int64_t* sel_rows, size_t n_sel, int32_t* ploidy);

/* cpu_backend.cpp:267-319 with decode_af.hpp:58-65 — per-(pop, SNP) integer counts read
 * from SNP-major records: ac2 = 2*ac (ac is a half-integer for pseudo-haploids) and
 * n = called allele count. pop_offsets[P+1] index sel_rows; ploidy[g] per selected
 * sample (NULL -> default_ploidy for all). Out: ac2/n [P x M] column-major. */
void or_decode_counts_pa(const uint8_t* records, size_t bytes_per_record, size_t n_snp,
                         const int64_t* sel_rows, const int64_t* pop_offsets, int P,
                         const int32_t* ploidy, int default_ploidy,
                         int32_t* ac2, int32_t* n);

/* cpu_backend.cpp:267-319 — decode_af on the canonical individual-major tile
 * (record g = selected individual g, ceil(M/4) bytes, SNP codes MSB-first).
 * sample_ploidy NULL and detect != 0 -> ploidy detected as in or_detect_ploidy_canonical;
 * sample_ploidy NULL and detect == 0 -> `ploidy` for all. Out: q, v, n [P x M]. */
void or_decode_af_canonical(const uint8_t* packed, size_t bytes_per_record, size_t n_snp,
                            size_t n_ind, const int64_t* pop_offsets, int P,
                            const int32_t* sample_ploidy, int ploidy, int detect,
                            double* q, double* v, double* n);

/* decode_af.hpp:87-97 — counts -> (q, v, n): q = (ac2/2)/n, v = 1, when n > 0. */
void or_counts_to_qvn(const int32_t* ac2, const int32_t* n, size_t count,
                      double* q, double* v, double* nd);

/* PACKEDANCESTRYMAP -> canonical individual-major tile (transpose_canonical_kernel.cu:40-74):
 * out record g (out_bpr = ceil(n_snp/4) bytes) holds the codes of file row sel_rows[g]. */
void or_transpose_pa_to_canonical(const uint8_t* records, size_t bytes_per_record,
                                  size_t n_snp, const int64_t* sel_rows, size_t n_sel,
                                  uint8_t* out);

/* cpu_backend.cpp:217-264 (+ :60-70 pairwise long-double sum, :155-174 per-pair body,
 * f2_estimator.hpp:22-46) — per-block f2 means and both-present counts.
 * block_id[M] must be non-decreasing in [0, n_block) (block_partition_rule.hpp:56-96).
 * Returns 0 on success, -1 on a malformed partition (the reference throws). P <= 0,
 * M <= 0 or n_block <= 0 give an all-zero result and return 0 (cpu_backend.cpp:234). */
int or_compute_f2_blocks(const double* Q, const double* V, const double* N, int P,
                         long M, const int32_t* block_id, int n_block,
                         double* f2, double* vpair, int32_t* block_sizes);

/* block_partition_rule.cpp:18-85 — the AT2 block walk. Writes block_id[M]; returns
 * n_block (0 for an illegal width or M <= 0). physpos may be NULL. */
int or_assign_blocks(const int32_t* chrom, const double* genpos_morgans, long M,
                     double block_size_morgans, const double* physpos, double bp_window,
                     int32_t* block_id);

/* cpu_backend.cpp:2674-2720 (compute_loo_and_total) and :2273-2306 (jackknife_diag),
 * applied to m = P*P per-pair block values x[k + m*b]: block-size-weighted estimate
 * est[k] and jackknife variance var[k]. */
void or_block_jackknife(const double* x, const int32_t* block_sizes, long m, int nb,
                        double* est, double* var);

/* cpu_backend.cpp:124-151 (survivor_blocks): keep[b] = 0 when block b has both a missing
 * pair (vpair not > 0, f2_estimator.hpp:49-51) and a present one, else 1. Returns the
 * number kept. */
int or_survivor_blocks(const double* vpair, int P, int nb, int32_t* keep);

/* f-statistics from an F2BlockTensor over its surviving blocks, with the block jackknife
 * of each (cpu_backend.cpp:2064-2216 assemble_f4 / assemble_f4_quartets /
 * assemble_f3_triples, then or_block_jackknife). kind 0: quartets idx[4k..4k+3] ->
 * 0.5(f2(p2,p3) + f2(p1,p4) - f2(p1,p3) - f2(p2,p4)); kind 1: triples (c, a, b) ->
 * 0.5(f2(c,a) + f2(c,b) - f2(a,b)); kind 2: left idx[0..n_left) and right
 * idx[n_left..n_left+n_right) with L0 = left[0], R0 = right[0]: statistic
 * k = j + nr*i (i < nl = n_left-1, j < nr = n_right-1) -> 0.5(f2(Li,R0) + f2(L0,Rj) -
 * f2(L0,R0) - f2(Li,Rj)). n_stat: quartets / triples count (kinds 0, 1) or n_left
 * (kind 2, n_right = n_idx - n_left). Returns the number of surviving blocks;
 * x_blocks (optional, n_out x survivors) receives the assembled per-block values. */
int or_fstats(const double* f2, const double* vpair, const int32_t* block_sizes, int P, int nb, int kind,
              const int32_t* idx, long n_idx, long n_stat, double* est, double* var, double* x_blocks);

/* extract-f2's per-SNP keep mask (src/io/filter/snp_summary_reduce.hpp:38-79,
 * src/io/filter/filter_decision.hpp:22-90, extract_f2_core.cpp:245-259): per SNP s the
 * pooled summary over populations p = 0..P-1 of Q / N [P x M] (i + P*s), ploidy 2, then the
 * keep rule (multiallelic, strand under Drop, MAF, monomorphic, transversions, autosomes
 * 1..22) and the population-coverage bound maxmiss. strand_mode 0 Drop, 1 Keep, 2 Flip.
 * summary4 (optional) [4 * M]: ref AF, minor AF, missing fraction, allele count. */
void or_keep_mask(const double* Q, const double* N, int P, long M, const char* ref, const char* alt,
                  const int32_t* chrom, double maf_min, double maxmiss, int autosomes_only, int drop_monomorphic,
                  int transversions_only, int strand_mode, double total_indiv, uint8_t* keep, double* summary4);

#ifdef __cplusplus
}
#endif

#endif /* STPF2_ORACLE_H */
