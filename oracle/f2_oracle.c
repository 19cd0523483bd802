/* oracle/f2_oracle.c
 *
 * TEST INFRASTRUCTURE ONLY — the CPU checker for the f2 extraction path (see
 * f2_oracle.h). Plain C11, single-threaded, compiled with -ffp-contract=off so the
 * double arithmetic is evaluated term by term exactly as the reference's x86-64 build
 * evaluates it (no fused multiply-adds).
 */
#include "f2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { kCodesPerByte = 4, kMissing = 3, kHet = 1, kPloidyDetectSnps = 1000 };

/* decode_af.hpp:38-43 */
int or_genotype_code(uint8_t byte, int k) {
    const int shift = (kCodesPerByte - 1 - (k % kCodesPerByte)) * 2;
    return (byte >> shift) & 3;
}

/* cpu_backend.cpp:73-95 */
void or_detect_ploidy_canonical(const uint8_t* packed, size_t bpr, size_t n_snp,
                                size_t n_ind, int32_t* ploidy) {
    const size_t window = n_snp < (size_t)kPloidyDetectSnps ? n_snp : (size_t)kPloidyDetectSnps;
    for (size_t g = 0; g < n_ind; ++g) {
        ploidy[g] = 1;
        const uint8_t* rec = packed + g * bpr;
        for (size_t s = 0; s < window; ++s) {
            if (or_genotype_code(rec[s / 4], (int)(s % 4)) == kHet) {
                ploidy[g] = 2;
                break;
            }
        }
    }
}

static inline int pa_code(const uint8_t* records, size_t bpr, size_t s, int64_t row) {
    return or_genotype_code(records[s * bpr + (size_t)(row / 4)], (int)(row % 4));
}

void or_detect_ploidy_pa(const uint8_t* records, size_t bpr, size_t n_snp,
                         const int64_t* sel_rows, size_t n_sel, int32_t* ploidy) {
    const size_t window = n_snp < (size_t)kPloidyDetectSnps ? n_snp : (size_t)kPloidyDetectSnps;
    for (size_t g = 0; g < n_sel; ++g) {
        ploidy[g] = 1;
        for (size_t s = 0; s < window; ++s) {
            if (pa_code(records, bpr, s, sel_rows[g]) == kHet) {
                ploidy[g] = 2;
                break;
            }
        }
    }
}

/* decode_af.hpp:58-65: a valid code with ploidy in {1,2} adds code/(3-ploidy) to ac and
 * ploidy to n. Carried as ac2 = 2*ac so the pseudo-haploid half-integers stay integral. */
static inline void fold(int code, int pl, int32_t* ac2, int32_t* n) {
    if (code != kMissing && (pl == 1 || pl == 2)) {
        *ac2 += (pl == 2) ? 2 * code : code;
        *n += pl;
    }
}

void or_decode_counts_pa(const uint8_t* records, size_t bpr, size_t n_snp,
                         const int64_t* sel_rows, const int64_t* pop_offsets, int P,
                         const int32_t* ploidy, int default_ploidy,
                         int32_t* ac2, int32_t* n) {
    for (size_t s = 0; s < n_snp; ++s) {
        for (int i = 0; i < P; ++i) {
            int32_t a = 0, c = 0;
            for (int64_t g = pop_offsets[i]; g < pop_offsets[i + 1]; ++g) {
                const int pl = ploidy ? ploidy[g] : default_ploidy;
                fold(pa_code(records, bpr, s, sel_rows[g]), pl, &a, &c);
            }
            ac2[(size_t)i + (size_t)P * s] = a;
            n[(size_t)i + (size_t)P * s] = c;
        }
    }
}

/* cpu_backend.cpp:267-319 */
void or_decode_af_canonical(const uint8_t* packed, size_t bpr, size_t n_snp, size_t n_ind,
                            const int64_t* pop_offsets, int P, const int32_t* sample_ploidy,
                            int ploidy, int detect, double* q, double* v, double* n) {
    const size_t pm = (size_t)P * n_snp;
    memset(q, 0, pm * sizeof(double));
    memset(v, 0, pm * sizeof(double));
    memset(n, 0, pm * sizeof(double));
    if (P <= 0 || n_snp == 0) return;
    int32_t* detected = NULL;
    const int32_t* eff = sample_ploidy;
    if (eff == NULL && detect) {
        detected = (int32_t*)malloc((n_ind ? n_ind : 1) * sizeof(int32_t));
        or_detect_ploidy_canonical(packed, bpr, n_snp, n_ind, detected);
        eff = detected;
    }
    for (int i = 0; i < P; ++i) {
        for (size_t s = 0; s < n_snp; ++s) {
            double ac = 0.0;
            int64_t cnt = 0;
            for (int64_t g = pop_offsets[i]; g < pop_offsets[i + 1]; ++g) {
                const int code = or_genotype_code(packed[(size_t)g * bpr + s / 4], (int)(s % 4));
                const int pl = eff ? eff[g] : ploidy;
                if (code != kMissing && (pl == 2 || pl == 1)) {
                    ac += (double)code / (3.0 - (double)pl);
                    cnt += pl;
                }
            }
            const size_t off = (size_t)i + (size_t)P * s;
            if (cnt > 0) {
                const double nd = (double)cnt;
                n[off] = nd;
                q[off] = ac / nd;
                v[off] = 1.0;
            }
        }
    }
    free(detected);
}

/* decode_af.hpp:87-97 (finalize_af_counts) on ac = ac2/2, which is exact in double. */
void or_counts_to_qvn(const int32_t* ac2, const int32_t* n, size_t count, double* q,
                      double* v, double* nd) {
    for (size_t k = 0; k < count; ++k) {
        if (n[k] > 0) {
            nd[k] = (double)n[k];
            q[k] = ((double)ac2[k] * 0.5) / nd[k];
            v[k] = 1.0;
        } else {
            nd[k] = 0.0;
            q[k] = 0.0;
            v[k] = 0.0;
        }
    }
}

/* transpose_canonical_kernel.cu:40-74 */
void or_transpose_pa_to_canonical(const uint8_t* records, size_t bpr, size_t n_snp,
                                  const int64_t* sel_rows, size_t n_sel, uint8_t* out) {
    const size_t out_bpr = (n_snp + 3) / 4;
    for (size_t g = 0; g < n_sel; ++g) {
        for (size_t b = 0; b < out_bpr; ++b) {
            uint8_t packed = 0;
            for (int k = 0; k < 4; ++k) {
                const size_t s = b * 4 + (size_t)k;
                if (s >= n_snp) break;
                const int code = pa_code(records, bpr, s, sel_rows[g]);
                packed |= (uint8_t)(code << ((3 - k) * 2));
            }
            out[g * out_bpr + b] = packed;
        }
    }
}

/* cpu_backend.cpp:60-70 — cascade summation, base case 128, in long double. */
static long double pairwise_sum(const long double* a, size_t n) {
    if (n == 0) return 0.0L;
    if (n <= 128) {
        long double s = 0.0L;
        for (size_t k = 0; k < n; ++k) s += a[k];
        return s;
    }
    const size_t h = n / 2;
    return pairwise_sum(a, h) + pairwise_sum(a + h, n - h);
}

/* f2_estimator.hpp:22-27 */
static double het_correction(double q, double n) {
    const double nm1 = n - 1.0;
    const double denom = (nm1 > 1.0) ? nm1 : 1.0;
    return q * (1.0 - q) / denom;
}

/* cpu_backend.cpp:217-264 with the per-pair body at :155-174 */
int or_compute_f2_blocks(const double* Q, const double* V, const double* N, int P, long M,
                         const int32_t* block_id, int n_block, double* f2, double* vpair,
                         int32_t* block_sizes) {
    if (n_block > 0) {
        const size_t total = (size_t)(P > 0 ? P : 0) * (size_t)(P > 0 ? P : 0) * (size_t)n_block;
        memset(f2, 0, total * sizeof(double));
        memset(vpair, 0, total * sizeof(double));
        memset(block_sizes, 0, (size_t)n_block * sizeof(int32_t));
    }
    if (P <= 0 || M <= 0 || n_block <= 0) return 0;

    /* block_partition_rule.hpp:56-96 — contiguous, non-decreasing partition */
    long* begin = (long*)calloc((size_t)n_block, sizeof(long));
    long* end = (long*)calloc((size_t)n_block, sizeof(long));
    int prev = -1;
    for (long s = 0; s < M;) {
        const int b = block_id[s];
        if (b < 0 || b >= n_block || b < prev) {
            free(begin);
            free(end);
            return -1;
        }
        long e = s;
        while (e < M && block_id[e] == b) ++e;
        begin[b] = s;
        end[b] = e;
        prev = b;
        s = e;
    }
    for (int b = 0; b < n_block; ++b) block_sizes[b] = (int32_t)(end[b] - begin[b]);

    long double* terms = (long double*)malloc((size_t)M * sizeof(long double));
    const size_t slab = (size_t)P * (size_t)P;
    for (int b = 0; b < n_block; ++b) {
        const size_t base = slab * (size_t)b;
        for (int i = 0; i < P; ++i) {
            for (int j = i; j < P; ++j) {
                long count = 0;
                for (long s = begin[b]; s < end[b]; ++s) {
                    const size_t oi = (size_t)i + (size_t)P * (size_t)s;
                    const size_t oj = (size_t)j + (size_t)P * (size_t)s;
                    if (V[oi] == 0.0 || V[oj] == 0.0) continue;
                    const double pi = Q[oi], pj = Q[oj];
                    const double hi = het_correction(pi, N[oi]);
                    const double hj = het_correction(pj, N[oj]);
                    const double d = pi - pj;
                    terms[count++] = (long double)(d * d - hi - hj);
                }
                const long double num = pairwise_sum(terms, (size_t)count);
                const double vp = (double)count;
                const double val = (vp > 0.0) ? ((double)num / vp) : 0.0;
                const size_t ij = base + (size_t)i + (size_t)P * (size_t)j;
                const size_t ji = base + (size_t)j + (size_t)P * (size_t)i;
                f2[ij] = val;
                f2[ji] = val;
                vpair[ij] = vp;
                vpair[ji] = vp;
            }
        }
    }
    free(terms);
    free(begin);
    free(end);
    return 0;
}

/* block_partition_rule.cpp:18-44 */
static int block_walk(const int32_t* chrom, const double* pos, long M, double window,
                      int32_t* block_id) {
    double fpos = -1.0e20;
    int prev_chrom = -1;
    long global = -1;
    for (long s = 0; s < M; ++s) {
        const int c = chrom[s];
        const double p = pos[s];
        if (c != prev_chrom || (p - fpos) >= window) {
            ++global;
            fpos = p;
            prev_chrom = c;
        }
        block_id[s] = (int32_t)global;
    }
    return (int)(global + 1);
}

static int all_zero(const double* pos, long M) {
    for (long s = 0; s < M; ++s)
        if (pos[s] != 0.0) return 0;
    return 1;
}

/* block_partition_rule.cpp:57-85 */
int or_assign_blocks(const int32_t* chrom, const double* genpos, long M, double bs,
                     const double* physpos, double bp_window, int32_t* block_id) {
    if (!(bs > 0.0)) return 0;
    if (M <= 0) return 0;
    if (physpos != NULL && bp_window > 0.0 && all_zero(genpos, M) && !all_zero(physpos, M))
        return block_walk(chrom, physpos, M, bp_window, block_id);
    return block_walk(chrom, genpos, M, bs, block_id);
}

/* cpu_backend.cpp:2674-2720 then :2273-2306 */
void or_block_jackknife(const double* x, const int32_t* block_sizes, long m, int nb,
                        double* est, double* var) {
    if (m <= 0 || nb <= 0) return;
    long double n_ld = 0.0L;
    for (int b = 0; b < nb; ++b) n_ld += (long double)block_sizes[b];
    const double n = (double)n_ld;
    double* loo = (double*)malloc((size_t)nb * sizeof(double));
    for (long k = 0; k < m; ++k) {
        long double num = 0.0L;
        for (int b = 0; b < nb; ++b)
            num += (long double)x[(size_t)k + (size_t)m * (size_t)b] * (long double)block_sizes[b];
        const double tot = (double)(num / n_ld);
        for (int b = 0; b < nb; ++b) {
            const double rel = (double)block_sizes[b] / n;
            const double xv = x[(size_t)k + (size_t)m * (size_t)b];
            loo[b] = (tot - xv * rel) / (1.0 - rel);
        }
        long double wnum = 0.0L, wden = 0.0L;
        for (int b = 0; b < nb; ++b) {
            const double w = 1.0 - (double)block_sizes[b] / n;
            wnum += (long double)loo[b] * (long double)w;
            wden += (long double)w;
        }
        const double totline = (double)(wnum / wden);
        long double diffsum = 0.0L;
        for (int b = 0; b < nb; ++b) diffsum += (long double)totline - (long double)loo[b];
        const double term1 = (double)(diffsum / (long double)nb) * (double)nb;
        long double wbl = 0.0L;
        for (int b = 0; b < nb; ++b) wbl += (long double)loo[b] * (long double)block_sizes[b];
        const double term2 = (double)(wbl / n_ld);
        const double e = term1 + term2;
        est[k] = e;
        long double acc = 0.0L;
        for (int b = 0; b < nb; ++b) {
            const double bl = (double)block_sizes[b];
            const double h = n / bl;
            const double sq = sqrt(h - 1.0);
            const double xtau = (e * h - loo[b] * (h - 1.0) - totline) / sq;
            acc += (long double)xtau * (long double)xtau;
        }
        var[k] = (double)(acc / (long double)nb);
    }
    free(loo);
}

/* cpu_backend.cpp:124-151. */
int or_survivor_blocks(const double* vpair, int P, int nb, int32_t* keep) {
    const size_t slab = (size_t)P * (size_t)P;
    int kept = 0;
    for (int b = 0; b < nb; ++b) {
        int any_missing = 0, any_present = 0;
        for (size_t e = 0; e < slab; ++e) {
            if (!(vpair[slab * (size_t)b + e] > 0.0)) any_missing = 1;
            else any_present = 1;
            if (any_missing && any_present) break;
        }
        keep[b] = !(any_missing && any_present);
        kept += keep[b];
    }
    return kept;
}

/* cpu_backend.cpp:2064-2216 then 2674-2720 / 2273-2306. */
int or_fstats(const double* f2, const double* vpair, const int32_t* block_sizes, int P, int nb, int kind,
              const int32_t* idx, long n_idx, long n_stat, double* est, double* var, double* x_blocks) {
    const size_t slab = (size_t)P * (size_t)P;
    long m = 0, nl = 0, nr = 0;
    if (kind == 0 || kind == 1) m = n_stat;
    else {
        nl = n_stat - 1;
        nr = n_idx - n_stat - 1;
        m = (nl > 0 && nr > 0) ? nl * nr : 0;
    }
    for (long k = 0; k < m; ++k) est[k] = var[k] = 0.0;
    if (m <= 0 || nb <= 0) return 0;
    int32_t* keep = (int32_t*)malloc((size_t)nb * sizeof(int32_t));
    const int ns = or_survivor_blocks(vpair, P, nb, keep);
    int32_t* bl = (int32_t*)malloc((size_t)(ns > 0 ? ns : 1) * sizeof(int32_t));
    double* x = (double*)malloc((size_t)m * (size_t)(ns > 0 ? ns : 1) * sizeof(double));
#define F2AT(i, j, b) f2[(size_t)(i) + (size_t)P * (size_t)(j) + slab * (size_t)(b)]
    int bs = 0;
    for (int b = 0; b < nb; ++b) {
        if (!keep[b]) continue;
        bl[bs] = block_sizes[b];
        for (long k = 0; k < m; ++k) {
            double v = 0.0;
            if (kind == 0) {
                const int p1 = idx[4 * k], p2 = idx[4 * k + 1], p3 = idx[4 * k + 2], p4 = idx[4 * k + 3];
                v = 0.5 * (F2AT(p2, p3, b) + F2AT(p1, p4, b) - F2AT(p1, p3, b) - F2AT(p2, p4, b));
            } else if (kind == 1) {
                const int pc = idx[3 * k], pa = idx[3 * k + 1], pb = idx[3 * k + 2];
                v = 0.5 * (F2AT(pc, pa, b) + F2AT(pc, pb, b) - F2AT(pa, pb, b));
            } else {
                const long i = k / nr, j = k % nr;  /* k = j + nr*i */
                const int L0 = idx[0], R0 = idx[n_stat], Li = idx[1 + i], Rj = idx[n_stat + 1 + j];
                v = 0.5 * (F2AT(Li, R0, b) + F2AT(L0, Rj, b) - F2AT(L0, R0, b) - F2AT(Li, Rj, b));
            }
            x[(size_t)k + (size_t)m * (size_t)bs] = v;
        }
        ++bs;
    }
#undef F2AT
    if (x_blocks) memcpy(x_blocks, x, (size_t)m * (size_t)ns * sizeof(double));
    if (ns > 0) or_block_jackknife(x, bl, m, ns, est, var);
    free(keep);
    free(bl);
    free(x);
    return ns;
}

/* ---- extract-f2 keep mask ---------------------------------------------------------------- */

/* filter_decision.hpp:43-58: A/C/G/T in either case, anything else is no allele (0). */
static char or_norm_allele(char a) {
    const char u = (a >= 'a' && a <= 'z') ? (char)(a - 0x20) : a;
    return (u == 'A' || u == 'C' || u == 'G' || u == 'T') ? u : 0;
}

static char or_complement(char a) {
    switch (a) {
        case 'A': return 'T';
        case 'T': return 'A';
        case 'C': return 'G';
        case 'G': return 'C';
    }
    return 0;
}

void or_keep_mask(const double* Q, const double* N, int P, long M, const char* ref, const char* alt,
                  const int32_t* chrom, double maf_min, double maxmiss, int autosomes_only, int drop_monomorphic,
                  int transversions_only, int strand_mode, double total_indiv, uint8_t* keep, double* summary4) {
    for (long s = 0; s < M; ++s) {
        /* snp_summary_reduce.hpp:38-59: products rounded before the add (no contraction). */
        double pooled = 0.0, alleles = 0.0, nonmiss = 0.0;
        int missing_pops = 0;
        for (int p = 0; p < P; ++p) {
            const long o = (long)P * s + p;
            const double prod = Q[o] * N[o];
            pooled = pooled + prod;
            alleles += N[o];
            nonmiss += N[o] / 2.0;
            if (N[o] <= 0.0) ++missing_pops;
        }
        const double ref_af = alleles > 0.0 ? pooled / alleles : 0.0;
        const double minor = (ref_af < 1.0 - ref_af) ? ref_af : (1.0 - ref_af);
        const double missing = total_indiv > 0.0 ? 1.0 - nonmiss / total_indiv : 1.0;
        if (summary4) {
            summary4[s] = ref_af;
            summary4[M + s] = minor;
            summary4[2 * M + s] = missing;
            summary4[3 * M + s] = alleles;
        }
        /* keep_decision_pooled (snp_summary_reduce.hpp:64-79), pooled missing bound 1. */
        const char a = or_norm_allele(ref[s]), b = or_norm_allele(alt[s]);
        int k = 1;
        if (a == 0 || b == 0 || a == b) k = 0;                                  /* multiallelic */
        else if (strand_mode == 0 && a == or_complement(b)) k = 0;             /* strand-ambiguous */
        else if (!(minor >= maf_min)) k = 0;
        else if (!(missing <= 1.0)) k = 0;
        else if (drop_monomorphic && minor == 0.0) k = 0;
        else if (transversions_only && ((a == 'A' || a == 'G') == (b == 'A' || b == 'G'))) k = 0;
        else if (autosomes_only && !(chrom[s] >= 1 && chrom[s] <= 22)) k = 0;
        /* the population-coverage bound (extract_f2_core.cpp:245-259) */
        if (k && maxmiss < 1.0 && (double)missing_pops / (double)P > maxmiss) k = 0;
        keep[s] = (uint8_t)k;
    }
}
