/* include/stpf2.h — C ABI of libstpf2.so, the B200 (sm_100a) f2 block-tensor extraction.
 *
 * One streaming pass turns 2-bit PACKEDANCESTRYMAP genotypes into the reference's
 * F2BlockTensor: per-jackknife-block f2 means and both-present SNP counts, FP64,
 * element (i, j, b) at i + P*j + P*P*b (include/steppe/fstats.hpp:19-59 in the
 * reference). Plain pointers and sizes only; no C++ or torch types cross this line.
 *
 * Each entry point names the reference interface it replaces. Errors come back as an
 * stp_status; stp_last_error() gives the message of the calling thread's last failure.
 * Degenerate extents (P <= 0, M <= 0, n_block <= 0) give empty/zero results, not errors,
 * as in the reference (src/device/cpu/cpu_backend.cpp:234).
 */
#ifndef STPF2_H
#define STPF2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STPF2_ABI_VERSION 2

/* Status codes. 0..5 keep the numbering of steppe::Status (include/steppe/error.hpp:14-26);
 * the rest stand for the reference's exception types (std::invalid_argument /
 * std::runtime_error / CudaError in src/device/cuda/check.cuh:34-60). */
typedef enum stp_status {
    STP_OK = 0,
    STP_DEVICE_OOM = 1,
    STP_INVALID_CONFIG = 5,
    STP_INVALID_ARGUMENT = 100, /* std::invalid_argument: bad sizes, null pointers */
    STP_RUNTIME_ERROR = 101,    /* std::runtime_error: malformed partition, M > INT_MAX */
    STP_CUDA_ERROR = 102,       /* CudaError: a CUDA runtime/driver call failed */
    STP_NO_DEVICE = 103,        /* no CUDA device (the reference's "GPU product" error) */
    STP_DEVICE_TIMEOUT = 104    /* a bounded device-side wait ran out; results invalid */
} stp_status;

/* Contraction arithmetic. The reference's Precision (include/steppe/config.hpp:74-95)
 * selects FP64 / emulated FP64 cuBLAS; this build's modes are: */
typedef enum stp_precision {
    STP_PREC_FP32_SIMT = 0,  /* plain FP32 CUDA-core contraction, FP64 combine */
    STP_PREC_SPLIT_BF16 = 1, /* tcgen05 split-BF16 (hi+lo, 3 products), FP32 TMEM, FP64 drain */
    STP_PREC_SPLIT_F16 = 2,  /* tcgen05 split-FP16 (scaled hi+lo, 3 products), same pipeline;
                                FP32 sums over 64-SNP chunks (max rel f2 error ~8e-7) */
    STP_PREC_SPLIT_F16_FINE = 3, /* split-FP16 with FP32 sums over 32-SNP chunks (~4.5e-7,
                                   ~15% slower contraction) */
    STP_PREC_FIXED_I8 = 4 /* tcgen05 kind::i8 on 32-bit fixed-point operands held as four
                             int8 digits, exact int32 accumulation, FP64 combine: f2 within
                             ~1e-9 absolute of FP64 per SNP, far less on block means */
} stp_precision;

/* steppe::ExtractPloidy (include/steppe/extract.hpp) */
typedef enum stp_ploidy_mode {
    STP_PLOIDY_AUTO = 0,   /* per-sample detection over the first min(1000, M) SNPs */
    STP_PLOIDY_PSEUDO = 1, /* every sample pseudo-haploid */
    STP_PLOIDY_DIPLOID = 2 /* every sample diploid */
} stp_ploidy_mode;

/* steppe::StrandMode (include/steppe/config.hpp:128). The keep mask never flips alleles,
 * so FLIP keeps ambiguous SNPs as KEEP does (src/io/filter/snp_filter.hpp:6). */
typedef enum stp_strand_mode {
    STP_STRAND_DROP = 0,
    STP_STRAND_KEEP = 1,
    STP_STRAND_FLIP = 2
} stp_strand_mode;

/* The per-SNP filters of extract-f2 (FilterConfig, include/steppe/config.hpp:131-164, as
 * extract_f2_core.cpp:188-260 applies them; the include / exclude SNP lists are the
 * caller's to apply). A SNP is kept when its alleles are two distinct bases, it is not
 * strand-ambiguous (under STP_STRAND_DROP), its pooled minor allele frequency is >= maf_min,
 * it is polymorphic (when drop_monomorphic), a transversion (when transversions_only), on
 * chromosomes 1..22 (when autosomes_only), and at most maxmiss of the populations have no
 * call at it (maxmiss = 1: no bound). */
typedef struct stp_snp_filter {
    double maf_min;
    double maxmiss;
    int32_t autosomes_only;
    int32_t drop_monomorphic;
    int32_t transversions_only;
    int32_t strand_mode; /* stp_strand_mode */
} stp_snp_filter;

typedef struct stp_ctx stp_ctx;
typedef struct stp_plan stp_plan;

/* SNP-major PACKEDANCESTRYMAP records (the .geno payload after its header record):
 * record s holds individual r's code at byte r/4, MSB-first (src/io/eigenstrat_format.cpp
 * :17-85, src/io/geno_reader.cpp:465-514). */
typedef struct stp_geno_view {
    const uint8_t* records;    /* n_snp records, `pitch` bytes apart */
    uint64_t bytes_per_record; /* max(48, ceil(n_ind/4)) */
    uint64_t pitch;            /* distance between records in bytes (>= bytes_per_record) */
    int64_t n_snp;
    int64_t n_ind;             /* individuals in the file (.ind rows) */
    int32_t on_device;         /* records is a device pointer (DecodeTileView::packed_on_device) */
} stp_geno_view;

/* One extraction request (the inputs of steppe::run_extract_f2 after the front end:
 * src/app/extract_f2_core.cpp:93-407). Host pointers unless stated. */
typedef struct stp_f2_request {
    stp_geno_view geno;
    const int64_t* sel_rows;      /* [n_sel] file rows of the selected samples, pop-contiguous */
    const int64_t* pop_offsets;   /* [n_pop+1] into sel_rows (io::GenoReader::build_selection) */
    int32_t n_pop;
    const int32_t* sample_ploidy; /* [n_sel] 1/2, or NULL to use ploidy_mode */
    int32_t ploidy_mode;          /* stp_ploidy_mode, used when sample_ploidy is NULL */
    const int32_t* block_id;      /* [n_snp] (or [n_kept]) non-decreasing in [0, n_block) (core::assign_blocks) */
    int32_t n_block;
    int32_t precision;            /* stp_precision */
    /* Optional SNP compaction (the kept set of extract_f2_core.cpp:188-291): kept_rows[k] is
     * the record row of the request's k-th SNP, strictly increasing, k < n_kept. The decode
     * reads those records in place (no compacted copy is made); block_id then has n_kept
     * entries. Ploidy is still detected on the first min(1000, n_snp) records, as the
     * reference detects it before filtering. NULL: every record, in order. In
     * stp_f2_extract_batch a request with kept rows runs on its own. */
    const int64_t* kept_rows;
    int64_t n_kept;
} stp_f2_request;

/* Caller-owned result buffers in F2BlockTensor layout. */
typedef struct stp_f2_output {
    double* f2;            /* [P*P*n_block] per-block f2 means */
    double* vpair;         /* [P*P*n_block] both-present SNP counts */
    int32_t* block_sizes;  /* [n_block] host */
    int32_t on_device;     /* f2 / vpair are device pointers */
    int32_t* ploidy_out;   /* optional [n_sel] host: the ploidy used per selected sample */
} stp_f2_output;

/* ---- context ------------------------------------------------------------------------ */

/* make_cuda_backend(device) (src/device/backend_factory.hpp:18-21). */
stp_ctx* stp_create(int device, stp_status* status);
void stp_destroy(stp_ctx* ctx);
/* Message of the calling thread's last failed call ("" if none). */
const char* stp_last_error(void);
int stp_abi_version(void);
/* Kernel launches issued by this context since creation (every kernel of this library). */
uint64_t stp_launch_count(const stp_ctx* ctx);

/* ---- decode ------------------------------------------------------------------------- */

/* ComputeBackend::detect_sample_ploidy_device (src/device/backend.hpp:765) on SNP-major
 * records: ploidy[g] = 2 if selected sample g has a het within the first min(1000, n_snp)
 * SNPs, else 1. */
stp_status stp_detect_ploidy(stp_ctx* ctx, const stp_geno_view* geno, const int64_t* sel_rows,
                             int64_t n_sel, int32_t* ploidy);

/* ComputeBackend::detect_sample_ploidy_device(DecodeTileView) (src/device/backend.hpp:765)
 * on the canonical individual-major tile: record r (bytes_per_record >= ceil(n_snp/4))
 * holds individual r's SNP codes MSB-first; ploidy[r] = 2 if a het occurs within its first
 * min(1000, n_snp) SNPs, else 1. `packed` is a device pointer when packed_on_device != 0. */
stp_status stp_detect_ploidy_tile(stp_ctx* ctx, const uint8_t* packed, uint64_t bytes_per_record,
                                  int64_t n_snp, int64_t n_ind, int32_t packed_on_device,
                                  int32_t* ploidy);

/* Integer decode (decode_af.hpp:58-65): ac2 = 2*ac and n per (pop, SNP), column-major
 * [P x n_snp] host arrays. The bit-exact form of ComputeBackend::decode_af. */
stp_status stp_decode_counts(stp_ctx* ctx, const stp_geno_view* geno, const int64_t* sel_rows,
                             const int64_t* pop_offsets, int32_t n_pop,
                             const int32_t* sample_ploidy, int32_t ploidy_mode,
                             int32_t* ac2, int32_t* n);

/* Allocation-free form of stp_decode_counts. No counterpart in the reference (its backends
 * allocate per call). For callers that cannot allocate device memory at call time: a
 * process whose caching allocator or memory pool already owns the device's free memory
 * (a cudaMalloc there fails or forces the pool to release memory and synchronise), and a
 * caller on a latency-critical stream (cudaFree synchronises the whole device).
 *
 * Records must be on the device (geno->on_device = 1) with a 16-byte aligned base and
 * pitch; d_ac2 / d_n are caller-owned device buffers of n_pop * n_snp int32, written in
 * the column-major layout of stp_decode_counts. Every intermediate lives in one static
 * device array of 32 MiB (every GPU that loads the library holds it until the process
 * exits), whose address the library takes once per device
 * (cudaGetSymbolAddress) on the first call; make that first call before any stream
 * capture. A request needing more scratch than that (about n_sel * n_snp / 4 bytes of
 * canonical genotypes plus 12 bytes per SNP) fails with STP_INVALID_ARGUMENT. The call
 * sets the scratch that must start at a fixed value (file-row map, error flag) itself.
 * Calls share the scratch: calls on one device that overlap in time (other threads or
 * streams) race and must be serialised by the caller. Work runs on `stream` (NULL = the
 * context stream); the call returns after it has finished. */
stp_status stp_decode_counts_noalloc(stp_ctx* ctx, const stp_geno_view* geno, const int64_t* sel_rows,
                                     const int64_t* pop_offsets, int32_t n_pop,
                                     const int32_t* sample_ploidy, int32_t ploidy_mode,
                                     int32_t* d_ac2, int32_t* d_n, void* stream);

/* extract-f2's per-SNP keep mask, on the device (the regime-B mask of
 * src/device/cuda/decode_compact_kernel.cu:39-68): exact counts of the selected samples
 * (as stp_decode_counts), then per SNP the pooled summary of
 * src/io/filter/snp_summary_reduce.hpp:38-59 over the populations in order (q = ac / n, the
 * product q * n rounded before it is added, ploidy 2) and the rules of stp_snp_filter.
 * ref / alt / chrom: host [n_snp] (.snp alleles and chromosome codes). Out: keep [n_snp]
 * host (1 = keep), *n_kept, and optionally summary [4 * n_snp] host: pooled ref allele
 * frequency, pooled minor allele frequency, missing fraction, pooled called-allele count
 * (io::filter::PerSnpSummary). The kept rows are what stp_f2_request.kept_rows takes. */
stp_status stp_snp_keep_mask(stp_ctx* ctx, const stp_geno_view* geno, const int64_t* sel_rows,
                             const int64_t* pop_offsets, int32_t n_pop, const int32_t* sample_ploidy,
                             int32_t ploidy_mode, const char* ref, const char* alt, const int32_t* chrom,
                             const stp_snp_filter* filter, uint8_t* keep, int64_t* n_kept, double* summary);

/* The canonical individual-major tile of a DecodeTileView (record g: individual g's SNP
 * codes, MSB-first; bytes_per_record >= ceil(n_snp/4)) rewritten as SNP-major
 * PACKEDANCESTRYMAP records in device memory, the layout stp_geno_view reads: record s at
 * d_records + s * pitch holds individual g's code at byte g/4 (pitch >= ceil(n_ind/4)). Lets
 * a caller holding the reference's tile (extract_f2_core.cpp:113-160) use the record-based
 * entry points, e.g. the streamed extraction with kept rows (RedecodeSource, the streamed
 * tiers of src/device/stream_f2_blocks.hpp:44-63). */
stp_status stp_canonical_to_records(stp_ctx* ctx, const uint8_t* packed, uint64_t bytes_per_record,
                                    int64_t n_snp, int64_t n_ind, int32_t packed_on_device,
                                    uint8_t* d_records, uint64_t pitch);

/* ComputeBackend::decode_af_compact_filter (src/device/backend.hpp:914-925) on the
 * canonical individual-major tile (as stp_decode_af): the keep mask of stp_snp_keep_mask
 * over the tile's SNPs (total_indiv: the selection's individual count for the missing
 * fraction), then q / v / n of the kept SNPs only, [P x n_kept] column-major FP64, device
 * pointers when out_on_device. With q = v = n = NULL only keep [n_snp] (host) and *n_kept are
 * written: a caller that sizes its outputs from *n_kept calls twice. */
stp_status stp_decode_af_compact_filter(stp_ctx* ctx, const uint8_t* packed, uint64_t bytes_per_record,
                                        int64_t n_snp, int64_t n_ind, const int64_t* pop_offsets, int32_t n_pop,
                                        const int32_t* sample_ploidy, int32_t ploidy, int32_t packed_on_device,
                                        const char* ref, const char* alt, const int32_t* chrom,
                                        const stp_snp_filter* filter, double total_indiv, uint8_t* keep,
                                        int64_t* n_kept, double* q, double* v, double* n, int32_t out_on_device);

/* ComputeBackend::decode_af(DecodeTileView) (src/device/backend.hpp:736) on the canonical
 * individual-major tile: record g (bytes_per_record >= ceil(n_snp/4)) holds selected
 * sample g's SNP codes MSB-first; pop_offsets[P+1] index records. sample_ploidy NULL with
 * detect != 0 detects ploidy; NULL with detect == 0 uses `ploidy`. Out: q, v, n host
 * [P x n_snp] column-major FP64. */
stp_status stp_decode_af(stp_ctx* ctx, const uint8_t* packed, uint64_t bytes_per_record,
                         int64_t n_snp, int64_t n_ind, const int64_t* pop_offsets, int32_t n_pop,
                         const int32_t* sample_ploidy, int32_t ploidy, int32_t detect,
                         int32_t packed_on_device, double* q, double* v, double* n);

/* ---- f2 ------------------------------------------------------------------------------ */

/* ComputeBackend::compute_f2_blocks(MatView Q, V, N, block_id, n_block, Precision)
 * (src/device/backend.hpp:687-692). Q/V/N host [P x M] column-major. */
stp_status stp_f2_from_qvn(stp_ctx* ctx, const double* Q, const double* V, const double* N,
                           int32_t P, int64_t M, const int32_t* block_id, int32_t n_block,
                           int32_t precision, double* f2, double* vpair, int32_t* block_sizes);

/* ComputeBackend::compute_f2_blocks_device (src/device/backend.hpp:694-701): the same as
 * stp_f2_from_qvn with the result left on the device, d_f2 / d_vpair device buffers of
 * P*P*n_block doubles (DeviceF2Blocks); Q / V / N are device pointers when qvn_on_device
 * (a DeviceDecodeResult's q / v / n), host pointers otherwise. */
stp_status stp_f2_from_qvn_device(stp_ctx* ctx, const double* Q, const double* V, const double* N,
                                  int32_t P, int64_t M, const int32_t* block_id, int32_t n_block,
                                  int32_t precision, int32_t qvn_on_device, double* d_f2, double* d_vpair,
                                  int32_t* block_sizes);

/* Receives one finished run of blocks [b0, b1) of a streamed extraction: (b1 - b0) P x P
 * slabs of f2 and of vpair in F2BlockTensor order (slab b - b0 at f2 + (b - b0)*P*P), in
 * host memory that stays valid until the callback returns. Runs arrive in block order on
 * the calling thread. Return 0 to go on; anything else stops the call with
 * STP_RUNTIME_ERROR. */
typedef int (*stp_slab_sink)(void* user, int32_t b0, int32_t b1, const double* f2, const double* vpair);

/* ComputeBackend::compute_f2_blocks_streamed (src/device/backend.hpp:724-734) over dense Q /
 * V / N: the f2 blocks of stp_f2_from_qvn handed to `sink` in runs of blocks (the reference's
 * StreamTarget tiers, host RAM or disk), so the whole P x P x n_block tensor never has to
 * exist on the device or in one host buffer. Tensor-core precisions only. */
stp_status stp_f2_from_qvn_streamed(stp_ctx* ctx, const double* Q, const double* V, const double* N,
                                    int32_t P, int64_t M, const int32_t* block_id, int32_t n_block,
                                    int32_t precision, stp_slab_sink sink, void* user,
                                    int32_t* block_sizes);

/* The extract-f2 hot path streamed to `sink` (the out-of-core tiers of
 * src/device/cuda/cuda_backend_f2_blocks.cu:349-603): records (host or device) in, runs of
 * finished blocks out, two runs in flight. block_sizes (optional host [n_block]).
 * Tensor-core precisions only. */
stp_status stp_f2_extract_streamed(stp_ctx* ctx, const stp_f2_request* req, stp_slab_sink sink, void* user,
                                   int32_t* block_sizes);

/* The extract-f2 hot path: packed genotypes -> ploidy -> decode -> per-block contraction
 * -> FP64 F2BlockTensor (src/app/extract_f2_core.cpp:93-407, Resident tier). With host
 * records and host outputs on the tensor cores, the call streams segments of whole blocks
 * and downloads only the upper 128-row bands of each (exactly symmetric) slab; it fills
 * the lower tiles of the host outputs itself, on up to hardware_concurrency host threads,
 * before it returns. */
stp_status stp_f2_extract_blocks(stp_ctx* ctx, const stp_f2_request* req, stp_f2_output* out);

/* Many independent requests (each its own populations and block map). The reference runs
 * requests one at a time (run_extract_f2 per request, src/app/extract_f2_core.cpp:93-407);
 * it has no batch entry. Tensor-core requests that read the same panel (same geno view)
 * with the same arithmetic run as one group: one ploidy pass and one canonical transpose
 * over the union of their samples, a decode per request into its own operand images, and
 * one persistent contraction launch over every request's (block, tile pair) items. FP32
 * SIMT and empty requests run one by one. Outputs and errors are per request as in
 * stp_f2_extract_blocks. */
stp_status stp_f2_extract_batch(stp_ctx* ctx, const stp_f2_request* reqs, int32_t n_req,
                                stp_f2_output* outs);

/* f-statistics from an F2BlockTensor and their block jackknife, FP64 on the device.
 * Blocks where some pair is missing (vpair = 0) and another present are dropped
 * (survivor_blocks, src/device/cpu/cpu_backend.cpp:124-151); per surviving block the
 * statistic is assembled from f2 slabs (assemble_f4_quartets / assemble_f3_triples /
 * assemble_f4, cpu_backend.cpp:2064-2216) and est / var are the block-size-weighted
 * estimate and jackknife variance (compute_loo_and_total + jackknife_diag, :2674-2720,
 * :2273-2306). kind STP_FSTAT_F4: idx holds n_stat quartets (p1, p2, p3, p4) ->
 * (f2(p2,p3) + f2(p1,p4) - f2(p1,p3) - f2(p2,p4)) / 2; STP_FSTAT_F3: n_stat triples
 * (c, a, b) -> (f2(c,a) + f2(c,b) - f2(a,b)) / 2; STP_FSTAT_F4_LEFT_RIGHT: idx holds the
 * n_stat left indices then the n_idx - n_stat right ones, and statistic j + nr*i
 * (nl = n_stat - 1, nr = n_idx - n_stat - 1) is (f2(Li,R0) + f2(L0,Rj) - f2(L0,R0) -
 * f2(Li,Rj)) / 2. f2 / vpair: [P x P x n_block] (host, or device when on_device);
 * block_sizes, idx, est, var: host. With no surviving block est = var = 0. */
typedef enum stp_fstat_kind {
    STP_FSTAT_F4 = 0,
    STP_FSTAT_F3 = 1,
    STP_FSTAT_F4_LEFT_RIGHT = 2
} stp_fstat_kind;

stp_status stp_fstats(stp_ctx* ctx, const double* f2, const double* vpair, const int32_t* block_sizes,
                      int32_t P, int32_t n_block, int32_t on_device, int32_t kind, const int32_t* idx,
                      int64_t n_idx, int64_t n_stat, double* est, double* var, int32_t* n_survivors);

/* Completion time of each request of this context's last stp_f2_extract_batch call, in ms
 * from the start of its group's device work (%globaltimer stamps written by the last work
 * item of each request); NaN for requests that ran on their own. No counterpart in the
 * reference. */
stp_status stp_last_batch_times(stp_ctx* ctx, double* ms, int32_t n);

/* The bound on every device-side wait of the fixed-point contraction (STP_PREC_FIXED_I8),
 * and a test hook. No counterpart in the reference, whose kernels do not wait on one
 * another. timeout_ns (0 = the default of 4 s) bounds each wait; when one runs out the kernel
 * stops, frees its tensor memory and the call returns STP_DEVICE_TIMEOUT with the context
 * still usable. withhold_stage >= 0 makes the f2 kernel's feed stop before that pipeline
 * stage (its MMA issuer's wait then runs out: how the timeout path is tested); -1 turns it
 * off. Per context. */
stp_status stp_set_wait_bounds(stp_ctx* ctx, uint64_t timeout_ns, int64_t withhold_stage);

/* Tile classes of the fixed-point contraction (the per-size-class choices of
 * cuda_backend_f2_blocks.cu:55-74, made per work item here): bit k of partial_feed_mask set
 * makes an operand tile side with 8k+1 .. 8k+8 valid populations (of 128 rows) stage only its
 * valid 8-row groups per plane (nine copies) instead of the whole 36 KiB side (two copies).
 * Results do not depend on it. The default is the measured table that
 * steppecu_b200/autotune.py writes (steppecu_b200/tile_classes.json). Per context. */
stp_status stp_set_tile_classes(stp_ctx* ctx, uint32_t partial_feed_mask);

/* Block jackknife over per-block values (cpu_backend.cpp:2674-2720, :2273-2306), FP64 on
 * the device: x[k + m*b] with m = P*P -> est[m], var[m]. Host pointers. */
stp_status stp_f2_jackknife(stp_ctx* ctx, const double* x, const int32_t* block_sizes, int64_t m,
                            int32_t n_block, double* est, double* var);

/* ---- plans: device-resident repeated extraction --------------------------------------- */

/* Builds everything a request needs once (operand buffers, block layout, work list,
 * ploidy) so stp_plan_run only launches kernels. The request's genotype records must be on
 * the device; the plan keeps no reference to host arrays. A plan uses its context's stream
 * and workspaces: destroy every plan of a context before the context (stp_destroy does
 * not free them). */
stp_plan* stp_plan_create(stp_ctx* ctx, const stp_f2_request* req, stp_status* status);
/* Enqueues decode + contraction on `stream` (a cudaStream_t, NULL = the context stream);
 * d_f2/d_vpair are device buffers of P*P*n_block doubles. Asynchronous. */
stp_status stp_plan_run(stp_plan* plan, const uint8_t* d_records, double* d_f2, double* d_vpair,
                        void* stream);
/* The same pass as stp_plan_run, replayed from one CUDA graph: the first call for a given
 * (d_records, d_f2, d_vpair) captures the pass's kernels (ploidy, transpose, decode,
 * contraction) into a graph and instantiates it; later calls only launch it on `stream`.
 * Plan timing must be off. Asynchronous. */
stp_status stp_plan_run_graph(stp_plan* plan, const uint8_t* d_records, double* d_f2, double* d_vpair,
                              void* stream);
/* Comparison form of the contraction (tensor-core plans): one launch per jackknife block
 * instead of one persistent launch over every block's tile pairs. Same results. */
stp_status stp_plan_set_per_block_launch(stp_plan* plan, int32_t enable);
/* Kernel launches one stp_plan_run issues. */
int32_t stp_plan_launches(const stp_plan* plan);
/* Timing: with timing enabled, every stp_plan_run records CUDA events on its stream around
 * the decode (ploidy + decode kernels) and the contraction kernel. stp_plan_last_times
 * returns the mean device time of each, in ms, over all runs since timing was (re-)enabled
 * (0 if none). Enabling resets the set of timed runs. */
stp_status stp_plan_set_timing(stp_plan* plan, int32_t enable);
stp_status stp_plan_last_times(const stp_plan* plan, float* decode_ms, float* contract_ms);
void stp_plan_destroy(stp_plan* plan);

#ifdef __cplusplus
}
#endif

#endif /* STPF2_H */
