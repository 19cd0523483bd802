// steppecu_b200/adapter/b200_backend.cpp
//
// The drop-in on the reference side: steppe::ComputeBackend (src/device/backend.hpp:673-1654)
// implemented over libstpf2.so's C ABI (include/stpf2.h). A maintainer adds this file to
// the reference's device library, links -lstpf2, declares make_b200_backend next to
// make_cuda_backend (src/device/backend_factory.hpp:18-21) and selects it where Resources
// builds gpus[g].backend (src/device/resources.hpp:45-70). It is compiled against the
// reference's headers by tests/test_integration_adapter.py; nothing in libstpf2.so
// includes it.
//
// Hot-path virtuals, each forwarded:
//   compute_f2, compute_f2_blocks          -> stp_f2_from_qvn
//   compute_f2_blocks_device               -> stp_f2_from_qvn_device (DeviceF2Blocks)
//   compute_f2_blocks_into                 -> stp_f2_from_qvn (host slabs at dst)
//   compute_f2_blocks_streamed             -> stp_f2_from_qvn_streamed, or with a
//                                             RedecodeSource stp_canonical_to_records +
//                                             stp_f2_extract_streamed over the kept rows
//   decode_af                              -> stp_decode_af
//   decode_af_compact_filter               -> stp_decode_af_compact_filter (DeviceDecodeResult)
//   detect_sample_ploidy_device            -> stp_detect_ploidy_tile
// Every other virtual keeps the base-class behaviour ("not supported by this backend").
//
// Precision: the reference's Precision asks for FP64 GEMMs (Fp64) or Ozaki-emulated FP64
// with a mantissa budget (EmulatedFp64, default 40 bits; docs/userguide/precision-and-
// tiers.md:23-24 puts emu32 at ~8.6e-9 worst case). This library computes f2 in
// STP_PREC_FIXED_I8: exact int32 tensor-core sums over 32-bit fixed-point operands, within
// ~5e-10 of exact per SNP term. EmulatedFp64 with mantissa_bits <= 32 maps to it (its error
// is no larger than the emulation asked for); Tf32 maps to the FP32 CUDA-core form; Fp64
// and wider emulation are refused with Status::InvalidConfig unless the backend was created
// with accept_fixed_point, which is the caller's statement that ~1e-9 suffices.
#include <cstdio>
#include <cstring>
#include <memory>
#include <source_location>
#include <span>
#include <string>
#include <vector>

#include "device/backend.hpp"
#include "device/cuda/check.cuh"                   // CudaError (-> Status::DeviceOom)
#include "device/cuda/device_decode_result_impl.cuh"  // DeviceDecodeResult::Impl (DeviceBuffer owners)
#include "device/cuda/device_f2_blocks_impl.cuh"   // DeviceF2Blocks::Impl
#include "device/f2_blocks_out.hpp"                // DiskF2Blocks
#include "device/f2_disk_format.hpp"               // F2DiskHeader, STPF2BK1
#include "device/stream_f2_blocks.hpp"             // StreamTarget, RedecodeSource
#include "stpf2.h"

namespace steppe {
namespace {

// A status other than STP_OK becomes the exception the reference throws for it
// (src/device/cuda/check.cuh:34-60, include/steppe/error.hpp:14-26).
[[noreturn]] void raise(stp_status s) {
    const std::string m = stp_last_error();
    switch (s) {
        case STP_INVALID_ARGUMENT: throw std::invalid_argument(m);
        case STP_INVALID_CONFIG: throw std::invalid_argument("invalid config: " + m);
        case STP_DEVICE_OOM:  // -> Status::DeviceOom, exit 3
            throw device::CudaError(cudaErrorMemoryAllocation, m.c_str(), std::source_location::current());
        default: throw std::runtime_error(m);
    }
}
void check(stp_status s) {
    if (s != STP_OK) raise(s);
}

// The arithmetic for a reference Precision (the policy in the file header).
int32_t precision_mode(const Precision& p, bool accept_fixed_point) {
    switch (p.kind) {
        case Precision::Kind::Tf32: return STP_PREC_FP32_SIMT;
        case Precision::Kind::EmulatedFp64:
            if (p.mantissa_bits <= 32 || accept_fixed_point) return STP_PREC_FIXED_I8;
            break;
        case Precision::Kind::Fp64:
            if (accept_fixed_point) return STP_PREC_FIXED_I8;
            break;
    }
    throw std::invalid_argument(
        "invalid config: the B200 backend computes f2 in 32-bit fixed point with exact integer sums "
        "(~1e-9 of FP64); FP64 and emulated FP64 wider than 32 bits need make_cuda_backend, or "
        "create the B200 backend with accept_fixed_point");
}

std::vector<int64_t> offsets64(const std::size_t* po, int n_pop) {
    std::vector<int64_t> o(static_cast<std::size_t>(n_pop) + 1);
    for (int i = 0; i <= n_pop; ++i) o[static_cast<std::size_t>(i)] = static_cast<int64_t>(po[i]);
    return o;
}

}  // namespace

class B200Backend final : public ComputeBackend {
  public:
    explicit B200Backend(int device, bool accept_fixed_point = false)
        : device_(device), accept_fixed_point_(accept_fixed_point) {
        stp_status st = STP_OK;
        ctx_ = stp_create(device, &st);
        if (!ctx_) raise(st);
    }
    ~B200Backend() override { stp_destroy(ctx_); }

    // backend.hpp:682-685: f2 over the whole SNP range is the one-block case.
    F2Result compute_f2(const core::MatView& Q, const core::MatView& V, const core::MatView& N,
                        const Precision& prec) override {
        F2Result r;
        r.P = Q.P;
        const std::size_t n = static_cast<std::size_t>(Q.P) * static_cast<std::size_t>(Q.P);
        r.f2.assign(n, 0.0);
        r.vpair.assign(n, 0.0);
        if (Q.P <= 0 || Q.M <= 0) return r;
        std::vector<int32_t> block_id(static_cast<std::size_t>(Q.M), 0);
        int32_t block_size = 0;
        check(stp_f2_from_qvn(ctx_, Q.data, V.data, N.data, Q.P, Q.M, block_id.data(), 1, mode(prec), r.f2.data(),
                              r.vpair.data(), &block_size));
        return r;
    }

    // backend.hpp:687-692
    F2BlockTensor compute_f2_blocks(const core::MatView& Q, const core::MatView& V, const core::MatView& N,
                                    const int* block_id, int n_block, const Precision& prec) override {
        F2BlockTensor t;
        t.P = Q.P;
        t.n_block = n_block;
        t.f2.assign(t.size(), 0.0);
        t.vpair.assign(t.size(), 0.0);
        t.block_sizes.assign(static_cast<std::size_t>(std::max(n_block, 0)), 0);
        if (Q.P <= 0 || Q.M <= 0 || n_block <= 0) return t;  // cpu_backend.cpp:234: empty, not an error
        check(stp_f2_from_qvn(ctx_, Q.data, V.data, N.data, Q.P, Q.M, block_id, n_block, mode(prec), t.f2.data(),
                              t.vpair.data(), t.block_sizes.data()));
        return t;
    }

    // backend.hpp:694-701: the tensor stays in device memory, owned by the handle.
    device::DeviceF2Blocks compute_f2_blocks_device(const core::MatView& Q, const core::MatView& V,
                                                    const core::MatView& N, const int* block_id, int n_block,
                                                    const Precision& prec) override {
        device::DeviceF2Blocks d;
        d.P = Q.P;
        d.n_block = n_block;
        d.device_id = device_;
        d.block_sizes.assign(static_cast<std::size_t>(std::max(n_block, 0)), 0);
        d.impl = std::make_unique<device::DeviceF2Blocks::Impl>();
        if (d.empty()) return d;
        d.impl->f2 = device::DeviceBuffer<double>(d.size());
        d.impl->vpair = device::DeviceBuffer<double>(d.size());
        check(stp_f2_from_qvn_device(ctx_, Q.data, V.data, N.data, Q.P, Q.M, block_id, n_block, mode(prec),
                                     /*qvn_on_device=*/0, d.impl->f2.data(), d.impl->vpair.data(),
                                     d.block_sizes.data()));
        return d;
    }

    // backend.hpp:712-721: this call's blocks into a caller's host tensor at block b0 (the
    // multi-GPU fan-out's shard write, f2_blocks_multigpu_core.cpp:40-85).
    void compute_f2_blocks_into(const core::MatView& Q, const core::MatView& V, const core::MatView& N,
                                const int* block_id, int n_block, int b0, double* dst_f2, double* dst_vpair,
                                int* block_sizes_dst, const Precision& prec) override {
        if (n_block <= 0) return;
        const std::size_t off = static_cast<std::size_t>(Q.P) * static_cast<std::size_t>(Q.P) *
                                static_cast<std::size_t>(b0);
        check(stp_f2_from_qvn(ctx_, Q.data, V.data, N.data, Q.P, Q.M, block_id, n_block, mode(prec), dst_f2 + off,
                              dst_vpair + off, block_sizes_dst + b0));
    }

    // backend.hpp:724-734: runs of finished blocks into the StreamTarget (host RAM or a
    // STPF2BK1 file), never the whole tensor on the device.
    void compute_f2_blocks_streamed(const core::MatView& Q, const core::MatView& V, const core::MatView& N,
                                    const int* block_id, int n_block, const Precision& prec,
                                    device::StreamTarget& target, const device::RedecodeSource* redecode) override {
        const int P = redecode ? static_cast<int>(redecode->n_pop) : Q.P;
        std::unique_ptr<Sink> sink;
        if (target.tier == device::OutputTier::HostRam) {
            if (!target.host_dst) throw std::runtime_error("compute_f2_blocks_streamed: HostRam tier needs host_dst");
            sink = std::make_unique<HostSink>(*target.host_dst, P, n_block);
        } else if (target.tier == device::OutputTier::Disk) {
            if (!target.disk_dst) throw std::runtime_error("compute_f2_blocks_streamed: Disk tier needs disk_dst");
            sink = std::make_unique<DiskSink>(target.disk_path, P, n_block);
        } else {
            throw std::runtime_error("compute_f2_blocks_streamed: the Resident tier does not stream");
        }
        std::vector<int32_t> sizes(static_cast<std::size_t>(std::max(n_block, 0)), 0);
        if (P > 0 && n_block > 0) {
            if (redecode) streamed_from_tile(*redecode, block_id, n_block, prec, *sink, sizes.data());
            else
                check(stp_f2_from_qvn_streamed(ctx_, Q.data, V.data, N.data, P, Q.M, block_id, n_block, mode(prec),
                                               &Sink::call, sink.get(), sizes.data()));
        }
        sink->finish(sizes, target);
    }

    // backend.hpp:736
    DecodeResult decode_af(const DecodeTileView& v) override {
        DecodeResult r;
        r.P = v.n_pop;
        r.M = static_cast<long>(v.n_snp);
        const std::size_t n = static_cast<std::size_t>(std::max(v.n_pop, 0)) * v.n_snp;
        r.q.resize(n);
        r.v.resize(n);
        r.n.resize(n);
        if (n == 0) return r;
        const std::vector<int64_t> po = offsets64(v.pop_offsets, v.n_pop);
        check(stp_decode_af(ctx_, v.packed, v.bytes_per_record, static_cast<int64_t>(v.n_snp),
                            static_cast<int64_t>(v.n_individuals), po.data(), v.n_pop, v.sample_ploidy, v.ploidy,
                            v.detect_ploidy_on_device, v.packed_on_device, r.q.data(), r.v.data(), r.n.data()));
        return r;
    }

    // backend.hpp:765
    std::vector<int> detect_sample_ploidy_device(const DecodeTileView& v) override {
        std::vector<int> out(v.n_individuals);
        if (v.n_individuals == 0) return out;
        check(stp_detect_ploidy_tile(ctx_, v.packed, v.bytes_per_record, static_cast<int64_t>(v.n_snp),
                                     static_cast<int64_t>(v.n_individuals), v.packed_on_device, out.data()));
        return out;
    }

    // backend.hpp:914-925: the tile's SNP window [s_lo, s_lo + n_snp) decoded, filtered by
    // extract-f2's keep mask, and its kept columns left on the device.
    device::DeviceDecodeResult decode_af_compact_filter(const DecodeTileView& tile, std::span<const char> ref,
                                                        std::span<const char> alt, std::span<const int> chrom,
                                                        std::span<const double> genpos,
                                                        std::span<const double> physpos, const FilterConfig& cfg,
                                                        std::span<const std::size_t> pop_individuals, int ploidy,
                                                        double maxmiss, long s_lo) override {
        (void)ploidy;  // the pooled summary counts alleles per diploid individual, as the reference's extract path
        device::DeviceDecodeResult out;
        out.device_id = device_;
        out.P = tile.n_pop;
        out.impl = std::make_unique<device::DeviceDecodeResult::Impl>();
        const int64_t M = static_cast<int64_t>(tile.n_snp);
        if (tile.n_pop <= 0 || M <= 0) return out;
        if (s_lo % 4 != 0) throw std::invalid_argument("decode_af_compact_filter: the SNP window must start on a byte");
        const std::uint8_t* packed = tile.packed + s_lo / 4;  // every record shifts by the same bytes
        const std::vector<int64_t> po = offsets64(tile.pop_offsets, tile.n_pop);
        double total = 0.0;
        for (std::size_t p : pop_individuals) total += static_cast<double>(p);
        if (pop_individuals.size() != static_cast<std::size_t>(tile.n_pop)) total = static_cast<double>(po.back());
        const stp_snp_filter f = filter_of(cfg, maxmiss);
        std::vector<std::uint8_t> keep(static_cast<std::size_t>(M));
        int64_t n_kept = 0;
        auto call = [&](double* q, double* v, double* n) {
            check(stp_decode_af_compact_filter(ctx_, packed, tile.bytes_per_record, M,
                                               static_cast<int64_t>(tile.n_individuals), po.data(), tile.n_pop,
                                               tile.sample_ploidy, tile.ploidy, tile.packed_on_device, ref.data(),
                                               alt.data(), chrom.data(), &f, total, keep.data(), &n_kept, q, v, n,
                                               /*out_on_device=*/1));
        };
        call(nullptr, nullptr, nullptr);  // the keep mask and the kept count
        out.M_kept = n_kept;
        if (n_kept <= 0) return out;
        const std::size_t pm = static_cast<std::size_t>(tile.n_pop) * static_cast<std::size_t>(n_kept);
        out.impl->q = device::DeviceBuffer<double>(pm);
        out.impl->v = device::DeviceBuffer<double>(pm);
        out.impl->n = device::DeviceBuffer<double>(pm);
        call(out.impl->q.data(), out.impl->v.data(), out.impl->n.data());
        for (int64_t s = 0; s < M; ++s) {
            if (!keep[static_cast<std::size_t>(s)]) continue;
            out.chrom_kept.push_back(chrom[static_cast<std::size_t>(s)]);
            out.genpos_kept.push_back(genpos[static_cast<std::size_t>(s)]);
            if (physpos.size() == static_cast<std::size_t>(M)) out.physpos_kept.push_back(physpos[static_cast<std::size_t>(s)]);
        }
        return out;
    }

  private:
    // Where a streamed extraction's runs of finished blocks go (StreamTarget's tiers).
    struct Sink {
        virtual ~Sink() = default;
        virtual void take(int b0, int b1, const double* f2, const double* vpair) = 0;
        virtual void finish(const std::vector<int32_t>& sizes, device::StreamTarget& target) = 0;
        static int call(void* user, int32_t b0, int32_t b1, const double* f2, const double* vpair) {
            try {
                static_cast<Sink*>(user)->take(b0, b1, f2, vpair);
                return 0;
            } catch (...) {
                return 1;  // the library stops and reports STP_RUNTIME_ERROR
            }
        }
    };

    // OutputTier::HostRam: the runs land in the caller's F2BlockTensor.
    struct HostSink final : Sink {
        F2BlockTensor& t;
        std::size_t slab;
        HostSink(F2BlockTensor& dst, int P, int n_block) : t(dst), slab(static_cast<std::size_t>(P) * P) {
            t.P = P;
            t.n_block = n_block;
            t.f2.assign(t.size(), 0.0);
            t.vpair.assign(t.size(), 0.0);
        }
        void take(int b0, int b1, const double* f2, const double* vpair) override {
            const std::size_t n = slab * static_cast<std::size_t>(b1 - b0);
            std::memcpy(t.f2.data() + slab * b0, f2, n * sizeof(double));
            std::memcpy(t.vpair.data() + slab * b0, vpair, n * sizeof(double));
        }
        void finish(const std::vector<int32_t>& sizes, device::StreamTarget&) override {
            t.block_sizes.assign(sizes.begin(), sizes.end());
        }
    };

    // OutputTier::Disk: an STPF2BK1 file (src/device/f2_disk_format.hpp:17-47) written run
    // by run at the blocks' offsets, then described in the DiskF2Blocks the caller reads.
    struct DiskSink final : Sink {
        std::string path;
        device::F2DiskHeader h{};
        std::FILE* f = nullptr;
        DiskSink(const std::string& p, int P, int n_block) : path(p) {
            std::memcpy(h.magic, device::kF2DiskMagic, sizeof(h.magic));
            h.version = device::kF2DiskVersion;
            h.dtype = device::kF2DiskDtypeFp64;
            h.P = P;
            h.n_block = n_block;
            const std::uint64_t bytes = static_cast<std::uint64_t>(P) * P * static_cast<std::uint64_t>(n_block) * 8;
            h.f2_offset = device::kF2DiskHeaderSize;
            h.vpair_offset = h.f2_offset + bytes;
            h.block_sizes_offset = h.vpair_offset + bytes;
            f = std::fopen(path.c_str(), "wb+");
            if (!f || std::fwrite(&h, sizeof(h), 1, f) != 1)
                throw std::runtime_error("compute_f2_blocks_streamed: cannot write " + path);
        }
        ~DiskSink() override {
            if (f) std::fclose(f);
        }
        void put(std::uint64_t off, const double* src, std::size_t n) {
            if (std::fseek(f, static_cast<long>(off), SEEK_SET) != 0 || std::fwrite(src, sizeof(double), n, f) != n)
                throw std::runtime_error("compute_f2_blocks_streamed: write to " + path + " failed");
        }
        void take(int b0, int b1, const double* f2, const double* vpair) override {
            const std::size_t n = static_cast<std::size_t>(h.P) * h.P * static_cast<std::size_t>(b1 - b0);
            put(device::f2_block_offset(h, b0), f2, n);
            put(device::vpair_block_offset(h, b0), vpair, n);
        }
        void finish(const std::vector<int32_t>& sizes, device::StreamTarget& target) override {
            if (std::fseek(f, static_cast<long>(h.block_sizes_offset), SEEK_SET) != 0 ||
                std::fwrite(sizes.data(), sizeof(int32_t), sizes.size(), f) != sizes.size())
                throw std::runtime_error("compute_f2_blocks_streamed: write to " + path + " failed");
            std::fclose(f);
            f = nullptr;
            device::DiskF2Blocks& d = *target.disk_dst;
            d.path = path;
            d.P = h.P;
            d.n_block = h.n_block;
            d.block_sizes.assign(sizes.begin(), sizes.end());
            d.read_handle.reset(std::fopen(path.c_str(), "rb"));
        }
    };

    // The RedecodeSource form: the canonical tile as SNP-major records on the device, then
    // the streamed extraction over the kept rows, read in place (no dense Q / V / N).
    void streamed_from_tile(const device::RedecodeSource& rd, const int* block_id, int n_block, const Precision& prec,
                            Sink& sink, int32_t* sizes) {
        static_assert(sizeof(long) == sizeof(int64_t), "kept_to_raw is read as int64");
        const DecodeTileView& v = *rd.base_view;
        const int64_t n_ind = static_cast<int64_t>(v.n_individuals), n_snp = static_cast<int64_t>(v.n_snp);
        const uint64_t pitch = (static_cast<uint64_t>(n_ind + 3) / 4 + 15) / 16 * 16;
        device::DeviceBuffer<std::uint8_t> rec(static_cast<std::size_t>(pitch) * static_cast<std::size_t>(n_snp));
        check(stp_canonical_to_records(ctx_, v.packed, v.bytes_per_record, n_snp, n_ind, v.packed_on_device, rec.data(),
                                       pitch));
        std::vector<int64_t> sel(static_cast<std::size_t>(n_ind));
        for (int64_t g = 0; g < n_ind; ++g) sel[static_cast<std::size_t>(g)] = g;
        const std::vector<int64_t> po = offsets64(v.pop_offsets, v.n_pop);
        stp_f2_request r{};
        r.geno = stp_geno_view{rec.data(), static_cast<uint64_t>(n_ind + 3) / 4, pitch, n_snp, n_ind, 1};
        r.sel_rows = sel.data();
        r.pop_offsets = po.data();
        r.n_pop = v.n_pop;
        r.sample_ploidy = v.sample_ploidy;
        r.ploidy_mode = v.detect_ploidy_on_device ? STP_PLOIDY_AUTO
                        : v.ploidy == 1               ? STP_PLOIDY_PSEUDO
                                                      : STP_PLOIDY_DIPLOID;
        r.block_id = block_id;
        r.n_block = n_block;
        r.precision = mode(prec);
        r.kept_rows = reinterpret_cast<const int64_t*>(rd.kept_to_raw);
        r.n_kept = rd.M_kept;
        check(stp_f2_extract_streamed(ctx_, &r, &Sink::call, &sink, sizes));
    }

    static stp_snp_filter filter_of(const FilterConfig& cfg, double maxmiss) {
        stp_snp_filter f{};
        f.maf_min = cfg.maf_min;
        f.maxmiss = maxmiss;
        f.autosomes_only = cfg.autosomes_only ? 1 : 0;
        f.drop_monomorphic = cfg.drop_monomorphic ? 1 : 0;
        f.transversions_only = cfg.transversions_only ? 1 : 0;
        f.strand_mode = cfg.strand_mode == StrandMode::Drop   ? STP_STRAND_DROP
                        : cfg.strand_mode == StrandMode::Keep ? STP_STRAND_KEEP
                                                              : STP_STRAND_FLIP;
        return f;
    }

    int32_t mode(const Precision& p) const { return precision_mode(p, accept_fixed_point_); }

    stp_ctx* ctx_ = nullptr;
    int device_ = 0;
    bool accept_fixed_point_ = false;
};

// Declared next to make_cuda_backend (src/device/backend_factory.hpp:18-21).
std::unique_ptr<ComputeBackend> make_b200_backend(int device, bool accept_fixed_point = false) {
    return std::make_unique<B200Backend>(device, accept_fixed_point);
}

}  // namespace steppe
