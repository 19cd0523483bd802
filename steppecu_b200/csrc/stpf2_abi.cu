// steppecu_b200/csrc/stpf2_abi.cu
//
// The C ABI of libstpf2.so (include/stpf2.h): contexts, plans, and the entry points that
// stand in for the reference's ComputeBackend f2/decode virtuals (src/device/backend.hpp
// :673-765) and its extract-f2 hot path (src/app/extract_f2_core.cpp:93-407). Host code
// only: it validates arguments, builds the block layout and work lists, moves data and
// launches the kernels in decode.cu, f2_simt.cu, f2_umma.cu and jackknife.cu. There is
// no CPU fallback: without a CUDA device every entry point returns STP_NO_DEVICE.
#include <algorithm>
#include <thread>
#include <exception>
#include <atomic>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "stpf2_internal.cuh"

struct stp_ctx : stpf2::Ctx {};

namespace stpf2 {

int simt_tile();

namespace {

thread_local std::string g_last_error;

template <class F>
stp_status guarded(F&& f) {
    try {
        f();
        return STP_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        g_last_error = "host out of memory";
        return STP_RUNTIME_ERROR;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return STP_RUNTIME_ERROR;
    }
}

void need(bool ok, const char* what) {
    if (!ok) fail(STP_INVALID_ARGUMENT, what);
}

void use_device(const Ctx& c) { STPF2_CUDA(cudaSetDevice(c.device)); }

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

template <class T>
void upload(DevBuf& b, const std::vector<T>& h, cudaStream_t s) {
    b.reserve(std::max<size_t>(h.size() * sizeof(T), 16));
    if (!h.empty())
        STPF2_CUDA(cudaMemcpyAsync(b.ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

}  // namespace

// ---- layout ---------------------------------------------------------------------------

BlockLayout make_block_layout(const int32_t* block_id, int64_t n_snp, int n_block, bool with_snp_col) {
    BlockLayout L;
    L.n_block = n_block;
    L.n_snp = n_snp;
    std::vector<int64_t> beg(static_cast<size_t>(n_block), 0), end(static_cast<size_t>(n_block), 0);
    int prev = -1;
    for (int64_t s = 0; s < n_snp;) {
        const int b = block_id[s];
        if (b < 0 || b >= n_block)
            fail(STP_RUNTIME_ERROR, "block_id[" + std::to_string(s) + "] = " + std::to_string(b) +
                                        " is out of range [0, " + std::to_string(n_block) + ")");
        if (b < prev)
            fail(STP_RUNTIME_ERROR, "block_id is not non-decreasing at column " + std::to_string(s) +
                                        "; the partition is not contiguous");
        int64_t e = s;
        while (e < n_snp && block_id[e] == b) ++e;
        beg[b] = s;
        end[b] = e;
        prev = b;
        s = e;
    }
    L.blocks.resize(static_cast<size_t>(n_block));
    L.snp_begin = beg;
    int64_t col = 0;
    for (int b = 0; b < n_block; ++b) {
        const int64_t k = end[b] - beg[b];
        if (k > INT_MAX) fail(STP_RUNTIME_ERROR, "block larger than INT_MAX SNPs");
        L.blocks[b] = BlockInfo{col, static_cast<int32_t>(k), b};
        col += (k + kColAlign - 1) / kColAlign * kColAlign;
    }
    L.ld = std::max<int64_t>(col, kColAlign);
    if (L.ld > INT_MAX)
        fail(STP_RUNTIME_ERROR, "padded SNP axis exceeds INT_MAX columns (M > INT_MAX)");
    if (!with_snp_col) return L;
    L.snp_col.resize(static_cast<size_t>(n_snp));
    for (int64_t s = 0; s < n_snp; ++s) {
        const int b = block_id[s];
        L.snp_col[s] = static_cast<int32_t>(L.blocks[b].col + (s - beg[b]));
    }
    return L;
}

std::vector<WorkItem> make_work_items(const BlockLayout& L, int P, int tile) {
    const int T = (P + tile - 1) / tile;
    std::vector<WorkItem> items;
    items.reserve(static_cast<size_t>(L.n_block) * T * (T + 1) / 2);
    for (int b = 0; b < L.n_block; ++b)
        for (int ti = 0; ti < T; ++ti)
            for (int tj = ti; tj < T; ++tj) items.push_back(WorkItem{b, static_cast<int16_t>(ti), static_cast<int16_t>(tj)});
    std::stable_sort(items.begin(), items.end(), [&](const WorkItem& a, const WorkItem& b) {
        return L.blocks[a.blk].k > L.blocks[b.blk].k;
    });
    return items;
}

std::vector<int32_t> make_vpair_units(const std::vector<WorkItem>& items) {
    std::vector<int32_t> u;
    u.reserve(items.size());
    for (size_t k = 0; k < items.size(); ++k) {
        u.push_back(static_cast<int32_t>(k));
        if (k + 1 < items.size() && vpair_pairs_with(items[k], items[k + 1])) ++k;
    }
    return u;
}

size_t operand_plane_bytes(OpFmt f, int P, int64_t ld) {
    if (f == OpFmt::F32) {
        const size_t pl = static_cast<size_t>(P) * static_cast<size_t>(ld);
        return align256(2 * pl * 4) + align256(pl);
    }
    const size_t tiles = static_cast<size_t>((P + kTileRows - 1) / kTileRows) * static_cast<size_t>(ld / kTileK);
    if (f == OpFmt::FX) return align256(tiles * (kFxImageBytes + kTile8Bytes));  // images, then the M tiles
    return align256(tiles * kImageBytes);
}

void bind_operand_planes(OperandPlanes& op, OpFmt f, int P, int64_t ld, void* base) {
    op.fmt = f;
    op.P = P;
    op.ld = ld;
    op.planes = base;
    op.scale_inv = (f == OpFmt::F16) ? 1.0 / double(1 << (2 * kF16PtShift)) : 1.0;
    if (f == OpFmt::F32) {
        const size_t pl = static_cast<size_t>(P) * static_cast<size_t>(ld);
        op.m_u8 = static_cast<uint8_t*>(base) + align256(2 * pl * 4);
        op.n_rt = 0;
        op.n_ck = 0;
    } else {
        op.n_rt = (P + kTileRows - 1) / kTileRows;
        op.n_ck = ld / kTileK;
        op.m_u8 = nullptr;  // the int8 M tiles live inside the operand images (FX: after them)
        op.mplanes = f == OpFmt::FX ? static_cast<uint8_t*>(base) + static_cast<size_t>(op.n_rt) * op.n_ck * kFxImageBytes
                                    : nullptr;
    }
}

// ---- plan ------------------------------------------------------------------------------

struct Plan {
    Ctx* ctx = nullptr;
    int P = 0;
    int64_t n_sel = 0, n_snp = 0;  // n_snp: the request's SNP axis (the kept SNPs with kept_rows)
    int64_t n_rec = 0;             // genotype records (the ploidy window and record copies span these)
    uint64_t pitch = 0;
    int precision = 0;
    bool detect = false;
    BlockLayout L;
    DevBuf sel, pop_off, pos, tiles, col_snp, rec_n, rec_nm1, canon, center, blocks, items, own_planes, repitched;
    DevBuf fold_order;  // per 64-population group, local indices largest first (null: all equal)
    DevBuf fx_table;    // FX: the term table of every (n, a2) (OperandPlanes::fx_table)
    DevBuf row_map;     // kept SNP -> record row (empty: SNP s is record s)
    std::vector<int64_t> kept;  // the same on the host (segment uploads of host records)
    uint64_t* canon_ptr = nullptr;  // canon's storage, or a context workspace (one-shot calls)
    double* center_ptr = nullptr;
    int64_t n_ind = 0, n_tiles = 0, n_sel_pad = 0;
    int n_items = 0;
    bool repitch = false;
    uint64_t src_pitch = 0, bpr = 0;
    OperandPlanes op;
    UmmaPlan* umma = nullptr;
    // Timing: three events per run (start, after decode, after contraction), one set per
    // run since timing was (re-)enabled, so a timed region of many runs is averaged.
    bool timing = false;
    std::vector<std::array<cudaEvent_t, 3>> ev;
    size_t n_timed = 0;
    // One executable graph of the whole pass, instantiated for one (records, f2, vpair).
    cudaGraphExec_t graph = nullptr;
    const void* graph_key[3] = {nullptr, nullptr, nullptr};
    bool per_block = false;  // comparison form: one contraction launch per block

    ~Plan() {
        if (graph) cudaGraphExecDestroy(graph);
        if (umma) umma_plan_destroy(umma);
        for (auto& t : ev)
            for (auto e : t)
                if (e) cudaEventDestroy(e);
    }

    int launches() const {
        int contract = (per_block && umma) ? static_cast<int>(L.blocks.size()) : 1;
        if (precision == STP_PREC_FIXED_I8) contract *= 2;  // the vpair kernel, then the f2 kernel
        return (detect ? 1 : 0) + 2 + contract;
    }
};

namespace {

// Validates a request and builds its plan. planes_base != nullptr borrows operand
// storage (at least operand_plane_bytes) instead of allocating it; borrow_ws takes the
// canonical genotypes and centres from the context's grow-only workspace as well (for
// one-shot calls, which finish before the next call on the context starts).
// The request's SNP axis: its kept SNPs when it names them, else every record.
int64_t snp_axis(const stp_f2_request& r) { return r.kept_rows ? r.n_kept : r.geno.n_snp; }

std::unique_ptr<Plan> build_plan(Ctx& c, const stp_f2_request& r, uint64_t pitch, void* planes_base,
                                 bool borrow_ws = false, bool counts_only = false) {
    need(r.n_pop >= 0 && r.geno.n_snp >= 0 && r.n_block >= 0, "negative extent");
    need(r.geno.bytes_per_record > 0 || r.geno.n_snp == 0, "bytes_per_record is 0");
    need(r.pop_offsets != nullptr || r.n_pop == 0, "pop_offsets is NULL");
    auto p = std::make_unique<Plan>();
    p->ctx = &c;
    p->P = r.n_pop;
    p->n_rec = r.geno.n_snp;
    p->n_snp = snp_axis(r);
    if (r.kept_rows && p->n_snp > 0) {
        need(p->n_snp < INT_MAX, "too many kept SNPs");
        p->kept.assign(r.kept_rows, r.kept_rows + p->n_snp);
        for (int64_t k = 0; k < p->n_snp; ++k) {
            need(p->kept[k] >= 0 && p->kept[k] < r.geno.n_snp, "kept_rows entry outside [0, n_snp)");
            need(k == 0 || p->kept[k] > p->kept[k - 1], "kept_rows must be strictly increasing");
        }
        std::vector<int32_t> rm(p->kept.begin(), p->kept.end());
        upload(p->row_map, rm, c.stream);
    }
    p->pitch = pitch;
    p->precision = r.precision;
    const OpFmt fmt = fmt_of(r.precision);
    const int64_t n_sel = r.n_pop > 0 ? r.pop_offsets[r.n_pop] : 0;
    p->n_sel = n_sel;
    need(r.n_pop == 0 || r.pop_offsets[0] == 0, "pop_offsets[0] must be 0");
    for (int i = 0; i < r.n_pop; ++i)
        need(r.pop_offsets[i + 1] >= r.pop_offsets[i], "pop_offsets must be non-decreasing");
    need(n_sel == 0 || r.sel_rows != nullptr, "sel_rows is NULL");
    need(n_sel < INT_MAX, "too many selected samples");
    need(r.block_id != nullptr || p->n_snp == 0, "block_id is NULL");

    cudaStream_t s = c.stream;
    std::vector<uint32_t> sel(static_cast<size_t>(n_sel));
    const bool auto_ploidy = r.sample_ploidy == nullptr && r.ploidy_mode == STP_PLOIDY_AUTO;
    for (int64_t g = 0; g < n_sel; ++g) {
        const int64_t row = r.sel_rows[g];
        need(row >= 0 && row < r.geno.n_ind, "sel_rows entry outside [0, n_ind)");
        need(static_cast<uint64_t>(row / 4) < r.geno.bytes_per_record, "sel_rows entry beyond the record");
        int pl = 0;
        if (r.sample_ploidy) pl = r.sample_ploidy[g];
        else if (r.ploidy_mode == STP_PLOIDY_PSEUDO) pl = 1;
        else if (r.ploidy_mode == STP_PLOIDY_DIPLOID) pl = 2;
        else need(auto_ploidy, "unknown ploidy_mode");
        if (pl != 1 && pl != 2) pl = 0;  // a bad ploidy contributes nothing (decode_af.hpp:58-65)
        sel[g] = pack_sel(row, pl);
    }
    p->detect = auto_ploidy;
    upload(p->sel, sel, s);

    std::vector<int32_t> po(static_cast<size_t>(r.n_pop) + 1, 0);
    int64_t max_pop = 0;
    for (int i = 0; i <= r.n_pop && r.n_pop > 0; ++i) po[i] = static_cast<int32_t>(r.pop_offsets[i]);
    for (int i = 0; i < r.n_pop; ++i) max_pop = std::max<int64_t>(max_pop, r.pop_offsets[i + 1] - r.pop_offsets[i]);
    need(max_pop <= 16383, "a population has more than 16383 samples");
    upload(p->pop_off, po, s);
    // The decode's fold order: within each group of 64 populations, largest first. Only
    // when sizes differ (equal sizes keep the natural order and no table).
    {
        bool uneven = false;
        for (int i = 1; i < r.n_pop && !uneven; ++i)
            uneven = (po[i + 1] - po[i]) != (po[1] - po[0]);
        if (uneven) {
            const int groups = (r.n_pop + 63) / 64;
            std::vector<int32_t> order(static_cast<size_t>(groups) * 64);
            for (int gidx = 0; gidx < groups; ++gidx) {
                int32_t* o = order.data() + 64 * gidx;
                for (int k = 0; k < 64; ++k) o[k] = k;
                auto size_of = [&](int k) {
                    const int i = 64 * gidx + k;
                    return i < r.n_pop ? po[i + 1] - po[i] : -1;
                };
                std::stable_sort(o, o + 64, [&](int32_t x, int32_t y) { return size_of(x) > size_of(y); });
            }
            upload(p->fold_order, order, s);
        }
    }

    // File row -> selected index (each row may be selected once).
    p->n_ind = r.geno.n_ind;
    std::vector<int32_t> pos(static_cast<size_t>(std::max<int64_t>(r.geno.n_ind, 0)), -1);
    for (int64_t g = 0; g < n_sel; ++g) {
        int32_t& slot = pos[static_cast<size_t>(r.sel_rows[g])];
        need(slot < 0, "a sample is selected more than once");
        slot = static_cast<int32_t>(g);
    }
    upload(p->pos, pos, s);

    // 1/n and 1/max(n-1, 1) for every called-allele count a population can reach.
    const int64_t n_max = 2 * max_pop + 1;
    std::vector<double> rn(static_cast<size_t>(n_max) + 1, 0.0), rnm1(static_cast<size_t>(n_max) + 1, 1.0);
    for (int64_t n = 1; n <= n_max; ++n) {
        rn[n] = 1.0 / static_cast<double>(n);
        rnm1[n] = 1.0 / std::max(static_cast<double>(n) - 1.0, 1.0);
    }
    upload(p->rec_n, rn, s);
    upload(p->rec_nm1, rnm1, s);

    p->L = make_block_layout(r.block_id, p->n_snp, r.n_block);
    // 32-column tiles of the padded column space (blocks start on 64-column boundaries,
    // so a tile never spans two blocks).
    p->n_tiles = p->L.ld / 32;
    std::vector<TileInfo> tiles(static_cast<size_t>(p->n_tiles), TileInfo{0, 0});
    std::vector<int32_t> col_snp(static_cast<size_t>(p->L.ld), -1);
    for (int b = 0; b < p->L.n_block; ++b) {
        const BlockInfo& bi = p->L.blocks[b];
        for (int64_t off = 0; off < (bi.k + 31) / 32 * 32; off += 32) {
            TileInfo& ti = tiles[static_cast<size_t>((bi.col + off) / 32)];
            ti.snp0 = static_cast<int32_t>(p->L.snp_begin[b] + off);
            ti.nvalid = static_cast<int32_t>(std::min<int64_t>(32, bi.k - off));
        }
        for (int64_t k = 0; k < bi.k; ++k) col_snp[static_cast<size_t>(bi.col + k)] = static_cast<int32_t>(p->L.snp_begin[b] + k);
    }
    upload(p->tiles, tiles, s);
    upload(p->col_snp, col_snp, s);
    p->n_sel_pad = (n_sel + 3) / 4 * 4;
    {
        const size_t canon_bytes = std::max<size_t>(static_cast<size_t>((p->n_tiles + 3) / 4) * p->n_sel_pad * 32, 64);
        const size_t center_bytes = std::max<size_t>(static_cast<size_t>(p->L.ld) * 8, 64);
        DevBuf& cb = borrow_ws ? c.ws_canon : p->canon;
        DevBuf& eb = borrow_ws ? c.ws_center : p->center;
        cb.reserve(canon_bytes);
        eb.reserve(center_bytes);
        p->canon_ptr = cb.as<uint64_t>();
        p->center_ptr = eb.as<double>();
    }

    // The transpose reads records with 4-byte (16-byte when aligned so) copies: records of
    // a pitch that is not a multiple of 4 are copied once per run into a 16-byte pitch.
    p->bpr = r.geno.bytes_per_record;
    p->src_pitch = pitch;
    const uint64_t need_bytes = static_cast<uint64_t>((r.geno.n_ind + 63) / 64) * 16;
    p->repitch = (pitch % 4 != 0) || pitch < static_cast<uint64_t>((r.geno.n_ind + 3) / 4) ||
                 (r.geno.on_device && reinterpret_cast<uintptr_t>(r.geno.records) % 4 != 0);
    if (p->repitch) {
        p->pitch = (std::max<uint64_t>(r.geno.bytes_per_record, need_bytes) + 15) / 16 * 16;
        p->repitched.reserve(std::max<size_t>(static_cast<size_t>(p->pitch) * p->n_rec, 64));
    }
    upload(p->blocks, p->L.blocks, s);
    if (counts_only) return p;  // decode to counts only: no operand planes, no contraction

    const size_t ob = operand_plane_bytes(fmt, std::max(r.n_pop, 1), p->L.ld);
    if (!planes_base) {
        p->own_planes.reserve(ob);
        planes_base = p->own_planes.ptr;
    }
    // Padding columns must read as zero; decode only ever writes real SNP columns. A plan
    // cached on the context relies on that for the shared planes workspace, so building
    // another plan there drops it.
    if (planes_base == c.ws_misc.ptr) c.plan_cache.reset();
    STPF2_CUDA(cudaMemsetAsync(planes_base, 0, ob, s));
    bind_operand_planes(p->op, fmt, r.n_pop, p->L.ld, planes_base);
    if (fmt == OpFmt::FX && fx_table_entries(n_max) > 0) {
        p->fx_table.reserve(static_cast<size_t>(fx_table_entries(n_max)) * sizeof(uint2));
        launch_fx_table(c, p->rec_n.as<double>(), p->rec_nm1.as<double>(), n_max, p->fx_table.as<uint2>(), s);
        p->op.fx_table = p->fx_table.as<uint2>();
        p->op.fx_table_ld = static_cast<int32_t>(2 * n_max + 1);
    }

    if (r.precision == STP_PREC_FP32_SIMT) {
        const std::vector<WorkItem> items = make_work_items(p->L, r.n_pop, simt_tile());
        p->n_items = static_cast<int>(items.size());
        upload(p->items, items, s);
    } else if (r.n_pop > 0 && r.n_block > 0) {
        p->umma = umma_plan_create(c, p->op, p->L, chunk_stages_of(r.precision));
    }
    return p;
}

// Ploidy (when detected) -> transpose to canonical tiles -> per-population decode into the
// operand planes (and, for tests, the integer counts).
// Tiles [t0, t1) only (t1 < 0: to the end): a tile range whose canonical quads and
// centres are indexed from t0, for the pipelined host-buffer path; detect runs the ploidy
// pass first (it reads the first min(1000, M) SNPs).
void launch_decode(Plan& p, const uint8_t* d_records, int32_t* cnt_ac2, int32_t* cnt_n, cudaStream_t s,
                   int64_t t0 = 0, int64_t t1 = -1, bool detect = true, uint32_t* cnt_packed = nullptr) {
    Ctx& c = *p.ctx;
    if (p.n_snp <= 0) return;
    if (t1 < 0) t1 = p.n_tiles;
    const uint8_t* rec = d_records;
    if (p.repitch) {
        STPF2_CUDA(cudaMemcpy2DAsync(p.repitched.ptr, p.pitch, d_records, p.src_pitch, p.bpr,
                                     static_cast<size_t>(p.n_rec), cudaMemcpyDeviceToDevice, s));
        rec = p.repitched.as<uint8_t>();
    }
    if (p.detect && detect)
        launch_detect_ploidy_words(c, rec, p.pitch, p.n_rec, p.n_ind, p.pos.as<int32_t>(), p.sel.as<uint32_t>(), s);
    if (t1 <= t0) return;
    launch_transpose_pa(c, rec, p.pitch, p.n_ind, p.tiles.as<TileInfo>() + t0, t1 - t0, p.pos.as<int32_t>(),
                        p.n_sel_pad, p.canon_ptr, p.center_ptr + t0 * kTileK, s, p.row_map.as<int32_t>());
    CanonDecodeArgs a;
    a.canon = p.canon_ptr;
    a.n_tiles = t1 - t0;
    a.n_sel = p.n_sel_pad;
    a.sel = p.sel.as<uint32_t>();
    a.pop_off = p.pop_off.as<int32_t>();
    a.P = p.P;
    a.center = p.center_ptr + t0 * kTileK;
    a.rec_n = p.rec_n.as<double>();
    a.rec_nm1 = p.rec_nm1.as<double>();
    a.col_snp = p.col_snp.as<int32_t>() + t0 * kTileK;
    a.col_base = t0 * kTileK;
    a.op = p.op;
    if (cnt_ac2) a.op.planes = nullptr;
    a.cnt_ac2 = cnt_ac2;
    a.cnt_n = cnt_n;
    if (cnt_packed) {
        a.op.planes = nullptr;
        a.cnt_packed = cnt_packed;
        a.cnt_ld = p.n_snp;
    }
    a.fold_order = p.fold_order.as<int32_t>();
    launch_decode_canon(c, a, s);
}

void run_plan(Plan& p, const uint8_t* d_records, double* d_f2, double* d_vpair, cudaStream_t s) {
    Ctx& c = *p.ctx;
    const size_t out_elems = static_cast<size_t>(p.P) * p.P * p.L.n_block;
    if (p.P <= 0 || p.L.n_block <= 0) return;
    if (p.n_snp <= 0) {  // no SNPs: every block is empty -> zeros (cpu_backend.cpp:234)
        STPF2_CUDA(cudaMemsetAsync(d_f2, 0, out_elems * sizeof(double), s));
        STPF2_CUDA(cudaMemsetAsync(d_vpair, 0, out_elems * sizeof(double), s));
        return;
    }
    std::array<cudaEvent_t, 3>* tev = nullptr;
    if (p.timing) {
        if (p.n_timed == p.ev.size()) {
            std::array<cudaEvent_t, 3> t{};
            for (auto& e : t) STPF2_CUDA(cudaEventCreate(&e));
            p.ev.push_back(t);
        }
        tev = &p.ev[p.n_timed++];
        STPF2_CUDA(cudaEventRecord((*tev)[0], s));
    }
    launch_decode(p, d_records, nullptr, nullptr, s);
    if (tev) STPF2_CUDA(cudaEventRecord((*tev)[1], s));
    if (p.precision == STP_PREC_FP32_SIMT)
        launch_f2_simt(c, p.items.as<WorkItem>(), p.n_items, p.blocks.as<BlockInfo>(), p.op, d_f2, d_vpair, s);
    else
        launch_f2_umma(c, p.umma, d_f2, d_vpair, s, p.per_block);
    if (tev) STPF2_CUDA(cudaEventRecord((*tev)[2], s));
}

void copy_block_sizes(const BlockLayout& L, int32_t* out) {
    for (int b = 0; b < L.n_block; ++b) out[b] = L.blocks[b].k;
}

// Device pitch for host records: their own pitch when the transpose can read it (a
// multiple of 4 bytes), so the upload is one contiguous copy; else rounded up to 16.
uint64_t device_pitch(const stp_geno_view& g) {
    const uint64_t hp = g.pitch ? g.pitch : g.bytes_per_record;
    return hp % 4 == 0 ? hp : (g.bytes_per_record + 15) / 16 * 16;
}

// Copies record rows [s0, s0 + n) from the host into d (pitch dp) on stream st: one
// contiguous copy when the pitches agree (the last row only up to bytes_per_record, which
// is all a host buffer is sure to hold), else a pitched copy.
void upload_rows(const stp_geno_view& g, uint8_t* d, uint64_t dp, int64_t s0, int64_t n, cudaStream_t st) {
    if (n <= 0) return;
    const uint64_t hp = g.pitch ? g.pitch : g.bytes_per_record;
    if (hp == dp) {
        const size_t bytes = static_cast<size_t>(n - 1) * hp + g.bytes_per_record;
        STPF2_CUDA(cudaMemcpyAsync(d + s0 * static_cast<int64_t>(dp), g.records + s0 * static_cast<int64_t>(hp), bytes,
                                   cudaMemcpyHostToDevice, st));
    } else {
        STPF2_CUDA(cudaMemcpy2DAsync(d + s0 * static_cast<int64_t>(dp), dp, g.records + s0 * static_cast<int64_t>(hp), hp,
                                     g.bytes_per_record, static_cast<size_t>(n), cudaMemcpyHostToDevice, st));
    }
}

// Runs f(i) for i in [0, n) on up to hardware_concurrency threads; rethrows the first error.
template <class F>
void parallel_for(int n, F&& f) {
    const int nt = std::max(1, std::min<int>(n, static_cast<int>(std::thread::hardware_concurrency())));
    std::atomic<int> next{0};
    std::vector<std::exception_ptr> errs(static_cast<size_t>(nt));
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            try {
                for (int i = next++; i < n; i = next++) f(i);
            } catch (...) {
                errs[t] = std::current_exception();
            }
        });
    for (auto& x : th) x.join();
    for (auto& e : errs)
        if (e) std::rethrow_exception(e);
}

// Copies the upper tiles (row tile <= column tile, the diagonal tiles whole) of slabs
// [0, nb) of a device slab run into the host run: per column tile, one 3-D copy of rows
// [0, c0 + T) x columns [c0, c0 + T) x every slab. Element (i, j) is at i + P * j, so each
// column of a copy is one contiguous run of c0 + T doubles. The column tiles alternate
// between two streams: runs this short keep one copy engine at ~30 GB/s, two run together.
void download_upper_tiles(double* host, const double* dev, int64_t P, int64_t T, int64_t nb, cudaStream_t st0,
                          cudaStream_t st1) {
    for (int64_t c0 = 0; c0 < P; c0 += T) {
        const cudaStream_t st = ((c0 / T) & 1) ? st1 : st0;
        const int64_t nr = std::min(P, c0 + T), nc = std::min(T, P - c0);
        cudaMemcpy3DParms m{};
        m.srcPtr = make_cudaPitchedPtr(const_cast<double*>(dev), static_cast<size_t>(P) * sizeof(double),
                                       static_cast<size_t>(P) * sizeof(double), static_cast<size_t>(P));
        m.dstPtr = make_cudaPitchedPtr(host, static_cast<size_t>(P) * sizeof(double),
                                       static_cast<size_t>(P) * sizeof(double), static_cast<size_t>(P));
        m.srcPos = make_cudaPos(0, static_cast<size_t>(c0), 0);
        m.dstPos = m.srcPos;
        m.extent = make_cudaExtent(static_cast<size_t>(nr) * sizeof(double), static_cast<size_t>(nc),
                                   static_cast<size_t>(nb));
        m.kind = cudaMemcpyDeviceToHost;
        STPF2_CUDA(cudaMemcpy3DAsync(&m, st));
    }
}

// Fork of independent launches from stream s onto the context's side streams, round robin,
// and their join back into s (events; destruction joins too, so an error path leaves no
// side-stream work unordered after s).
struct SideFork {
    Ctx& c;
    cudaStream_t s;
    cudaEvent_t ev[Ctx::kSideStreams + 1] = {};
    int k = 0;
    bool joined = false;
    SideFork(Ctx& c_, cudaStream_t s_) : c(c_), s(s_) {
        for (auto& e : ev) STPF2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        STPF2_CUDA(cudaEventRecord(ev[0], s));
        for (cudaStream_t x : c.side) STPF2_CUDA(cudaStreamWaitEvent(x, ev[0], 0));
    }
    cudaStream_t next() { return c.side[k++ % Ctx::kSideStreams]; }
    void join() {
        if (joined) return;
        joined = true;
        for (int i = 0; i < Ctx::kSideStreams; ++i) {
            STPF2_CUDA(cudaEventRecord(ev[i + 1], c.side[i]));
            STPF2_CUDA(cudaStreamWaitEvent(s, ev[i + 1], 0));
        }
    }
    ~SideFork() {
        if (!joined) {
            joined = true;
            for (int i = 0; i < Ctx::kSideStreams; ++i) {
                cudaEventRecord(ev[i + 1], c.side[i]);
                cudaStreamWaitEvent(s, ev[i + 1], 0);
            }
        }
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    }
};

// On an error, copies between the device and the caller's buffers may still be in flight:
// drains the context's streams before the error reaches the caller (who may free them).
struct DrainOnError {
    Ctx& c;
    ~DrainOnError() {
        if (std::uncaught_exceptions() == 0) return;
        cudaStreamSynchronize(c.h2d);
        cudaStreamSynchronize(c.stream);
        cudaStreamSynchronize(c.d2h);
        for (cudaStream_t x : c.side) cudaStreamSynchronize(x);
    }
};

// Host buffers in and out, tensor-core arithmetic: the pass runs in segments of whole
// blocks (about a twelfth of the SNPs each, the first covering the ploidy window) so the
// upload of segment k+1, the decode and contraction of segment k and the download of
// segment k-1's f2 / vpair slabs overlap on three streams. A segment's records are a
// contiguous run of SNP rows, its operand columns a tile range, its output a contiguous
// run of block slabs. The device holds only two segments' slabs (a ring: segment k's
// contraction waits for the download of segment k-2 from the same buffer), so the output
// tensor itself may exceed device memory (the out-of-core tier: only the host holds all
// P x P x B slabs).
// Segments of whole blocks: bounds[k]..bounds[k+1] are segment k's blocks. Most hold about
// a twelfth of the SNPs; the first two and the last two ramp (1/48, 1/24 of the SNPs), so
// the first download starts soon after the call and the host's work on the last segment
// is short. The first segment covers at least the ploidy window.
std::vector<int> segment_bounds(const BlockLayout& L) {
    const int B = L.n_block;
    const int64_t M = L.n_snp;
    const int64_t window = std::min<int64_t>(M, 1000);
    const int64_t full = std::max<int64_t>((M + 11) / 12, window);
    const int64_t ramp[2] = {std::max<int64_t>((M + 47) / 48, window), std::max<int64_t>((M + 23) / 24, window)};
    // The tail: the last blocks, walked backwards, into segments of 1/48 and 1/24.
    std::vector<int> tail;  // first block of each tail segment, last segment first
    {
        int64_t acc = 0;
        int t = 0;
        for (int b = B - 1; b > 0 && t < 2; --b) {
            acc += L.blocks[b].k;
            if (acc >= ramp[t]) {
                tail.push_back(b);
                acc = 0;
                ++t;
            }
        }
    }
    const int tail_begin = tail.empty() ? B : tail.back();
    std::vector<int> bounds{0};
    int64_t acc = 0;
    int seg = 0;
    for (int b = 0; b < tail_begin; ++b) {
        acc += L.blocks[b].k;
        const int64_t target = seg < 2 ? ramp[seg] : full;
        if (acc >= target && b + 1 < tail_begin) {
            bounds.push_back(b + 1);
            acc = 0;
            ++seg;
        }
    }
    // The first segment must still reach the ploidy window when the head is all there is.
    for (auto it = tail.rbegin(); it != tail.rend(); ++it)
        if (*it > bounds.back()) bounds.push_back(*it);
    bounds.push_back(B);
    // The ploidy window: merge leading segments until the first spans it.
    int64_t first = 0;
    size_t merge = 1;
    for (; merge + 1 < bounds.size(); ++merge) {
        for (int b = bounds[merge - 1]; b < bounds[merge]; ++b) first += L.blocks[b].k;
        if (first >= window) break;
    }
    if (merge > 1) bounds.erase(bounds.begin() + 1, bounds.begin() + static_cast<long>(merge));
    return bounds;
}

// Where the host side of a segmented pass puts each segment's slabs: straight into the
// caller's F2BlockTensor (f2, vpair), or into a two-segment pinned staging ring handed to
// a callback once the segment is complete (the streamed tiers: the caller keeps or writes
// the slabs, and no whole tensor needs to exist anywhere).
struct SlabTarget {
    double* f2 = nullptr;
    double* vpair = nullptr;
    stp_slab_sink sink = nullptr;
    void* user = nullptr;
};

// The segmented contraction pass with host output. before(k) enqueues what segment k needs
// on the context stream before its contraction (uploads, decode); the contraction of
// segment k goes into a two-segment device ring (it waits for the downloads of segment
// k - 2 from the same buffers). Every slab is exactly symmetric (the contraction stores one
// value at (i, j) and (j, i)), so only its upper 128 x 128 tiles cross PCIe: f2's in place
// (one 3-D copy per column tile), vpair's as packed 16-bit counts (counts_pack.cu). Once a
// segment has landed, host threads fill each f2 slab's lower tiles by transposition and
// widen its counts into both halves of the vpair slab (host_expand.cpp). With a sink, at
// most two segments are in flight and each is handed over before its staging slot is
// reused.
template <class Before>
void contract_segments(Ctx& c, UmmaPlan* up, int P, const BlockLayout& L, const std::vector<int>& bounds,
                       const SlabTarget& t, Before&& before) {
    const size_t slab = static_cast<size_t>(P) * static_cast<size_t>(P);
    const size_t nseg = bounds.size() - 1;
    size_t ring = 1;  // slabs per ring buffer: the largest segment
    for (size_t k = 0; k < nseg; ++k) ring = std::max<size_t>(ring, static_cast<size_t>(bounds[k + 1] - bounds[k]));
    int32_t kmax = 0;
    for (const BlockInfo& b : L.blocks) kmax = std::max(kmax, b.k);
    const bool wide = kmax > 65535;  // counts past 16 bits: 32-bit packing
    const size_t cnt_slab = packed_counts_bytes(P, 1, wide);
    c.ws_f2.reserve(2 * ring * slab * sizeof(double));
    c.ws_vpair.reserve(2 * ring * slab * sizeof(double));
    c.ws_counts.reserve(2 * ring * cnt_slab);
    if (t.sink) {
        c.pin_stage.reserve(4 * ring * slab * sizeof(double));
        c.pin_counts.reserve(2 * ring * cnt_slab);
    } else {
        c.pin_counts.reserve(static_cast<size_t>(L.n_block) * cnt_slab);
    }
    std::vector<cudaEvent_t> ev(2 * nseg, nullptr);  // per segment: contracted and packed, downloaded
    std::vector<cudaEvent_t> ev2(nseg, nullptr);     // per segment: the second copy queue done
    struct Free {
        std::vector<cudaEvent_t>& ev;
        ~Free() {
            for (auto e : ev)
                if (e) cudaEventDestroy(e);
        }
    } free_events{ev}, free_events2{ev2};
    for (auto& e : ev) STPF2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : ev2) STPF2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    auto host_f2 = [&](size_t k) {
        return t.sink ? c.pin_stage.as<double>() + (k % 2) * ring * slab : t.f2 + slab * bounds[k];
    };
    auto host_vp = [&](size_t k) {
        return t.sink ? c.pin_stage.as<double>() + (2 + k % 2) * ring * slab : t.vpair + slab * bounds[k];
    };
    auto host_cnt = [&](size_t k) {
        return c.pin_counts.as<uint8_t>() + (t.sink ? (k % 2) * ring : static_cast<size_t>(bounds[k])) * cnt_slab;
    };
    auto enqueue = [&](size_t k) {
        const int b0 = bounds[k], b1 = bounds[k + 1];
        const size_t nb = static_cast<size_t>(b1 - b0);
        double* f2k = c.ws_f2.as<double>() + (k % 2) * ring * slab;
        double* vpk = c.ws_vpair.as<double>() + (k % 2) * ring * slab;
        uint8_t* cntk = c.ws_counts.as<uint8_t>() + (k % 2) * ring * cnt_slab;
        before(k);
        if (k >= 2) STPF2_CUDA(cudaStreamWaitEvent(c.stream, ev[2 * (k - 2) + 1], 0));  // ring buffers free
        launch_f2_umma_blocks(c, up, b0, b1, f2k, vpk, c.stream, true);
        launch_pack_counts(c, vpk, P, static_cast<int64_t>(nb), wide, cntk, c.stream);
        STPF2_CUDA(cudaEventRecord(ev[2 * k], c.stream));
        STPF2_CUDA(cudaStreamWaitEvent(c.d2h, ev[2 * k], 0));
        STPF2_CUDA(cudaStreamWaitEvent(c.side[0], ev[2 * k], 0));
        download_upper_tiles(host_f2(k), f2k, P, 128, static_cast<int64_t>(nb), c.d2h, c.side[0]);
        STPF2_CUDA(cudaMemcpyAsync(host_cnt(k), cntk, nb * cnt_slab, cudaMemcpyDeviceToHost, c.d2h));
        STPF2_CUDA(cudaEventRecord(ev2[k], c.side[0]));  // the second copy queue joins the first
        STPF2_CUDA(cudaStreamWaitEvent(c.d2h, ev2[k], 0));
        STPF2_CUDA(cudaEventRecord(ev[2 * k + 1], c.d2h));
    };
    const size_t depth = t.sink ? 2 : nseg;
    size_t queued = 0;
    for (size_t k = 0; k < nseg; ++k) {
        while (queued < nseg && queued < k + depth) enqueue(queued++);
        STPF2_CUDA(cudaEventSynchronize(ev[2 * k + 1]));
        const int nb = bounds[k + 1] - bounds[k];
        double* f2h = host_f2(k);
        double* vph = host_vp(k);
        const uint8_t* cnt = host_cnt(k);
        parallel_for(2 * nb, [&](int u) {
            if (u % 2 == 0) mirror_lower_tiles(f2h + slab * static_cast<size_t>(u / 2), P, 128);
            else expand_counts(cnt + (u / 2) * cnt_slab, wide, vph + slab * static_cast<size_t>(u / 2), P);
        });
        if (t.sink && t.sink(t.user, bounds[k], bounds[k + 1], f2h, vph) != 0)
            fail(STP_RUNTIME_ERROR, "the slab sink stopped the extraction");
    }
    STPF2_CUDA(cudaStreamSynchronize(c.d2h));
    STPF2_CUDA(cudaStreamSynchronize(c.stream));
}

// Genotype records in, host output: the pass runs in segments of whole blocks so the
// upload of segment k+1 (host records), the decode and contraction of segment k and the
// download of segment k-1's slabs overlap on three streams. A segment's records are a
// contiguous run of rows, its operand columns a tile range, its output a run of block
// slabs. The device holds only two segments' slabs, so the output tensor may exceed device
// memory (the out-of-core tiers: only the host, or the sink, sees all P x P x B slabs).
void run_pipelined(Ctx& c, const stp_f2_request& r, const SlabTarget& t, Plan& p, uint8_t* d_rec, uint64_t dp) {
    const BlockLayout& L = p.L;
    const int B = L.n_block;
    const std::vector<int> bounds = segment_bounds(L);
    const bool upload = !r.geno.on_device;
    std::vector<int64_t> snp0(bounds.size(), 0);
    for (size_t k = 0; k + 1 < bounds.size(); ++k) {
        int64_t nsnp = 0;
        for (int b = bounds[k]; b < bounds[k + 1]; ++b) nsnp += L.blocks[b].k;
        snp0[k + 1] = snp0[k] + nsnp;
    }
    std::vector<cudaEvent_t> up_ev(bounds.size() - 1, nullptr);
    struct Free {
        std::vector<cudaEvent_t>& ev;
        ~Free() {
            for (auto e : ev)
                if (e) cudaEventDestroy(e);
        }
    } free_events{up_ev};
    for (auto& e : up_ev) STPF2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    int64_t rec_end = 0;
    contract_segments(c, p.umma, p.P, L, bounds, t, [&](size_t k) {
        const int b0 = bounds[k], b1 = bounds[k + 1];
        const int64_t nsnp = snp0[k + 1] - snp0[k];
        if (upload) {
            // The records this segment reads: its SNPs' rows (a run of kept rows spans from
            // the first to the last), the first segment also the ploidy window; never a row
            // twice.
            int64_t r0 = snp0[k], r1 = snp0[k] + nsnp;
            if (!p.kept.empty() && nsnp > 0) {
                r0 = p.kept[static_cast<size_t>(snp0[k])];
                r1 = p.kept[static_cast<size_t>(snp0[k] + nsnp - 1)] + 1;
            }
            if (k == 0) {
                r0 = 0;
                r1 = std::max<int64_t>(r1, std::min<int64_t>(p.n_rec, 1000));
            }
            r0 = std::max(r0, rec_end);
            r1 = std::max(r1, r0);
            rec_end = r1;
            upload_rows(r.geno, d_rec, dp, r0, r1 - r0, c.h2d);
            STPF2_CUDA(cudaEventRecord(up_ev[k], c.h2d));
            STPF2_CUDA(cudaStreamWaitEvent(c.stream, up_ev[k], 0));
        }
        const int64_t t0 = L.blocks[b0].col / kTileK;
        const int64_t t1 = (b1 < B ? L.blocks[b1].col : L.ld) / kTileK;
        launch_decode(p, d_rec, nullptr, nullptr, c.stream, t0, t1, k == 0);
    });
}

// The plan of the last one-shot extraction, kept on the context with a copy of everything
// it was built from: a later call whose request is identical (same shapes, selection,
// ploidy, block ids and kept rows, compared element by element, and the same workspace
// the plan borrows) reuses its validated tables instead of building and uploading them
// again. The records are not part of the key: every pass re-detects ploidy and re-decodes.
struct PlanCache {
    std::unique_ptr<Plan> plan;
    int32_t n_pop = 0, n_block = 0, precision = 0, ploidy_mode = 0;
    int64_t n_snp = 0, n_ind = 0, n_kept = 0;
    uint64_t bpr = 0, pitch = 0;
    int32_t on_device = 0;
    std::vector<int64_t> sel_rows, pop_offsets, kept_rows;
    std::vector<int32_t> sample_ploidy, block_id;
    const void* ws[3] = {nullptr, nullptr, nullptr};

    template <class T>
    static bool same(const std::vector<T>& v, const T* a, size_t n) {
        if (a == nullptr) return v.empty() && n == 0;
        return v.size() == n && (n == 0 || std::memcmp(v.data(), a, n * sizeof(T)) == 0);
    }
    bool matches(const Ctx& c, const stp_f2_request& r, uint64_t dpitch) const {
        const int64_t n_sel = r.n_pop > 0 ? r.pop_offsets[r.n_pop] : 0;
        const size_t n_axis = static_cast<size_t>(r.kept_rows ? r.n_kept : r.geno.n_snp);
        return plan && r.n_pop == n_pop && r.n_block == n_block && r.precision == precision &&
               r.ploidy_mode == ploidy_mode && r.geno.n_snp == n_snp && r.geno.n_ind == n_ind &&
               r.n_kept == n_kept && r.geno.bytes_per_record == bpr && dpitch == pitch &&
               r.geno.on_device == on_device && ws[0] == c.ws_misc.ptr && ws[1] == c.ws_canon.ptr &&
               ws[2] == c.ws_center.ptr && n_sel >= 0 &&
               same(pop_offsets, r.pop_offsets, r.n_pop > 0 ? static_cast<size_t>(r.n_pop) + 1 : 0) &&
               same(sel_rows, r.sel_rows, static_cast<size_t>(n_sel)) &&
               same(sample_ploidy, r.sample_ploidy, r.sample_ploidy ? static_cast<size_t>(n_sel) : 0) &&
               same(kept_rows, r.kept_rows, r.kept_rows ? static_cast<size_t>(r.n_kept) : 0) &&
               same(block_id, r.block_id, n_axis);
    }
};

// The cached plan for this request, or null (the cache is emptied either way: a plan is
// owned by one call at a time).
std::unique_ptr<Plan> take_cached_plan(Ctx& c, const stp_f2_request& r, uint64_t dpitch) {
    auto pc = std::static_pointer_cast<PlanCache>(c.plan_cache);
    if (!pc || !pc->matches(c, r, dpitch)) return nullptr;
    return std::move(pc->plan);
}

// Keeps a plan that a call has finished with, keyed by the request it was built from.
void keep_plan(Ctx& c, const stp_f2_request& r, uint64_t dpitch, std::unique_ptr<Plan> p, bool hit) {
    auto pc = std::static_pointer_cast<PlanCache>(c.plan_cache);
    if (hit && pc) {  // the key is unchanged
        pc->plan = std::move(p);
        return;
    }
    pc = std::make_shared<PlanCache>();
    const int64_t n_sel = r.n_pop > 0 ? r.pop_offsets[r.n_pop] : 0;
    const size_t n_axis = static_cast<size_t>(r.kept_rows ? r.n_kept : r.geno.n_snp);
    pc->n_pop = r.n_pop;
    pc->n_block = r.n_block;
    pc->precision = r.precision;
    pc->ploidy_mode = r.ploidy_mode;
    pc->n_snp = r.geno.n_snp;
    pc->n_ind = r.geno.n_ind;
    pc->n_kept = r.n_kept;
    pc->bpr = r.geno.bytes_per_record;
    pc->pitch = dpitch;
    pc->on_device = r.geno.on_device;
    if (r.n_pop > 0) pc->pop_offsets.assign(r.pop_offsets, r.pop_offsets + r.n_pop + 1);
    if (n_sel > 0) pc->sel_rows.assign(r.sel_rows, r.sel_rows + n_sel);
    if (r.sample_ploidy && n_sel > 0) pc->sample_ploidy.assign(r.sample_ploidy, r.sample_ploidy + n_sel);
    if (r.kept_rows && r.n_kept > 0) pc->kept_rows.assign(r.kept_rows, r.kept_rows + r.n_kept);
    if (r.block_id && n_axis > 0) pc->block_id.assign(r.block_id, r.block_id + n_axis);
    pc->ws[0] = c.ws_misc.ptr;
    pc->ws[1] = c.ws_canon.ptr;
    pc->ws[2] = c.ws_center.ptr;
    pc->plan = std::move(p);
    c.plan_cache = pc;
}

void extract_one(Ctx& c, const stp_f2_request& r, stp_f2_output& o) {
    // The padded SNP axis is 32-bit: refuse M > INT_MAX before reading or allocating
    // anything (the reference throws std::runtime_error for it).
    if (r.geno.n_snp > INT_MAX) fail(STP_RUNTIME_ERROR, "n_snp exceeds INT_MAX (M > INT_MAX is not supported)");
    DrainOnError drain{c};
    need(o.f2 != nullptr || r.n_pop == 0 || r.n_block == 0, "output f2 is NULL");
    need(o.vpair != nullptr || r.n_pop == 0 || r.n_block == 0, "output vpair is NULL");
    cudaStream_t s = c.stream;
    const uint8_t* d_rec = r.geno.records;
    uint64_t pitch = r.geno.pitch ? r.geno.pitch : r.geno.bytes_per_record;
    need(pitch >= r.geno.bytes_per_record, "pitch < bytes_per_record");
    const bool host_in = !r.geno.on_device && r.geno.n_snp > 0;
    const bool pipelined = host_in && !o.on_device && r.precision != STP_PREC_FP32_SIMT && r.n_pop > 0 &&
                           r.n_block >= 2;
    uint64_t dp = 0;
    if (host_in) {
        need(r.geno.records != nullptr, "records is NULL");
        dp = device_pitch(r.geno);
        c.ws_records.reserve(static_cast<size_t>(dp) * r.geno.n_snp);
        if (!pipelined) upload_rows(r.geno, c.ws_records.as<uint8_t>(), dp, 0, r.geno.n_snp, s);
        d_rec = c.ws_records.as<uint8_t>();
        pitch = dp;
    }
    // A repeated request reuses its plan (whose operand planes already sit in the
    // workspace); otherwise the operand planes borrow the context's grow-only workspace.
    std::unique_ptr<Plan> p = take_cached_plan(c, r, pitch);
    const bool hit = p != nullptr;
    if (!hit) {
        const BlockLayout probe = make_block_layout(r.block_id, snp_axis(r), r.n_block);
        c.ws_misc.reserve(operand_plane_bytes(fmt_of(r.precision), std::max(r.n_pop, 1), probe.ld));
        p = build_plan(c, r, pitch, c.ws_misc.ptr, true);
    }
    if (o.block_sizes) copy_block_sizes(p->L, o.block_sizes);
    const size_t out_elems = static_cast<size_t>(std::max(r.n_pop, 0)) * std::max(r.n_pop, 0) * std::max(r.n_block, 0);
    if (pipelined && p->umma && !p->repitch && out_elems) {
        STPF2_CUDA(cudaStreamSynchronize(s));  // the plan's tables are uploaded on s
        SlabTarget t;
        t.f2 = o.f2;
        t.vpair = o.vpair;
        run_pipelined(c, r, t, *p, c.ws_records.as<uint8_t>(), dp);
    } else {
        double* d_f2 = o.f2;
        double* d_vp = o.vpair;
        if (!o.on_device && out_elems) {
            c.ws_f2.reserve(out_elems * sizeof(double));
            c.ws_vpair.reserve(out_elems * sizeof(double));
            d_f2 = c.ws_f2.as<double>();
            d_vp = c.ws_vpair.as<double>();
        }
        if (pipelined) upload_rows(r.geno, c.ws_records.as<uint8_t>(), dp, 0, r.geno.n_snp, s);
        run_plan(*p, d_rec, d_f2, d_vp, s);
        if (!o.on_device && out_elems) {
            STPF2_CUDA(cudaMemcpyAsync(o.f2, d_f2, out_elems * sizeof(double), cudaMemcpyDeviceToHost, s));
            STPF2_CUDA(cudaMemcpyAsync(o.vpair, d_vp, out_elems * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
    }
    if (o.ploidy_out && p->n_sel > 0) {
        std::vector<uint32_t> sel(static_cast<size_t>(p->n_sel));
        STPF2_CUDA(cudaMemcpyAsync(sel.data(), p->sel.ptr, sel.size() * 4, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaStreamSynchronize(s));
        for (size_t g = 0; g < sel.size(); ++g) o.ploidy_out[g] = static_cast<int32_t>(sel[g] & 3u);
    }
    STPF2_CUDA(cudaStreamSynchronize(s));
    umma_check(p->umma);
    keep_plan(c, r, pitch, std::move(p), hit);
}

// ---- grouped batch ----------------------------------------------------------------------

// Requests that read the same genotype panel, so a batch can share one upload, one ploidy
// pass and one canonical transpose.
bool same_panel(const stp_geno_view& a, const stp_geno_view& b) {
    return a.records == b.records && a.bytes_per_record == b.bytes_per_record && a.pitch == b.pitch &&
           a.n_snp == b.n_snp && a.n_ind == b.n_ind && a.on_device == b.on_device;
}

// One request of a grouped batch: what the host prepares (in parallel with the others)
// and the device tables it uploads. A population is identified by its samples and their
// ploidy (key: sorted row * 4 + ploidy code, code 3 = detect), so requests that select the
// same population share its decoded counts.
struct BatchMember {
    int k = 0;  // index of the request
    int P = 0;
    int64_t n_sel = 0;
    BlockLayout L;
    std::vector<std::vector<int64_t>> keys;  // per population
    std::vector<int32_t> plcode;             // per selected sample: 0/1/2, or 3 = detect
    std::vector<int32_t> upop;               // population -> batch population
    size_t img_bytes = 0, out_bytes = 0, vpc_bytes = 0;
    OperandPlanes op;
};

// Validates request r (the rules of build_plan) and fills m's host tables. Host only,
// safe to run for several members at once.
void prepare_member(const stp_f2_request& r, const stp_f2_output& o, int64_t n_ind, OpFmt fmt, BatchMember& m) {
    need(r.n_pop > 0 && r.n_block > 0, "empty request in a batch");
    need(r.pop_offsets != nullptr, "pop_offsets is NULL");
    need(r.pop_offsets[0] == 0, "pop_offsets[0] must be 0");
    for (int i = 0; i < r.n_pop; ++i) need(r.pop_offsets[i + 1] >= r.pop_offsets[i], "pop_offsets must be non-decreasing");
    const int64_t n_sel = r.pop_offsets[r.n_pop];
    need(n_sel == 0 || r.sel_rows != nullptr, "sel_rows is NULL");
    need(n_sel < INT_MAX, "too many selected samples");
    need(r.block_id != nullptr, "block_id is NULL");
    m.P = r.n_pop;
    m.n_sel = n_sel;
    const bool auto_ploidy = r.sample_ploidy == nullptr && r.ploidy_mode == STP_PLOIDY_AUTO;
    m.plcode.resize(static_cast<size_t>(n_sel));
    std::vector<char> seen(static_cast<size_t>(n_ind), 0);
    for (int64_t g = 0; g < n_sel; ++g) {
        const int64_t row = r.sel_rows[g];
        need(row >= 0 && row < n_ind, "sel_rows entry outside [0, n_ind)");
        need(static_cast<uint64_t>(row / 4) < r.geno.bytes_per_record, "sel_rows entry beyond the record");
        need(!seen[static_cast<size_t>(row)], "a sample is selected more than once");
        seen[static_cast<size_t>(row)] = 1;
        int pl = 3;
        if (r.sample_ploidy) pl = r.sample_ploidy[g];
        else if (r.ploidy_mode == STP_PLOIDY_PSEUDO) pl = 1;
        else if (r.ploidy_mode == STP_PLOIDY_DIPLOID) pl = 2;
        else need(auto_ploidy, "unknown ploidy_mode");
        if (!auto_ploidy && pl != 1 && pl != 2) pl = 0;  // a bad ploidy contributes nothing (decode_af.hpp:58-65)
        m.plcode[g] = pl;
    }
    m.keys.resize(static_cast<size_t>(r.n_pop));
    for (int i = 0; i < r.n_pop; ++i) {
        const int64_t g0 = r.pop_offsets[i], g1 = r.pop_offsets[i + 1];
        need(g1 - g0 <= 16383, "a population has more than 16383 samples");
        auto& key = m.keys[i];
        key.reserve(static_cast<size_t>(g1 - g0));
        for (int64_t g = g0; g < g1; ++g) key.push_back(r.sel_rows[g] * 4 + m.plcode[g]);
        std::sort(key.begin(), key.end());
    }
    m.L = make_block_layout(r.block_id, r.geno.n_snp, r.n_block, false);
    m.img_bytes = align256(operand_plane_bytes(fmt, r.n_pop, m.L.ld));
    if (fmt == OpFmt::FX) {  // the compact vpair tiles of the member's work items (context workspace)
        const int64_t T = (r.n_pop + kTileRows - 1) / kTileRows;
        m.vpc_bytes = fx_vpc_bytes(static_cast<int>(std::min<int64_t>(INT_MAX, r.n_block * T * (T + 1) / 2)));
    }
    const size_t elems = static_cast<size_t>(r.n_pop) * r.n_pop * r.n_block;
    m.out_bytes = o.on_device ? 0 : 2 * align256(elems * sizeof(double));
}


// A batch of requests over one panel, all on the tensor cores with one arithmetic:
//   1. the union of their samples goes through one ploidy pass and one transpose into
//      canonical genotypes in contiguous SNP tiles;
//   2. every distinct population of the batch is decoded once from that copy into packed
//      exact counts (ac2 | n << 16, population-major);
//   3. each request's operand images are emitted from its populations' counts through its
//      own block layout (column and tile maps built on the device), with the arithmetic of
//      the one-request decode, so results are bit-identical to it;
//   4. one persistent launch contracts every request's (block, tile pair) items.
// The requests' host tables are prepared in parallel while the device runs steps 1-2.
// Requests whose images do not fit in free device memory together run in consecutive
// waves of steps 3-4. The images are not cleared: step 3 writes every column of rows < P,
// and rows >= P of a request's last row tile only reach accumulator rows that are never
// stored. done_ms[m] receives request idx[m]'s completion time from the start of the group.
void extract_batch_grouped(Ctx& c, const stp_f2_request* reqs, stp_f2_output* outs, const std::vector<int>& idx,
                           std::vector<double>& done_ms) {
    DrainOnError drain{c};
    cudaStream_t s = c.stream;
    const stp_geno_view& g = reqs[idx[0]].geno;
    const int64_t M = g.n_snp, n_ind = g.n_ind;
    need(g.records != nullptr, "records is NULL");
    need(n_ind > 0, "n_ind must be positive");
    need(g.bytes_per_record > 0, "bytes_per_record is 0");
    need(M < INT_MAX, "too many SNPs");
    uint64_t pitch = g.pitch ? g.pitch : g.bytes_per_record;
    need(pitch >= g.bytes_per_record, "pitch < bytes_per_record");
    const int prec = reqs[idx[0]].precision;
    const OpFmt fmt = fmt_of(prec);

    // Records on the device at a pitch the transpose reads (a multiple of 4 bytes).
    const uint8_t* d_rec = g.records;
    DevBuf repitched;
    if (!g.on_device) {
        const uint64_t dp = device_pitch(g);
        c.ws_records.reserve(static_cast<size_t>(dp) * M);
        upload_rows(g, c.ws_records.as<uint8_t>(), dp, 0, M, s);
        d_rec = c.ws_records.as<uint8_t>();
        pitch = dp;
    } else if (pitch % 4 != 0 || pitch < static_cast<uint64_t>((n_ind + 3) / 4) ||
               reinterpret_cast<uintptr_t>(g.records) % 4 != 0) {
        const uint64_t need_bytes = static_cast<uint64_t>((n_ind + 63) / 64) * 16;
        const uint64_t dp = (std::max<uint64_t>(g.bytes_per_record, need_bytes) + 15) / 16 * 16;
        repitched.reserve(static_cast<size_t>(dp) * M);
        STPF2_CUDA(cudaMemcpy2DAsync(repitched.ptr, dp, g.records, pitch, g.bytes_per_record, static_cast<size_t>(M),
                                     cudaMemcpyDeviceToDevice, s));
        d_rec = repitched.as<uint8_t>();
        pitch = dp;
    }

    // The union of the selected samples, in file order.
    std::vector<int32_t> pos_u(static_cast<size_t>(n_ind), -1);
    bool any_auto = false;
    for (int k : idx) {
        const stp_f2_request& r = reqs[k];
        need(r.pop_offsets != nullptr, "pop_offsets is NULL");
        const int64_t n_sel = r.pop_offsets[r.n_pop];
        need(n_sel == 0 || r.sel_rows != nullptr, "sel_rows is NULL");
        for (int64_t q = 0; q < n_sel; ++q) {
            need(r.sel_rows[q] >= 0 && r.sel_rows[q] < n_ind, "sel_rows entry outside [0, n_ind)");
            pos_u[static_cast<size_t>(r.sel_rows[q])] = 0;
        }
        any_auto = any_auto || (r.sample_ploidy == nullptr && r.ploidy_mode == STP_PLOIDY_AUTO);
    }
    std::vector<uint32_t> desc_u;
    for (int64_t row = 0; row < n_ind; ++row)
        if (pos_u[static_cast<size_t>(row)] == 0) {
            pos_u[static_cast<size_t>(row)] = static_cast<int32_t>(desc_u.size());
            desc_u.push_back(pack_sel(row, 0));
        }
    const int64_t n_u = static_cast<int64_t>(desc_u.size());
    const int64_t n_u_pad = (n_u + 3) / 4 * 4;
    const int64_t n_utiles = (M + kTileK - 1) / kTileK;
    // The contiguous SNP layout of the shared copy (one block of every SNP), the union's
    // tables, its canonical genotypes and centres: one workspace, the host tables staged
    // through pinned memory in one upload.
    const BlockInfo one_block{0, static_cast<int32_t>(M), 0};
    const int64_t zero = 0;
    Packing pa;
    const size_t o_pos = pa.add(pos_u.size() * 4);
    const size_t o_desc = pa.add(desc_u.size() * 4);
    const size_t o_one = pa.add(sizeof(BlockInfo));
    const size_t o_zero = pa.add(sizeof(int64_t));
    const size_t staged_a = pa.end;
    const size_t o_tiles = pa.add(static_cast<size_t>(n_utiles) * sizeof(TileInfo));
    const size_t o_cols = pa.add(static_cast<size_t>(n_utiles) * kTileK * 4);
    const size_t o_canon = pa.add(static_cast<size_t>((n_utiles + 3) / 4) * n_u_pad * 32);
    const size_t o_center = pa.add(static_cast<size_t>(n_utiles) * kTileK * 8);
    const size_t o_t0 = pa.add(16);
    c.pin_union.reserve(staged_a);
    c.ws_union.reserve(pa.end);
    {
        uint8_t* h = c.pin_union.as<uint8_t>();
        std::memcpy(h + o_pos, pos_u.data(), pos_u.size() * 4);
        std::memcpy(h + o_desc, desc_u.data(), desc_u.size() * 4);
        std::memcpy(h + o_one, &one_block, sizeof(BlockInfo));
        std::memcpy(h + o_zero, &zero, sizeof(int64_t));
        STPF2_CUDA(cudaMemcpyAsync(c.ws_union.ptr, h, staged_a, cudaMemcpyHostToDevice, s));
    }
    uint8_t* U = c.ws_union.as<uint8_t>();
    auto* d_pos_u = reinterpret_cast<int32_t*>(U + o_pos);
    auto* d_desc_u = reinterpret_cast<uint32_t*>(U + o_desc);
    auto* d_tiles_u = reinterpret_cast<TileInfo*>(U + o_tiles);
    auto* d_cols_u = reinterpret_cast<int32_t*>(U + o_cols);
    auto* d_canon_u = reinterpret_cast<uint64_t*>(U + o_canon);
    auto* d_center_u = reinterpret_cast<double*>(U + o_center);
    auto* d_t0 = reinterpret_cast<unsigned long long*>(U + o_t0);

    launch_timestamp(c, d_t0, s);
    launch_layout_tables(c, reinterpret_cast<BlockInfo*>(U + o_one), reinterpret_cast<int64_t*>(U + o_zero), 1,
                         n_utiles * kTileK, d_cols_u, d_tiles_u, s);
    if (any_auto) launch_detect_ploidy_words(c, d_rec, pitch, M, n_ind, d_pos_u, d_desc_u, s);
    launch_transpose_pa(c, d_rec, pitch, n_ind, d_tiles_u, n_utiles, d_pos_u, n_u_pad, d_canon_u, d_center_u, s);

    // Host tables of every request, in parallel, while the device runs the shared passes.
    std::vector<BatchMember> mem(idx.size());
    parallel_for(static_cast<int>(idx.size()), [&](int m) {
        mem[m].k = idx[m];
        prepare_member(reqs[idx[m]], outs[idx[m]], n_ind, fmt, mem[m]);
    });

    // The batch's distinct populations, decoded once into packed counts.
    std::map<std::vector<int64_t>, int32_t> pop_index;
    std::vector<const std::vector<int64_t>*> pops;
    for (BatchMember& m : mem) {
        m.upop.resize(static_cast<size_t>(m.P));
        for (int i = 0; i < m.P; ++i) {
            auto it = pop_index.emplace(m.keys[i], static_cast<int32_t>(pops.size()));
            if (it.second) pops.push_back(&it.first->first);
            m.upop[i] = it.first->second;
        }
    }
    const int UP = static_cast<int>(pops.size());
    std::vector<uint32_t> sel_up;
    std::vector<int32_t> umap_up, off_up{0};
    int64_t max_pop = 0;
    for (const auto* key : pops) {
        for (int64_t e : *key) {
            sel_up.push_back(pack_sel(e >> 2, static_cast<int>(e & 3)));
            umap_up.push_back(pos_u[static_cast<size_t>(e >> 2)]);
        }
        off_up.push_back(static_cast<int32_t>(sel_up.size()));
        max_pop = std::max<int64_t>(max_pop, static_cast<int64_t>(key->size()));
    }
    const int64_t n_max = 2 * max_pop + 1;
    std::vector<double> rn(static_cast<size_t>(n_max) + 1, 0.0), rnm1(static_cast<size_t>(n_max) + 1, 1.0);
    for (int64_t n = 1; n <= n_max; ++n) {
        rn[n] = 1.0 / static_cast<double>(n);
        rnm1[n] = 1.0 / std::max(static_cast<double>(n) - 1.0, 1.0);
    }
    // The batch populations' tables and every request's tables (staged in one upload), then
    // the requests' device-built column and tile maps and the packed counts.
    Packing pb;
    const size_t o_sel = pb.add(sel_up.size() * 4);
    const size_t o_umap = pb.add(umap_up.size() * 4);
    const size_t o_off = pb.add(off_up.size() * 4);
    const size_t o_rn = pb.add(rn.size() * 8);
    const size_t o_rnm1 = pb.add(rn.size() * 8);
    struct MemberOffsets {
        size_t upop, blocks, begin, cols, tiles;
    };
    std::vector<MemberOffsets> mo(mem.size());
    for (size_t m = 0; m < mem.size(); ++m) {
        mo[m].upop = pb.add(mem[m].upop.size() * 4);
        mo[m].blocks = pb.add(mem[m].L.blocks.size() * sizeof(BlockInfo));
        mo[m].begin = pb.add(mem[m].L.snp_begin.size() * sizeof(int64_t));
    }
    const size_t staged_b = pb.end;
    for (size_t m = 0; m < mem.size(); ++m) {
        mo[m].cols = pb.add(static_cast<size_t>(mem[m].L.ld) * 4);
        mo[m].tiles = pb.add(static_cast<size_t>(mem[m].L.ld / kTileK) * sizeof(TileInfo));
    }
    // Rows of the union's counts, padded to a multiple of 4 words plus 4 (the emission reads
    // eight consecutive SNPs as three aligned 16-byte loads, up to 4 words past the last).
    const int64_t cnt_ld = (M + 3) / 4 * 4 + 4;
    const size_t o_counts = pb.add(static_cast<size_t>(UP) * static_cast<size_t>(cnt_ld) * 4);
    c.pin_tables.reserve(staged_b);
    c.ws_tables.reserve(pb.end);
    {
        uint8_t* h = c.pin_tables.as<uint8_t>();
        std::memcpy(h + o_sel, sel_up.data(), sel_up.size() * 4);
        std::memcpy(h + o_umap, umap_up.data(), umap_up.size() * 4);
        std::memcpy(h + o_off, off_up.data(), off_up.size() * 4);
        std::memcpy(h + o_rn, rn.data(), rn.size() * 8);
        std::memcpy(h + o_rnm1, rnm1.data(), rnm1.size() * 8);
        for (size_t m = 0; m < mem.size(); ++m) {
            std::memcpy(h + mo[m].upop, mem[m].upop.data(), mem[m].upop.size() * 4);
            std::memcpy(h + mo[m].blocks, mem[m].L.blocks.data(), mem[m].L.blocks.size() * sizeof(BlockInfo));
            std::memcpy(h + mo[m].begin, mem[m].L.snp_begin.data(), mem[m].L.snp_begin.size() * sizeof(int64_t));
        }
        STPF2_CUDA(cudaMemcpyAsync(c.ws_tables.ptr, h, staged_b, cudaMemcpyHostToDevice, s));
    }
    uint8_t* T = c.ws_tables.as<uint8_t>();
    auto* d_counts = reinterpret_cast<uint32_t*>(T + o_counts);
    auto* d_rn = reinterpret_cast<const double*>(T + o_rn);
    auto* d_rnm1 = reinterpret_cast<const double*>(T + o_rnm1);
    const uint2* d_fxtab = nullptr;
    if (fmt == OpFmt::FX && fx_table_entries(n_max) > 0) {
        c.ws_fxtab.reserve(static_cast<size_t>(fx_table_entries(n_max)) * sizeof(uint2));
        launch_fx_table(c, d_rn, d_rnm1, n_max, c.ws_fxtab.as<uint2>(), s);
        d_fxtab = c.ws_fxtab.as<uint2>();
    }
    if (any_auto)
        launch_copy_union_ploidy(c, reinterpret_cast<uint32_t*>(T + o_sel), reinterpret_cast<int32_t*>(T + o_umap),
                                 static_cast<int64_t>(sel_up.size()), d_desc_u, s);
    {
        CanonDecodeArgs a;
        a.canon = d_canon_u;
        a.n_tiles = n_utiles;
        a.n_sel = n_u_pad;
        a.sel = reinterpret_cast<const uint32_t*>(T + o_sel);
        a.pop_off = reinterpret_cast<const int32_t*>(T + o_off);
        a.P = UP;
        a.rec_n = d_rn;
        a.rec_nm1 = d_rnm1;
        a.col_snp = d_cols_u;
        a.op.fmt = fmt;
        a.op.planes = nullptr;  // counts only
        a.umap = reinterpret_cast<const int32_t*>(T + o_umap);
        a.center_snp = d_center_u;
        a.cnt_packed = d_counts;
        a.cnt_ld = cnt_ld;
        launch_decode_canon(c, a, s);
    }
    for (size_t m = 0; m < mem.size(); ++m)
        launch_layout_tables(c, reinterpret_cast<const BlockInfo*>(T + mo[m].blocks),
                             reinterpret_cast<const int64_t*>(T + mo[m].begin), mem[m].L.n_block, mem[m].L.ld,
                             reinterpret_cast<int32_t*>(T + mo[m].cols), reinterpret_cast<TileInfo*>(T + mo[m].tiles), s);

    // Waves of requests whose operand images (and device-side outputs) fit together.
    STPF2_CUDA(cudaStreamSynchronize(s));
    size_t free_b = 0, total_b = 0;
    STPF2_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t held = c.ws_batch.bytes + c.ws_f2.bytes + c.ws_vpair.bytes + c.ws_vpc.bytes;  // reusable here
    const size_t avail = free_b + held;
    const size_t budget = avail > (size_t(2) << 30) ? (avail - (size_t(2) << 30)) * 9 / 10 : 0;
    std::vector<std::vector<size_t>> waves(1);
    size_t acc = 0;
    for (size_t m = 0; m < mem.size(); ++m) {
        const size_t b = mem[m].img_bytes + mem[m].out_bytes + mem[m].vpc_bytes;
        if (!waves.back().empty() && acc + b > budget) {
            waves.emplace_back();
            acc = 0;
        }
        waves.back().push_back(m);
        acc += b;
    }
    std::vector<uint32_t> desc_h;  // detected ploidy of the union samples, for ploidy_out
    unsigned long long t0 = 0;
    for (const auto& wave : waves) {
        size_t img_total = 0, out_total = 0;
        for (size_t m : wave) {
            img_total += mem[m].img_bytes;
            out_total += mem[m].out_bytes / 2;
        }
        c.ws_batch.reserve(std::max<size_t>(img_total, 256));
        if (out_total) {
            c.ws_f2.reserve(out_total);
            c.ws_vpair.reserve(out_total);
        }
        std::vector<GroupSpec> specs(wave.size());
        size_t io = 0, oo = 0;
        // The emissions are independent (each writes its own request's images): they run on
        // the side streams, round robin, so one launch's tail overlaps the next; the
        // contraction waits for all of them.
        SideFork fork(c, s);
        for (size_t w = 0; w < wave.size(); ++w) {
            BatchMember& p = mem[wave[w]];
            const MemberOffsets& q = mo[wave[w]];
            const stp_f2_output& o = outs[p.k];
            bind_operand_planes(p.op, fmt, p.P, p.L.ld, c.ws_batch.as<uint8_t>() + io);
            p.op.fx_table = d_fxtab;
            p.op.fx_table_ld = static_cast<int32_t>(2 * n_max + 1);
            io += p.img_bytes;
            launch_emit_counts(c, d_counts, cnt_ld, M, reinterpret_cast<const int32_t*>(T + q.upop), p.P, p.L.ld / kTileK,
                               reinterpret_cast<const int32_t*>(T + q.cols), d_center_u, d_rn, d_rnm1, p.op,
                               fork.next());
            double* f2 = o.f2;
            double* vp = o.vpair;
            if (!o.on_device) {
                f2 = reinterpret_cast<double*>(c.ws_f2.as<uint8_t>() + oo);
                vp = reinterpret_cast<double*>(c.ws_vpair.as<uint8_t>() + oo);
                oo += p.out_bytes / 2;
            }
            specs[w].L = &p.L;
            specs[w].info = GroupInfo{static_cast<const uint8_t*>(p.op.planes), f2, vp, p.op.n_ck, p.P, 0, p.op.mplanes};
            if (o.block_sizes) copy_block_sizes(p.L, o.block_sizes);
        }
        fork.join();
        std::vector<unsigned long long> stamps;
        launch_f2_umma_grouped(c, fmt, mem[wave[0]].op.scale_inv, chunk_stages_of(prec), specs, s, &stamps);
        if (t0 == 0) STPF2_CUDA(cudaMemcpy(&t0, d_t0, sizeof(t0), cudaMemcpyDeviceToHost));
        for (size_t w = 0; w < wave.size(); ++w) {
            BatchMember& p = mem[wave[w]];
            done_ms[wave[w]] = stamps[w] >= t0 ? static_cast<double>(stamps[w] - t0) * 1e-6 : 0.0;
            const stp_f2_output& o = outs[p.k];
            const size_t elems = static_cast<size_t>(p.P) * p.P * p.L.n_block;
            if (!o.on_device && elems) {
                STPF2_CUDA(cudaMemcpyAsync(o.f2, specs[w].info.f2, elems * sizeof(double), cudaMemcpyDeviceToHost, s));
                STPF2_CUDA(cudaMemcpyAsync(o.vpair, specs[w].info.vpair, elems * sizeof(double), cudaMemcpyDeviceToHost, s));
            }
            if (o.ploidy_out && p.n_sel > 0) {
                if (desc_h.empty()) {
                    desc_h.resize(desc_u.size());
                    STPF2_CUDA(cudaMemcpyAsync(desc_h.data(), d_desc_u, desc_h.size() * 4, cudaMemcpyDeviceToHost, s));
                    STPF2_CUDA(cudaStreamSynchronize(s));
                }
                const stp_f2_request& r = reqs[p.k];
                for (int64_t q = 0; q < p.n_sel; ++q)
                    o.ploidy_out[q] = p.plcode[q] == 3
                                          ? static_cast<int32_t>(desc_h[static_cast<size_t>(pos_u[static_cast<size_t>(r.sel_rows[q])])] & 3u)
                                          : p.plcode[q];
            }
        }
        STPF2_CUDA(cudaStreamSynchronize(s));
    }
}

}  // namespace
}  // namespace stpf2

struct stp_plan {
    std::unique_ptr<stpf2::Plan> p;
};

using namespace stpf2;

extern "C" {

int stp_abi_version(void) { return STPF2_ABI_VERSION; }

const char* stp_last_error(void) { return g_last_error.c_str(); }

stp_ctx* stp_create(int device, stp_status* status) {
    stp_ctx* out = nullptr;
    const stp_status st = guarded([&] {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0)
            fail(STP_NO_DEVICE, "no CUDA device available (a CUDA-capable B200 is required)");
        need(device >= 0 && device < n, "device ordinal out of range");
        STPF2_CUDA(cudaSetDevice(device));
        int major = 0, minor = 0;
        STPF2_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
        STPF2_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
        if (major != 10 || minor != 0)
            fail(STP_NO_DEVICE, "libstpf2 is built for sm_100a (B200); device has sm_" +
                                    std::to_string(major) + std::to_string(minor));
        auto c = std::make_unique<stp_ctx>();
        c->device = device;
        STPF2_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
        STPF2_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        STPF2_CUDA(cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking));
        STPF2_CUDA(cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking));
        for (auto& x : c->side) STPF2_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
        out = c.release();
    });
    if (status) *status = st;
    return out;
}

void stp_destroy(stp_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (cudaStream_t s : {ctx->stream, ctx->h2d, ctx->d2h, ctx->side[0], ctx->side[1], ctx->side[2], ctx->side[3]}) {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
    delete ctx;
}

uint64_t stp_launch_count(const stp_ctx* ctx) { return ctx ? ctx->launches.load() : 0; }

stp_status stp_detect_ploidy(stp_ctx* ctx, const stp_geno_view* geno, const int64_t* sel_rows, int64_t n_sel,
                             int32_t* ploidy) {
    return guarded([&] {
        need(ctx && geno, "null argument");
        use_device(*ctx);
        if (n_sel <= 0) return;
        need(sel_rows && ploidy, "null argument");
        cudaStream_t s = ctx->stream;
        std::vector<uint32_t> sel(static_cast<size_t>(n_sel));
        for (int64_t g = 0; g < n_sel; ++g) {
            need(sel_rows[g] >= 0 && sel_rows[g] < geno->n_ind, "sel_rows entry outside [0, n_ind)");
            sel[g] = pack_sel(sel_rows[g], 0);
        }
        DevBuf d_sel, d_rec;
        upload(d_sel, sel, s);
        const uint8_t* rec = geno->records;
        uint64_t pitch = geno->pitch ? geno->pitch : geno->bytes_per_record;
        const int64_t window = std::min<int64_t>(geno->n_snp, 1000);
        if (!geno->on_device && window > 0) {
            d_rec.reserve(static_cast<size_t>(pitch) * window);
            STPF2_CUDA(cudaMemcpyAsync(d_rec.ptr, rec, static_cast<size_t>(pitch) * window, cudaMemcpyHostToDevice, s));
            rec = d_rec.as<uint8_t>();
        }
        launch_detect_ploidy_pa(*ctx, rec, pitch, geno->n_snp, d_sel.as<uint32_t>(), n_sel, s);
        STPF2_CUDA(cudaMemcpyAsync(sel.data(), d_sel.ptr, sel.size() * 4, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaStreamSynchronize(s));
        for (int64_t g = 0; g < n_sel; ++g) ploidy[g] = static_cast<int32_t>(sel[g] & 3u);
    });
}

stp_status stp_decode_counts(stp_ctx* ctx, const stp_geno_view* geno, const int64_t* sel_rows,
                             const int64_t* pop_offsets, int32_t n_pop, const int32_t* sample_ploidy,
                             int32_t ploidy_mode, int32_t* ac2, int32_t* n) {
    return guarded([&] {
        need(ctx && geno, "null argument");
        use_device(*ctx);
        if (n_pop <= 0 || geno->n_snp <= 0) return;
        need(ac2 && n, "null output");
        cudaStream_t s = ctx->stream;
        // One block spanning all SNPs: the counts do not depend on the block layout.
        std::vector<int32_t> bid(static_cast<size_t>(geno->n_snp), 0);
        stp_f2_request r{};
        r.geno = *geno;
        r.sel_rows = sel_rows;
        r.pop_offsets = pop_offsets;
        r.n_pop = n_pop;
        r.sample_ploidy = sample_ploidy;
        r.ploidy_mode = ploidy_mode;
        r.block_id = bid.data();
        r.n_block = 1;
        r.precision = STP_PREC_FP32_SIMT;
        const uint8_t* d_rec = geno->records;
        uint64_t pitch = geno->pitch ? geno->pitch : geno->bytes_per_record;
        DevBuf rec;
        if (!geno->on_device) {
            const uint64_t dp = device_pitch(*geno);
            rec.reserve(static_cast<size_t>(dp) * geno->n_snp);
            upload_rows(*geno, rec.as<uint8_t>(), dp, 0, geno->n_snp, s);
            d_rec = rec.as<uint8_t>();
            pitch = dp;
        }
        std::unique_ptr<Plan> p = build_plan(*ctx, r, pitch, nullptr);
        const size_t cnt = static_cast<size_t>(n_pop) * geno->n_snp;
        DevBuf d_ac2, d_n;
        d_ac2.reserve(cnt * 4);
        d_n.reserve(cnt * 4);
        launch_decode(*p, d_rec, d_ac2.as<int32_t>(), d_n.as<int32_t>(), s);
        STPF2_CUDA(cudaMemcpyAsync(ac2, d_ac2.ptr, cnt * 4, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaMemcpyAsync(n, d_n.ptr, cnt * 4, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaStreamSynchronize(s));
    });
}

namespace {

void check_filter(const stp_snp_filter* f) {
    need(f != nullptr, "filter is NULL");
    need(f->strand_mode >= STP_STRAND_DROP && f->strand_mode <= STP_STRAND_FLIP, "unknown strand_mode");
    need(f->maxmiss == f->maxmiss && f->maf_min == f->maf_min, "filter thresholds must not be NaN");
}

// The .snp columns the keep mask reads, on the device.
struct SnpColumns {
    DevBuf ref, alt, chrom;
    SnpColumns(const char* r, const char* a, const int32_t* c, int64_t M, cudaStream_t s) {
        need(r && a && c, "ref / alt / chrom is NULL");
        ref.reserve(static_cast<size_t>(M));
        alt.reserve(static_cast<size_t>(M));
        chrom.reserve(static_cast<size_t>(M) * 4);
        STPF2_CUDA(cudaMemcpyAsync(ref.ptr, r, static_cast<size_t>(M), cudaMemcpyHostToDevice, s));
        STPF2_CUDA(cudaMemcpyAsync(alt.ptr, a, static_cast<size_t>(M), cudaMemcpyHostToDevice, s));
        STPF2_CUDA(cudaMemcpyAsync(chrom.ptr, c, static_cast<size_t>(M) * 4, cudaMemcpyHostToDevice, s));
    }
};

}  // namespace

stp_status stp_snp_keep_mask(stp_ctx* ctx, const stp_geno_view* geno, const int64_t* sel_rows,
                             const int64_t* pop_offsets, int32_t n_pop, const int32_t* sample_ploidy,
                             int32_t ploidy_mode, const char* ref, const char* alt, const int32_t* chrom,
                             const stp_snp_filter* filter, uint8_t* keep, int64_t* n_kept, double* summary) {
    return guarded([&] {
        need(ctx && geno && n_kept, "null argument");
        use_device(*ctx);
        check_filter(filter);
        *n_kept = 0;
        const int64_t M = geno->n_snp;
        if (M <= 0) return;
        need(keep != nullptr, "keep is NULL");
        need(M <= INT_MAX, "n_snp exceeds INT_MAX (M > INT_MAX is not supported)");
        cudaStream_t s = ctx->stream;
        SnpColumns cols(ref, alt, chrom, M, s);
        DevBuf d_keep, d_sum;
        d_keep.reserve(static_cast<size_t>(M));
        if (summary) d_sum.reserve(static_cast<size_t>(M) * 4 * sizeof(double));
        if (n_pop > 0) {
            // Exact counts of every population at every SNP, population-major (one block over
            // all SNPs: counts do not depend on the block layout).
            std::vector<int32_t> bid(static_cast<size_t>(M), 0);
            stp_f2_request r{};
            r.geno = *geno;
            r.sel_rows = sel_rows;
            r.pop_offsets = pop_offsets;
            r.n_pop = n_pop;
            r.sample_ploidy = sample_ploidy;
            r.ploidy_mode = ploidy_mode;
            r.block_id = bid.data();
            r.n_block = 1;
            r.precision = STP_PREC_FP32_SIMT;
            const uint8_t* d_rec = geno->records;
            uint64_t pitch = geno->pitch ? geno->pitch : geno->bytes_per_record;
            DevBuf rec;
            if (!geno->on_device) {
                const uint64_t dp = device_pitch(*geno);
                rec.reserve(static_cast<size_t>(dp) * M);
                upload_rows(*geno, rec.as<uint8_t>(), dp, 0, M, s);
                d_rec = rec.as<uint8_t>();
                pitch = dp;
            }
            std::unique_ptr<Plan> p = build_plan(*ctx, r, pitch, nullptr, false, /*counts_only=*/true);
            DevBuf cnt;
            cnt.reserve(static_cast<size_t>(n_pop) * M * 4);
            launch_decode(*p, d_rec, nullptr, nullptr, s, 0, -1, true, cnt.as<uint32_t>());
            const double total = static_cast<double>(pop_offsets[n_pop]);
            launch_keep_mask_counts(*ctx, cnt.as<uint32_t>(), M, n_pop, M, cols.ref.as<char>(), cols.alt.as<char>(),
                                    cols.chrom.as<int32_t>(), *filter, total, d_keep.as<uint8_t>(),
                                    summary ? d_sum.as<double>() : nullptr, s);
            STPF2_CUDA(cudaMemcpyAsync(keep, d_keep.ptr, static_cast<size_t>(M), cudaMemcpyDeviceToHost, s));
            if (summary)
                STPF2_CUDA(cudaMemcpyAsync(summary, d_sum.ptr, static_cast<size_t>(M) * 4 * sizeof(double),
                                           cudaMemcpyDeviceToHost, s));
            STPF2_CUDA(cudaStreamSynchronize(s));
        } else {
            std::fill(keep, keep + M, uint8_t(0));
        }
        int64_t k = 0;
        for (int64_t i = 0; i < M; ++i) k += keep[i] ? 1 : 0;
        *n_kept = k;
    });
}

stp_status stp_canonical_to_records(stp_ctx* ctx, const uint8_t* packed, uint64_t bpr, int64_t n_snp, int64_t n_ind,
                                    int32_t packed_on_device, uint8_t* d_records, uint64_t pitch) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        use_device(*ctx);
        if (n_snp <= 0 || n_ind <= 0) return;
        need(packed && d_records, "null argument");
        need(bpr * 4 >= static_cast<uint64_t>(n_snp), "bytes_per_record too small for n_snp");
        need(pitch * 4 >= static_cast<uint64_t>(n_ind), "pitch too small for n_ind");
        cudaStream_t s = ctx->stream;
        DevBuf d_pk;
        const uint8_t* pk = packed;
        if (!packed_on_device) {
            d_pk.reserve(static_cast<size_t>(bpr) * n_ind);
            STPF2_CUDA(cudaMemcpyAsync(d_pk.ptr, packed, static_cast<size_t>(bpr) * n_ind, cudaMemcpyHostToDevice, s));
            pk = d_pk.as<uint8_t>();
        }
        launch_canonical_to_records(*ctx, pk, bpr, n_snp, n_ind, d_records, pitch, s);
        STPF2_CUDA(cudaStreamSynchronize(s));
    });
}

stp_status stp_decode_af_compact_filter(stp_ctx* ctx, const uint8_t* packed, uint64_t bpr, int64_t n_snp, int64_t n_ind,
                                        const int64_t* pop_offsets, int32_t n_pop, const int32_t* sample_ploidy,
                                        int32_t ploidy, int32_t packed_on_device, const char* ref, const char* alt,
                                        const int32_t* chrom, const stp_snp_filter* filter, double total_indiv,
                                        uint8_t* keep, int64_t* n_kept, double* q, double* v, double* n,
                                        int32_t out_on_device) {
    return guarded([&] {
        need(ctx != nullptr && n_kept != nullptr, "null argument");
        use_device(*ctx);
        check_filter(filter);
        *n_kept = 0;
        if (n_pop <= 0 || n_snp <= 0) return;
        need(keep && pop_offsets, "null argument");
        need(bpr * 4 >= static_cast<uint64_t>(n_snp), "bytes_per_record too small for n_snp");
        need(pop_offsets[n_pop] <= n_ind, "pop_offsets exceed n_individuals");
        need((q == nullptr) == (v == nullptr) && (q == nullptr) == (n == nullptr), "q, v, n: all or none");
        cudaStream_t s = ctx->stream;
        DevBuf d_pk, d_pl, d_po, d_q, d_v, d_n, d_keep;
        const uint8_t* pk = packed;
        if (!packed_on_device) {
            d_pk.reserve(static_cast<size_t>(bpr) * std::max<int64_t>(n_ind, 1));
            STPF2_CUDA(cudaMemcpyAsync(d_pk.ptr, packed, static_cast<size_t>(bpr) * n_ind, cudaMemcpyHostToDevice, s));
            pk = d_pk.as<uint8_t>();
        }
        d_pl.reserve(sizeof(int32_t) * std::max<int64_t>(n_ind, 1));
        if (sample_ploidy) {
            STPF2_CUDA(cudaMemcpyAsync(d_pl.ptr, sample_ploidy, sizeof(int32_t) * n_ind, cudaMemcpyHostToDevice, s));
        } else {
            std::vector<int32_t> pl(static_cast<size_t>(n_ind), ploidy);
            upload(d_pl, pl, s);
        }
        std::vector<int32_t> po(static_cast<size_t>(n_pop) + 1);
        for (int i = 0; i <= n_pop; ++i) po[i] = static_cast<int32_t>(pop_offsets[i]);
        upload(d_po, po, s);
        const size_t cnt = static_cast<size_t>(n_pop) * n_snp;
        d_q.reserve(cnt * 8);
        d_v.reserve(cnt * 8);
        d_n.reserve(cnt * 8);
        launch_decode_canonical(*ctx, pk, bpr, n_snp, n_ind, d_po.as<int32_t>(), n_pop, d_pl.as<int32_t>(),
                                d_q.as<double>(), d_v.as<double>(), d_n.as<double>(), s);
        SnpColumns cols(ref, alt, chrom, n_snp, s);
        d_keep.reserve(static_cast<size_t>(n_snp));
        launch_keep_mask_qn(*ctx, d_q.as<double>(), d_n.as<double>(), n_pop, n_snp, cols.ref.as<char>(),
                            cols.alt.as<char>(), cols.chrom.as<int32_t>(), *filter, total_indiv, d_keep.as<uint8_t>(),
                            nullptr, s);
        STPF2_CUDA(cudaMemcpyAsync(keep, d_keep.ptr, static_cast<size_t>(n_snp), cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaStreamSynchronize(s));
        std::vector<int64_t> dst(static_cast<size_t>(n_snp), -1);
        int64_t k = 0;
        for (int64_t i = 0; i < n_snp; ++i)
            if (keep[i]) dst[static_cast<size_t>(i)] = k++;
        *n_kept = k;
        if (!q || k == 0) return;
        DevBuf d_dst, o_q, o_v, o_n;
        upload(d_dst, dst, s);
        const size_t out = static_cast<size_t>(n_pop) * k;
        double* tq = q;
        double* tv = v;
        double* tn = n;
        if (!out_on_device) {
            o_q.reserve(out * 8);
            o_v.reserve(out * 8);
            o_n.reserve(out * 8);
            tq = o_q.as<double>();
            tv = o_v.as<double>();
            tn = o_n.as<double>();
        }
        launch_compact_columns(*ctx, d_q.as<double>(), n_pop, n_snp, d_dst.as<int64_t>(), tq, s);
        launch_compact_columns(*ctx, d_v.as<double>(), n_pop, n_snp, d_dst.as<int64_t>(), tv, s);
        launch_compact_columns(*ctx, d_n.as<double>(), n_pop, n_snp, d_dst.as<int64_t>(), tn, s);
        if (!out_on_device) {
            STPF2_CUDA(cudaMemcpyAsync(q, tq, out * 8, cudaMemcpyDeviceToHost, s));
            STPF2_CUDA(cudaMemcpyAsync(v, tv, out * 8, cudaMemcpyDeviceToHost, s));
            STPF2_CUDA(cudaMemcpyAsync(n, tn, out * 8, cudaMemcpyDeviceToHost, s));
        }
        STPF2_CUDA(cudaStreamSynchronize(s));
    });
}

stp_status stp_decode_counts_noalloc(stp_ctx* ctx, const stp_geno_view* geno, const int64_t* sel_rows,
                                     const int64_t* pop_offsets, int32_t n_pop, const int32_t* sample_ploidy,
                                     int32_t ploidy_mode, int32_t* d_ac2, int32_t* d_n, void* stream) {
    return guarded([&] {
        need(ctx && geno, "null argument");
        use_device(*ctx);
        if (n_pop <= 0 || geno->n_snp <= 0) return;
        need(geno->on_device != 0, "the no-alloc decode reads device-resident records (geno->on_device = 1)");
        need(geno->records && pop_offsets && d_ac2 && d_n, "null argument");
        const uint64_t pitch = geno->pitch ? geno->pitch : geno->bytes_per_record;
        need(pitch % 16 == 0 && reinterpret_cast<uintptr_t>(geno->records) % 16 == 0,
             "the no-alloc decode needs 16-byte aligned records and pitch (it cannot repitch without a buffer)");
        need(pitch >= geno->bytes_per_record, "pitch smaller than bytes_per_record");
        need(pop_offsets[0] == 0, "pop_offsets[0] must be 0");
        for (int i = 0; i < n_pop; ++i) {
            need(pop_offsets[i + 1] >= pop_offsets[i], "pop_offsets must be non-decreasing");
            need(pop_offsets[i + 1] - pop_offsets[i] <= 16383, "a population has more than 16383 samples");
        }
        const int64_t n_sel = pop_offsets[n_pop];
        need(n_sel == 0 || sel_rows != nullptr, "sel_rows is NULL");
        need(n_sel < INT_MAX, "too many selected samples");
        for (int64_t g = 0; g < n_sel; ++g) {
            need(sel_rows[g] >= 0 && sel_rows[g] < geno->n_ind, "sel_rows entry outside [0, n_ind)");
            need(static_cast<uint64_t>(sel_rows[g] / 4) < geno->bytes_per_record, "sel_rows entry beyond the record");
        }
        int mode_pl = 0;
        bool detect = false;
        if (!sample_ploidy) {
            if (ploidy_mode == STP_PLOIDY_AUTO) detect = true;
            else if (ploidy_mode == STP_PLOIDY_PSEUDO) mode_pl = 1;
            else if (ploidy_mode == STP_PLOIDY_DIPLOID) mode_pl = 2;
            else need(false, "unknown ploidy_mode");
        }
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
        noalloc_decode_counts(*ctx, geno->records, pitch, geno->n_snp, geno->n_ind, sel_rows, n_sel, pop_offsets,
                              n_pop, sample_ploidy, mode_pl, detect, d_ac2, d_n, s);
    });
}

stp_status stp_decode_af(stp_ctx* ctx, const uint8_t* packed, uint64_t bpr, int64_t n_snp, int64_t n_ind,
                         const int64_t* pop_offsets, int32_t n_pop, const int32_t* sample_ploidy, int32_t ploidy,
                         int32_t detect, int32_t packed_on_device, double* q, double* v, double* n) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        use_device(*ctx);
        if (n_pop <= 0 || n_snp <= 0) return;
        need(q && v && n && pop_offsets, "null argument");
        need(bpr * 4 >= static_cast<uint64_t>(n_snp), "bytes_per_record too small for n_snp");
        need(pop_offsets[n_pop] <= n_ind, "pop_offsets exceed n_individuals");
        cudaStream_t s = ctx->stream;
        DevBuf d_pk, d_pl, d_po, d_q, d_v, d_n;
        const uint8_t* pk = packed;
        if (!packed_on_device) {
            d_pk.reserve(static_cast<size_t>(bpr) * std::max<int64_t>(n_ind, 1));
            STPF2_CUDA(cudaMemcpyAsync(d_pk.ptr, packed, static_cast<size_t>(bpr) * n_ind, cudaMemcpyHostToDevice, s));
            pk = d_pk.as<uint8_t>();
        }
        d_pl.reserve(sizeof(int32_t) * std::max<int64_t>(n_ind, 1));
        if (sample_ploidy) {
            STPF2_CUDA(cudaMemcpyAsync(d_pl.ptr, sample_ploidy, sizeof(int32_t) * n_ind, cudaMemcpyHostToDevice, s));
        } else if (detect) {
            launch_detect_ploidy_canonical(*ctx, pk, bpr, n_snp, n_ind, d_pl.as<int32_t>(), s);
        } else {
            std::vector<int32_t> pl(static_cast<size_t>(n_ind), ploidy);
            upload(d_pl, pl, s);
        }
        std::vector<int32_t> po(static_cast<size_t>(n_pop) + 1);
        for (int i = 0; i <= n_pop; ++i) po[i] = static_cast<int32_t>(pop_offsets[i]);
        upload(d_po, po, s);
        const size_t cnt = static_cast<size_t>(n_pop) * n_snp;
        d_q.reserve(cnt * 8);
        d_v.reserve(cnt * 8);
        d_n.reserve(cnt * 8);
        launch_decode_canonical(*ctx, pk, bpr, n_snp, n_ind, d_po.as<int32_t>(), n_pop, d_pl.as<int32_t>(),
                                d_q.as<double>(), d_v.as<double>(), d_n.as<double>(), s);
        STPF2_CUDA(cudaMemcpyAsync(q, d_q.ptr, cnt * 8, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaMemcpyAsync(v, d_v.ptr, cnt * 8, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaMemcpyAsync(n, d_n.ptr, cnt * 8, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaStreamSynchronize(s));
    });
}

stp_status stp_detect_ploidy_tile(stp_ctx* ctx, const uint8_t* packed, uint64_t bpr, int64_t n_snp, int64_t n_ind,
                                  int32_t packed_on_device, int32_t* ploidy) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        use_device(*ctx);
        if (n_ind <= 0) return;
        need(ploidy != nullptr && packed != nullptr, "null argument");
        need(n_snp >= 0 && bpr * 4 >= static_cast<uint64_t>(n_snp), "bytes_per_record too small for n_snp");
        cudaStream_t s = ctx->stream;
        DevBuf d_pk, d_pl;
        const uint8_t* pk = packed;
        if (!packed_on_device) {
            d_pk.reserve(static_cast<size_t>(bpr) * static_cast<size_t>(n_ind));
            STPF2_CUDA(cudaMemcpyAsync(d_pk.ptr, packed, static_cast<size_t>(bpr) * n_ind, cudaMemcpyHostToDevice, s));
            pk = d_pk.as<uint8_t>();
        }
        d_pl.reserve(sizeof(int32_t) * static_cast<size_t>(n_ind));
        launch_detect_ploidy_canonical(*ctx, pk, bpr, n_snp, n_ind, d_pl.as<int32_t>(), s);
        STPF2_CUDA(cudaMemcpyAsync(ploidy, d_pl.ptr, sizeof(int32_t) * n_ind, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaStreamSynchronize(s));
    });
}

namespace {

// compute_f2_blocks over Q / V / N (host, or device when qvn_on_device): the feeder turns
// them into operand planes, then the contraction writes f2 / vpair into t.f2 / t.vpair
// (device buffers when out_on_device, host buffers otherwise) or, with t.sink, streams them
// in segments of blocks to the sink (tensor-core arithmetics only).
void f2_from_qvn(Ctx& c, const double* Q, const double* V, const double* N, int P, int64_t M, const int32_t* block_id,
                 int n_block, int precision, bool qvn_on_device, const SlabTarget& t, bool out_on_device,
                 int32_t* block_sizes) {
    need(P >= 0 && M >= 0 && n_block >= 0, "negative extent");
    need(M <= INT_MAX, "M exceeds INT_MAX (M > INT_MAX is not supported)");
    const size_t out_elems = static_cast<size_t>(P) * P * n_block;
    if (n_block > 0 && block_sizes) std::fill(block_sizes, block_sizes + n_block, 0);
    if (P <= 0 || n_block <= 0) return;
    cudaStream_t s = c.stream;
    const OpFmt fmt = fmt_of(precision);
    if (t.sink) need(fmt != OpFmt::F32, "streamed output needs a tensor-core precision");
    else need(t.f2 && t.vpair, "null output");
    if (M <= 0) {  // every block is empty: zeros (cpu_backend.cpp:234)
        if (t.sink) {
            std::vector<double> z(static_cast<size_t>(P) * P * n_block, 0.0);
            if (t.sink(t.user, 0, n_block, z.data(), z.data()) != 0) fail(STP_RUNTIME_ERROR, "the slab sink stopped the extraction");
        } else if (out_on_device) {
            STPF2_CUDA(cudaMemsetAsync(t.f2, 0, out_elems * 8, s));
            STPF2_CUDA(cudaMemsetAsync(t.vpair, 0, out_elems * 8, s));
            STPF2_CUDA(cudaStreamSynchronize(s));
        } else {
            std::fill(t.f2, t.f2 + out_elems, 0.0);
            std::fill(t.vpair, t.vpair + out_elems, 0.0);
        }
        return;
    }
    need(Q && V && N && block_id, "null input");
    DrainOnError drain{c};
    const BlockLayout L = make_block_layout(block_id, M, n_block);
    if (block_sizes) copy_block_sizes(L, block_sizes);
    DevBuf d_qvn, d_col, d_planes, d_blocks, d_items, d_f2, d_vp;
    const size_t pm = static_cast<size_t>(P) * M;
    const double *dq = Q, *dv = V, *dn = N;
    if (!qvn_on_device) {
        d_qvn.reserve(3 * pm * 8);
        double* h = d_qvn.as<double>();
        STPF2_CUDA(cudaMemcpyAsync(h, Q, pm * 8, cudaMemcpyHostToDevice, s));
        STPF2_CUDA(cudaMemcpyAsync(h + pm, V, pm * 8, cudaMemcpyHostToDevice, s));
        STPF2_CUDA(cudaMemcpyAsync(h + 2 * pm, N, pm * 8, cudaMemcpyHostToDevice, s));
        dq = h;
        dv = h + pm;
        dn = h + 2 * pm;
    }
    upload(d_col, L.snp_col, s);
    upload(d_blocks, L.blocks, s);
    const size_t ob = operand_plane_bytes(fmt, P, L.ld);
    d_planes.reserve(ob);
    STPF2_CUDA(cudaMemsetAsync(d_planes.ptr, 0, ob, s));
    OperandPlanes op;
    bind_operand_planes(op, fmt, P, L.ld, d_planes.ptr);
    launch_feed_qvn(c, dq, dv, dn, P, M, d_col.as<int32_t>(), op, s);
    if (precision == STP_PREC_FP32_SIMT) {
        double* f2 = t.f2;
        double* vp = t.vpair;
        if (!out_on_device) {
            d_f2.reserve(out_elems * 8);
            d_vp.reserve(out_elems * 8);
            f2 = d_f2.as<double>();
            vp = d_vp.as<double>();
        }
        const std::vector<WorkItem> items = make_work_items(L, P, simt_tile());
        upload(d_items, items, s);
        launch_f2_simt(c, d_items.as<WorkItem>(), static_cast<int>(items.size()), d_blocks.as<BlockInfo>(), op, f2, vp, s);
        if (!out_on_device) {
            STPF2_CUDA(cudaMemcpyAsync(t.f2, f2, out_elems * 8, cudaMemcpyDeviceToHost, s));
            STPF2_CUDA(cudaMemcpyAsync(t.vpair, vp, out_elems * 8, cudaMemcpyDeviceToHost, s));
        }
        STPF2_CUDA(cudaStreamSynchronize(s));
        return;
    }
    std::unique_ptr<UmmaPlan, void (*)(UmmaPlan*)> up(umma_plan_create(c, op, L, chunk_stages_of(precision)),
                                                       umma_plan_destroy);
    if (out_on_device) {
        launch_f2_umma(c, up.get(), t.f2, t.vpair, s);
    } else {
        // Host output, streamed or not: segments of blocks through the device ring.
        STPF2_CUDA(cudaStreamSynchronize(s));
        contract_segments(c, up.get(), P, L, segment_bounds(L), t, [](size_t) {});
    }
    STPF2_CUDA(cudaStreamSynchronize(s));
    umma_check(up.get());
}

}  // namespace

stp_status stp_f2_from_qvn(stp_ctx* ctx, const double* Q, const double* V, const double* N, int32_t P, int64_t M,
                           const int32_t* block_id, int32_t n_block, int32_t precision, double* f2,
                           double* vpair, int32_t* block_sizes) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        use_device(*ctx);
        SlabTarget t;
        t.f2 = f2;
        t.vpair = vpair;
        f2_from_qvn(*ctx, Q, V, N, P, M, block_id, n_block, precision, false, t, false, block_sizes);
    });
}

stp_status stp_f2_from_qvn_device(stp_ctx* ctx, const double* Q, const double* V, const double* N, int32_t P, int64_t M,
                                  const int32_t* block_id, int32_t n_block, int32_t precision, int32_t qvn_on_device,
                                  double* d_f2, double* d_vpair, int32_t* block_sizes) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        use_device(*ctx);
        SlabTarget t;
        t.f2 = d_f2;
        t.vpair = d_vpair;
        f2_from_qvn(*ctx, Q, V, N, P, M, block_id, n_block, precision, qvn_on_device != 0, t, true, block_sizes);
    });
}

stp_status stp_f2_from_qvn_streamed(stp_ctx* ctx, const double* Q, const double* V, const double* N, int32_t P,
                                    int64_t M, const int32_t* block_id, int32_t n_block, int32_t precision,
                                    stp_slab_sink sink, void* user, int32_t* block_sizes) {
    return guarded([&] {
        need(ctx != nullptr && sink != nullptr, "null argument");
        use_device(*ctx);
        SlabTarget t;
        t.sink = sink;
        t.user = user;
        f2_from_qvn(*ctx, Q, V, N, P, M, block_id, n_block, precision, false, t, false, block_sizes);
    });
}

stp_status stp_f2_extract_streamed(stp_ctx* ctx, const stp_f2_request* req, stp_slab_sink sink, void* user,
                                   int32_t* block_sizes) {
    return guarded([&] {
        need(ctx && req && sink, "null argument");
        use_device(*ctx);
        Ctx& c = *ctx;
        const stp_f2_request& r = *req;
        if (r.n_block > 0 && block_sizes) std::fill(block_sizes, block_sizes + r.n_block, 0);
        if (r.n_pop <= 0 || r.n_block <= 0) return;
        need(r.precision != STP_PREC_FP32_SIMT, "streamed output needs a tensor-core precision");
        if (r.geno.n_snp > INT_MAX) fail(STP_RUNTIME_ERROR, "n_snp exceeds INT_MAX (M > INT_MAX is not supported)");
        DrainOnError drain{c};
        uint64_t pitch = r.geno.pitch ? r.geno.pitch : r.geno.bytes_per_record;
        need(pitch >= r.geno.bytes_per_record, "pitch < bytes_per_record");
        need(r.geno.records != nullptr || r.geno.n_snp == 0, "records is NULL");
        uint8_t* d_rec = const_cast<uint8_t*>(r.geno.records);
        uint64_t dp = pitch;
        if (!r.geno.on_device && r.geno.n_snp > 0) {
            dp = device_pitch(r.geno);
            c.ws_records.reserve(static_cast<size_t>(dp) * r.geno.n_snp);
            d_rec = c.ws_records.as<uint8_t>();
        }
        {
            const BlockLayout probe = make_block_layout(r.block_id, snp_axis(r), r.n_block);
            c.ws_misc.reserve(operand_plane_bytes(fmt_of(r.precision), std::max(r.n_pop, 1), probe.ld));
        }
        std::unique_ptr<Plan> p = build_plan(c, r, dp, c.ws_misc.ptr, true);
        need(!p->repitch, "streamed extraction of device records needs a 4-byte aligned pitch");
        if (block_sizes) copy_block_sizes(p->L, block_sizes);
        STPF2_CUDA(cudaStreamSynchronize(c.stream));
        SlabTarget t;
        t.sink = sink;
        t.user = user;
        if (p->n_snp <= 0) {  // no SNPs: every block is empty -> zeros (cpu_backend.cpp:234)
            std::vector<double> z(static_cast<size_t>(r.n_pop) * r.n_pop * r.n_block, 0.0);
            if (sink(user, 0, r.n_block, z.data(), z.data()) != 0) fail(STP_RUNTIME_ERROR, "the slab sink stopped the extraction");
            return;
        }
        run_pipelined(c, r, t, *p, d_rec, dp);
        umma_check(p->umma);
    });
}

stp_status stp_f2_extract_blocks(stp_ctx* ctx, const stp_f2_request* req, stp_f2_output* out) {
    return guarded([&] {
        need(ctx && req && out, "null argument");
        use_device(*ctx);
        if (req->n_block > 0 && out->block_sizes) std::fill(out->block_sizes, out->block_sizes + req->n_block, 0);
        if (req->n_pop <= 0 || req->n_block <= 0) return;
        extract_one(*ctx, *req, *out);
    });
}

stp_status stp_f2_extract_batch(stp_ctx* ctx, const stp_f2_request* reqs, int32_t n_req, stp_f2_output* outs) {
    return guarded([&] {
        need(ctx && (reqs || n_req == 0) && (outs || n_req == 0), "null argument");
        use_device(*ctx);
        ctx->last_batch_ms.assign(static_cast<size_t>(std::max(n_req, 0)), std::nan(""));
        // Tensor-core requests over the same panel with the same arithmetic run as one
        // grouped batch; the rest (FP32 SIMT, empty requests) run one by one.
        std::vector<std::vector<int>> groups;
        for (int32_t k = 0; k < n_req; ++k) {
            const stp_f2_request& r = reqs[k];
            if (r.n_block > 0 && outs[k].block_sizes)
                std::fill(outs[k].block_sizes, outs[k].block_sizes + r.n_block, 0);
            if (r.n_pop <= 0 || r.n_block <= 0) continue;
            need(outs[k].f2 != nullptr && outs[k].vpair != nullptr, "output f2 / vpair is NULL");
            fmt_of(r.precision);  // validates the mode
            if (r.precision == STP_PREC_FP32_SIMT || r.geno.n_snp <= 0 || r.kept_rows) {
                extract_one(*ctx, r, outs[k]);
                continue;
            }
            bool placed = false;
            for (auto& grp : groups) {
                const stp_f2_request& h = reqs[grp[0]];
                if (same_panel(h.geno, r.geno) && h.precision == r.precision) {
                    grp.push_back(k);
                    placed = true;
                    break;
                }
            }
            if (!placed) groups.push_back({k});
        }
        for (const auto& grp : groups) {
            std::vector<double> done(grp.size(), 0.0);
            extract_batch_grouped(*ctx, reqs, outs, grp, done);
            for (size_t m = 0; m < grp.size(); ++m) ctx->last_batch_ms[static_cast<size_t>(grp[m])] = done[m];
        }
    });
}

stp_status stp_fstats(stp_ctx* ctx, const double* f2, const double* vpair, const int32_t* block_sizes,
                      int32_t P, int32_t n_block, int32_t on_device, int32_t kind, const int32_t* idx,
                      int64_t n_idx, int64_t n_stat, double* est, double* var, int32_t* n_survivors) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        need(kind >= STP_FSTAT_F4 && kind <= STP_FSTAT_F4_LEFT_RIGHT, "unknown f-statistic kind");
        need(P >= 0 && n_block >= 0 && n_idx >= 0 && n_stat >= 0, "negative extent");
        use_device(*ctx);
        int64_t m = 0, nr = 0;
        if (kind == STP_FSTAT_F4) {
            need(n_idx == 4 * n_stat, "quartets: n_idx must be 4 * n_stat");
            m = n_stat;
        } else if (kind == STP_FSTAT_F3) {
            need(n_idx == 3 * n_stat, "triples: n_idx must be 3 * n_stat");
            m = n_stat;
        } else {
            need(n_stat <= n_idx, "left indices exceed n_idx");
            const int64_t nl = n_stat - 1;
            nr = n_idx - n_stat - 1;
            m = (nl > 0 && nr > 0) ? nl * nr : 0;
        }
        if (n_survivors) *n_survivors = 0;
        if (m > 0) {
            need(est != nullptr && var != nullptr, "null output");
            std::fill(est, est + m, 0.0);
            std::fill(var, var + m, 0.0);
        }
        if (m <= 0 || n_block <= 0 || P <= 0) return;
        need(f2 && vpair && block_sizes && idx, "null argument");
        for (int64_t q = 0; q < n_idx; ++q) need(idx[q] >= 0 && idx[q] < P, "population index outside [0, P)");
        cudaStream_t s = ctx->stream;
        const size_t elems = static_cast<size_t>(P) * P * n_block;
        const double* d_f2 = f2;
        const double* d_vp = vpair;
        if (!on_device) {
            ctx->ws_f2.reserve(elems * 8);
            ctx->ws_vpair.reserve(elems * 8);
            STPF2_CUDA(cudaMemcpyAsync(ctx->ws_f2.ptr, f2, elems * 8, cudaMemcpyHostToDevice, s));
            STPF2_CUDA(cudaMemcpyAsync(ctx->ws_vpair.ptr, vpair, elems * 8, cudaMemcpyHostToDevice, s));
            d_f2 = ctx->ws_f2.as<double>();
            d_vp = ctx->ws_vpair.as<double>();
        }
        // Scratch in one grow-only context workspace (per-call allocations would each free
        // with a device-wide synchronisation): keep flags, survivors, their sizes, the
        // indices, the per-block values (sized for every block surviving) and est / var.
        Packing pk;
        const size_t o_keep = pk.add(static_cast<size_t>(n_block) * 4), o_surv = pk.add(static_cast<size_t>(n_block) * 4),
                     o_bl = pk.add(static_cast<size_t>(n_block) * 4), o_idx = pk.add(static_cast<size_t>(n_idx) * 4),
                     o_x = pk.add(static_cast<size_t>(m) * n_block * 8), o_est = pk.add(static_cast<size_t>(m) * 8),
                     o_var = pk.add(static_cast<size_t>(m) * 8);
        ctx->ws_fstat.reserve(pk.end);
        uint8_t* W = ctx->ws_fstat.as<uint8_t>();
        auto* d_keep = reinterpret_cast<int32_t*>(W + o_keep);
        auto* d_surv = reinterpret_cast<int32_t*>(W + o_surv);
        auto* d_bl = reinterpret_cast<int32_t*>(W + o_bl);
        auto* d_idx = reinterpret_cast<int32_t*>(W + o_idx);
        auto* d_x = reinterpret_cast<double*>(W + o_x);
        auto* d_est = reinterpret_cast<double*>(W + o_est);
        auto* d_var = reinterpret_cast<double*>(W + o_var);
        launch_survivors(*ctx, d_vp, P, n_block, d_keep, s);
        std::vector<int32_t> keep(static_cast<size_t>(n_block));
        STPF2_CUDA(cudaMemcpyAsync(keep.data(), d_keep, keep.size() * 4, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaStreamSynchronize(s));
        std::vector<int32_t> surv, bl;
        for (int32_t b = 0; b < n_block; ++b)
            if (keep[b]) {
                surv.push_back(b);
                bl.push_back(block_sizes[b]);
            }
        const int ns = static_cast<int>(surv.size());
        if (n_survivors) *n_survivors = ns;
        if (ns == 0) return;
        STPF2_CUDA(cudaMemcpyAsync(d_surv, surv.data(), surv.size() * 4, cudaMemcpyHostToDevice, s));
        STPF2_CUDA(cudaMemcpyAsync(d_bl, bl.data(), bl.size() * 4, cudaMemcpyHostToDevice, s));
        STPF2_CUDA(cudaMemcpyAsync(d_idx, idx, static_cast<size_t>(n_idx) * 4, cudaMemcpyHostToDevice, s));
        launch_fstat_assemble(*ctx, d_f2, P, d_surv, ns, kind, d_idx, n_stat, m, nr, d_x, s);
        launch_jackknife(*ctx, d_x, d_bl, m, ns, d_est, d_var, s);
        STPF2_CUDA(cudaMemcpyAsync(est, d_est, static_cast<size_t>(m) * 8, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaMemcpyAsync(var, d_var, static_cast<size_t>(m) * 8, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaStreamSynchronize(s));
    });
}

stp_status stp_set_wait_bounds(stp_ctx* ctx, uint64_t timeout_ns, int64_t withhold_stage) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        need(withhold_stage >= -1, "withhold_stage must be -1 or a stage index");
        ctx->fx_tuning.timeout_ns = timeout_ns ? timeout_ns : FxTuning{}.timeout_ns;
        ctx->fx_tuning.withhold_stage = withhold_stage;
    });
}

stp_status stp_set_tile_classes(stp_ctx* ctx, uint32_t partial_feed_mask) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        ctx->fx_tuning.partial_feed = partial_feed_mask & 0xFFFFu;
    });
}

stp_status stp_last_batch_times(stp_ctx* ctx, double* ms, int32_t n) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        need(ms != nullptr || n <= 0, "null argument");
        for (int32_t k = 0; k < n; ++k)
            ms[k] = static_cast<size_t>(k) < ctx->last_batch_ms.size() ? ctx->last_batch_ms[static_cast<size_t>(k)] : std::nan("");
    });
}

stp_status stp_f2_jackknife(stp_ctx* ctx, const double* x, const int32_t* block_sizes, int64_t m, int32_t n_block,
                            double* est, double* var) {
    return guarded([&] {
        need(ctx != nullptr, "null context");
        use_device(*ctx);
        if (m <= 0 || n_block <= 0) return;
        need(x && block_sizes && est && var, "null argument");
        cudaStream_t s = ctx->stream;
        DevBuf d_x, d_b, d_e, d_v;
        const size_t xe = static_cast<size_t>(m) * n_block;
        d_x.reserve(xe * 8);
        STPF2_CUDA(cudaMemcpyAsync(d_x.ptr, x, xe * 8, cudaMemcpyHostToDevice, s));
        std::vector<int32_t> bs(block_sizes, block_sizes + n_block);
        upload(d_b, bs, s);
        d_e.reserve(static_cast<size_t>(m) * 8);
        d_v.reserve(static_cast<size_t>(m) * 8);
        launch_jackknife(*ctx, d_x.as<double>(), d_b.as<int32_t>(), m, n_block, d_e.as<double>(), d_v.as<double>(), s);
        STPF2_CUDA(cudaMemcpyAsync(est, d_e.ptr, static_cast<size_t>(m) * 8, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaMemcpyAsync(var, d_v.ptr, static_cast<size_t>(m) * 8, cudaMemcpyDeviceToHost, s));
        STPF2_CUDA(cudaStreamSynchronize(s));
    });
}

stp_plan* stp_plan_create(stp_ctx* ctx, const stp_f2_request* req, stp_status* status) {
    stp_plan* out = nullptr;
    const stp_status st = guarded([&] {
        need(ctx && req, "null argument");
        use_device(*ctx);
        need(req->geno.on_device || req->geno.n_snp == 0, "a plan needs device-resident genotype records");
        const uint64_t pitch = req->geno.pitch ? req->geno.pitch : req->geno.bytes_per_record;
        std::unique_ptr<Plan> p = build_plan(*ctx, *req, pitch, nullptr);
        STPF2_CUDA(cudaStreamSynchronize(ctx->stream));
        auto* sp = new stp_plan();
        sp->p = std::move(p);
        out = sp;
    });
    if (status) *status = st;
    return out;
}

stp_status stp_plan_run(stp_plan* plan, const uint8_t* d_records, double* d_f2, double* d_vpair, void* stream) {
    return guarded([&] {
        need(plan != nullptr, "null plan");
        Plan& p = *plan->p;
        use_device(*p.ctx);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p.ctx->stream;
        run_plan(p, d_records, d_f2, d_vpair, s);
    });
}

stp_status stp_plan_run_graph(stp_plan* plan, const uint8_t* d_records, double* d_f2, double* d_vpair,
                              void* stream) {
    return guarded([&] {
        need(plan != nullptr, "null plan");
        Plan& p = *plan->p;
        use_device(*p.ctx);
        need(!p.timing, "disable plan timing before replaying the plan as a graph");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p.ctx->stream;
        const void* key[3] = {d_records, d_f2, d_vpair};
        if (!p.graph || !std::equal(key, key + 3, p.graph_key)) {
            if (p.graph) {
                STPF2_CUDA(cudaGraphExecDestroy(p.graph));
                p.graph = nullptr;
            }
            const uint64_t before = p.ctx->launches.load();
            cudaGraph_t g = nullptr;
            STPF2_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                run_plan(p, d_records, d_f2, d_vpair, s);
            } catch (...) {
                cudaStreamEndCapture(s, &g);
                if (g) cudaGraphDestroy(g);
                p.ctx->launches = before;
                throw;
            }
            STPF2_CUDA(cudaStreamEndCapture(s, &g));
            const cudaError_t e = cudaGraphInstantiate(&p.graph, g, 0);
            cudaGraphDestroy(g);
            p.ctx->launches = before;  // capturing launched nothing
            STPF2_CUDA(e);
            std::copy(key, key + 3, p.graph_key);
        }
        STPF2_CUDA(cudaGraphLaunch(p.graph, s));
        p.ctx->launches += static_cast<uint64_t>(p.launches());
    });
}

int32_t stp_plan_launches(const stp_plan* plan) { return plan ? plan->p->launches() : 0; }

stp_status stp_plan_set_per_block_launch(stp_plan* plan, int32_t enable) {
    return guarded([&] {
        need(plan != nullptr, "null plan");
        plan->p->per_block = enable != 0;
        if (plan->p->graph) {  // the captured graph holds the other launch form
            STPF2_CUDA(cudaGraphExecDestroy(plan->p->graph));
            plan->p->graph = nullptr;
        }
    });
}

stp_status stp_plan_set_timing(stp_plan* plan, int32_t enable) {
    return guarded([&] {
        need(plan != nullptr, "null plan");
        plan->p->timing = enable != 0;
        plan->p->n_timed = 0;
    });
}

stp_status stp_plan_last_times(const stp_plan* plan, float* decode_ms, float* contract_ms) {
    return guarded([&] {
        need(plan != nullptr, "null plan");
        const Plan& p = *plan->p;
        double sa = 0.0, sb = 0.0;
        for (size_t k = 0; k < p.n_timed; ++k) {
            STPF2_CUDA(cudaEventSynchronize(p.ev[k][2]));
            float a = 0.f, b = 0.f;
            STPF2_CUDA(cudaEventElapsedTime(&a, p.ev[k][0], p.ev[k][1]));
            STPF2_CUDA(cudaEventElapsedTime(&b, p.ev[k][1], p.ev[k][2]));
            sa += a;
            sb += b;
        }
        STPF2_CUDA(cudaStreamSynchronize(p.ctx->stream));
        umma_check(p.umma);
        const double n = p.n_timed ? static_cast<double>(p.n_timed) : 1.0;
        if (decode_ms) *decode_ms = static_cast<float>(sa / n);
        if (contract_ms) *contract_ms = static_cast<float>(sb / n);
    });
}

void stp_plan_destroy(stp_plan* plan) {
    if (!plan) return;
    cudaSetDevice(plan->p->ctx->device);
    cudaStreamSynchronize(plan->p->ctx->stream);
    delete plan;
}

}  // extern "C"
