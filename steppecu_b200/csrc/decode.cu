// steppecu_b200/csrc/decode.cu
//
// Genotype decode for the f2 path (sm_100a), in two passes over an intermediate canonical
// copy of the selected samples' genotypes. transpose_pa_kernel reads the SNP-major
// PACKEDANCESTRYMAP records from HBM in staged slices and writes each selected sample's
// codes for 128 columns as one 32-byte sector (plus a per-column centre);
// decode_canon_kernel folds every selected sample of every population into exact integer
// counts (ac2 = 2*ac, n) following decode_af.hpp:58-65 and writes the contraction operands
// for those counts straight into the block-padded tile images the contraction kernels read.
// Also here: per-sample ploidy detection (detect_ploidy_kernel.cu:32-57), the
// canonical-tile decode behind ComputeBackend::decode_af (cpu_backend.cpp:267-319), the
// operand emit from packed counts used by grouped batches, and the Q/V/N feeder behind
// compute_f2_blocks(MatView...) (f2_block_kernel.cu:37-61 computes the same per-element
// terms).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>

#include "stpf2_internal.cuh"

namespace stpf2 {

namespace {

constexpr int kTileCols = 32;      // columns per canonical tile (8 bytes per sample)
constexpr int kTransThreads = 256; // transpose: (16 samples, tile) per thread
constexpr int kDecThreads2 = 256;  // decode: (64 populations) x (4 tiles) per CTA
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
    if constexpr (F == OpFmt::F32) {
        const int64_t row = static_cast<int64_t>(i) * op.ld + col;
        const int64_t plane = static_cast<int64_t>(op.P) * op.ld;
        float* p = static_cast<float*>(op.planes);
        p[row] = static_cast<float>(t.pt);
        p[plane + row] = static_cast<float>(t.ah);
        op.m_u8[row] = static_cast<uint8_t>(t.m != 0.0);
    } else {
        using T = typename std::conditional<F == OpFmt::BF16, __nv_bfloat16, __half>::type;
        const double sp = (F == OpFmt::F16) ? double(1 << kF16PtShift) : 1.0;
        const double sa = sp * sp;
        const double pt = t.pt * sp, ah = t.ah * sa;
        const T pth = to16<T>(pt);
        const T ptl = to16<T>(pt - from16<T>(pth));
        const T ahh = to16<T>(ah);
        const T ahl = to16<T>(ah - from16<T>(ahh));
        const int64_t tile = static_cast<int64_t>(i / kTileRows) * op.n_ck + col / kTileK;
        const int r = i % kTileRows, k = static_cast<int>(col % kTileK);
        uint8_t* img = static_cast<uint8_t*>(op.planes) + tile * kImageBytes;
        uint8_t* b = img + tile16_offset(r, k);
        *reinterpret_cast<T*>(b) = pth;
        *reinterpret_cast<T*>(b + kTile16Bytes) = ptl;
        *reinterpret_cast<T*>(b + 2 * kTile16Bytes) = ahh;
        *reinterpret_cast<T*>(b + 3 * kTile16Bytes) = ahl;
        *reinterpret_cast<T*>(b + 4 * kTile16Bytes) = to16<T>(t.m);
        img[5 * kTile16Bytes + tile8_offset(r, k)] = static_cast<uint8_t>(t.m != 0.0);
    }
}

// Operand terms of 8 consecutive columns of one population, rounded to FP32 (enough for
// the split planes' ~22 significant bits; the splits then run on packed FP32 conversions).
struct Terms8 {
    float pt[8], ah[8];
    uint32_t mbits;  // bit c: column c called
};

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 a, __nv_bfloat16 b) {
    return static_cast<uint32_t>(__bfloat16_as_ushort(a)) | (static_cast<uint32_t>(__bfloat16_as_ushort(b)) << 16);
}
__device__ __forceinline__ uint32_t pack2(__half a, __half b) {
    return static_cast<uint32_t>(__half_as_ushort(a)) | (static_cast<uint32_t>(__half_as_ushort(b)) << 16);
}

// hi/lo split of two FP32 values into packed 16-bit pairs (round to nearest each).
template <OpFmt F>
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
    if constexpr (F == OpFmt::BF16) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
        const float2 hf = __bfloat1622float2(h);
        const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
        hi = pack2(h.x, h.y);
        lo = pack2(l.x, l.y);
    } else {
        const __half2 h = __floats2half2_rn(x0, x1);
        const float2 hf = __half22float2(h);
        const __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
        hi = pack2(h.x, h.y);
        lo = pack2(l.x, l.y);
    }
}

// Writes 8 consecutive columns (starting at a multiple of 8) of every operand plane with
// 16-byte stores: row-major FP32 planes, or one 16-byte chunk of each tiled 16-bit image
// (and 8 bytes of the int8 image). Row i, columns col..col+7.
template <OpFmt F>
__device__ __forceinline__ void emit8(const OperandPlanes& op, int i, int64_t col, const Terms8& t) {
    uint2 mv;
    mv.x = 0;
    mv.y = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint32_t bit = (t.mbits >> c) & 1u;
        if (c < 4) mv.x |= bit << (8 * c);
        else mv.y |= bit << (8 * (c - 4));
    }
    if constexpr (F == OpFmt::F32) {
        const int64_t off = static_cast<int64_t>(i) * op.ld + col;
        const int64_t plane = static_cast<int64_t>(op.P) * op.ld;
        float* p = static_cast<float*>(op.planes);
        *reinterpret_cast<float4*>(p + off) = make_float4(t.pt[0], t.pt[1], t.pt[2], t.pt[3]);
        *reinterpret_cast<float4*>(p + off + 4) = make_float4(t.pt[4], t.pt[5], t.pt[6], t.pt[7]);
        *reinterpret_cast<float4*>(p + plane + off) = make_float4(t.ah[0], t.ah[1], t.ah[2], t.ah[3]);
        *reinterpret_cast<float4*>(p + plane + off + 4) = make_float4(t.ah[4], t.ah[5], t.ah[6], t.ah[7]);
        *reinterpret_cast<uint2*>(op.m_u8 + off) = mv;
    } else {
        const float sp = (F == OpFmt::F16) ? float(1 << kF16PtShift) : 1.0f;
        const float sa = sp * sp;
        uint4 ph, pl, ahh, ahl, mm;
        uint32_t* PH = &ph.x;
        uint32_t* PL = &pl.x;
        uint32_t* AH = &ahh.x;
        uint32_t* AL = &ahl.x;
        uint32_t* MM = &mm.x;
#pragma unroll
        for (int c = 0; c < 8; c += 2) {
            split2<F>(t.pt[c] * sp, t.pt[c + 1] * sp, PH[c / 2], PL[c / 2]);
            split2<F>(t.ah[c] * sa, t.ah[c + 1] * sa, AH[c / 2], AL[c / 2]);
            const uint32_t one = (F == OpFmt::BF16) ? 0x3F80u : 0x3C00u;  // 1.0
            MM[c / 2] = (((t.mbits >> c) & 1u) ? one : 0u) | ((((t.mbits >> (c + 1)) & 1u) ? one : 0u) << 16);
        }
        const int r = i % kTileRows, k = static_cast<int>(col % kTileK);
        const int64_t tile = static_cast<int64_t>(i / kTileRows) * op.n_ck + col / kTileK;
        uint8_t* img = static_cast<uint8_t*>(op.planes) + tile * kImageBytes;
        uint8_t* b = img + tile16_offset(r, k);
        *reinterpret_cast<uint4*>(b) = ph;
        *reinterpret_cast<uint4*>(b + kTile16Bytes) = pl;
        *reinterpret_cast<uint4*>(b + 2 * kTile16Bytes) = ahh;
        *reinterpret_cast<uint4*>(b + 3 * kTile16Bytes) = ahl;
        *reinterpret_cast<uint4*>(b + 4 * kTile16Bytes) = mm;
        *reinterpret_cast<uint2*>(img + 5 * kTile16Bytes + tile8_offset(r, k)) = mv;
    }
}

// ---- fixed-point operands (OpFmt::FX) -------------------------------------------------------
//
// x = q - 1/2 and a = x^2 - h in FP64 from the exact counts, rounded once to 32-bit fixed
// point: X = round(x * kFxScale) (|X| <= 127 * 2^24) and A = round(a * kFxAScale) (|A| <
// 2^31). Each is stored as four balanced int8 digits (base 256, digits in [-128, 127]):
// the bytes of (X + 0x80808080) ^ 0x80808080, least significant first. The image holds
// X's digits, the digits of -A, and M = 64 * [n > 0]; see f2_fx.cu for the products.

// Round to the nearest integer (ties to even) of |v| < 2^31, as the low word of v + 1.5 * 2^52.
__device__ __forceinline__ uint32_t fx_round_fma(double a, double b) {
    return static_cast<uint32_t>(__double2loint(fma(a, b, kFxRoundMagic)));
}

__device__ __forceinline__ uint32_t fx_digits(uint32_t v) { return (v + 0x80808080u) ^ 0x80808080u; }

// Fixed-point operands of one population at one SNP from its q (FP64) and called count n.
__device__ __forceinline__ void fx_terms(double q, double rnm1, uint32_t& X, uint32_t& NA) {
    const double h = q * (1.0 - q) * rnm1;
    const double x = q - 0.5;
    X = fx_round_fma(x, kFxScale);
    NA = fx_round_fma(-fma(x, x, -h), kFxAScale);
}

struct FxTerms8 {
    uint32_t x[8], na[8];  // digit bytes (fx_digits) of X and -A
    uint32_t mbits;        // bit c: column c called
};

__device__ __forceinline__ FxTerms8 fx_terms8_from_counts(const uint32_t (&v)[8], const double* __restrict__ rec_n,
                                                          const double* __restrict__ rec_nm1,
                                                          const uint2* __restrict__ table = nullptr, int ld = 0) {
    FxTerms8 t;
    t.mbits = 0;
    if (table) {  // the precomputed digit words of (n, a2): the same function, evaluated once
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const uint32_t n = v[c] >> 16, a2 = v[c] & 0xFFFFu;
            const uint2 e = __ldg(table + static_cast<int64_t>(n) * ld + a2);
            t.x[c] = e.x;
            t.na[c] = e.y;
            t.mbits |= (n > 0 ? 1u : 0u) << c;
        }
        return t;
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint32_t n = v[c] >> 16, a2 = v[c] & 0xFFFFu;
        uint32_t X = 0, NA = 0;
        if (n > 0) {
            const double a2d = __hiloint2double(0x43300000, static_cast<int>(a2)) - 4503599627370496.0;
            fx_terms(a2d * 0.5 * __ldg(rec_n + n), __ldg(rec_nm1 + n), X, NA);
            t.mbits |= 1u << c;
        }
        t.x[c] = fx_digits(X);
        t.na[c] = fx_digits(NA);
    }
    return t;
}

// 4 x 4 byte transpose: o[k] holds byte k of w0, w1, w2, w3 in its bytes 0..3 (eight PRMTs).
__device__ __forceinline__ void bytes4x4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t (&o)[4]) {
    const uint32_t a = __byte_perm(w0, w1, 0x5140), b = __byte_perm(w0, w1, 0x7362);  // bytes 0,1 / 2,3 of w0,w1
    const uint32_t c = __byte_perm(w2, w3, 0x5140), d = __byte_perm(w2, w3, 0x7362);
    o[0] = __byte_perm(a, c, 0x5410);
    o[1] = __byte_perm(a, c, 0x7632);
    o[2] = __byte_perm(b, d, 0x5410);
    o[3] = __byte_perm(b, d, 0x7632);
}


// Writes 8 consecutive columns (starting at a multiple of 8) of one population into its
// fixed-point operand image (nine int8 tiles, 8 bytes each) and into the separate M tiles.
__device__ __forceinline__ void emit8_fx(const OperandPlanes& op, int i, int64_t col, const FxTerms8& t) {
    const int r = i % kTileRows, k = static_cast<int>(col % kTileK);
    const int64_t tile = static_cast<int64_t>(i / kTileRows) * op.n_ck + col / kTileK;
    uint8_t* img = static_cast<uint8_t*>(op.planes) + tile * kFxImageBytes + tile8_offset(r, k);
    // Digit d of the 8 columns, per plane: two 4 x 4 byte transposes per digit word set.
    uint32_t x0[4], x1[4], n0[4], n1[4];
    bytes4x4(t.x[0], t.x[1], t.x[2], t.x[3], x0);
    bytes4x4(t.x[4], t.x[5], t.x[6], t.x[7], x1);
    bytes4x4(t.na[0], t.na[1], t.na[2], t.na[3], n0);
    bytes4x4(t.na[4], t.na[5], t.na[6], t.na[7], n1);
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        *reinterpret_cast<uint2*>(img + d * kTile8Bytes) = make_uint2(x0[d], x1[d]);
        *reinterpret_cast<uint2*>(img + (4 + d) * kTile8Bytes) = make_uint2(n0[d], n1[d]);
    }
    // M = 64 in byte c where column c is called: bit c of each nibble spread to bit 8c.
    static_assert(kFxM == 64, "M is 1 << 6");
    const uint32_t lo = t.mbits & 0xFu, hi = (t.mbits >> 4) & 0xFu;
    const uint2 mv = make_uint2(((lo * 0x00204081u) & 0x01010101u) << 6, ((hi * 0x00204081u) & 0x01010101u) << 6);
    *reinterpret_cast<uint2*>(op.mplanes + tile * kTile8Bytes + tile8_offset(r, k)) = mv;
}

// One element (the Q/V/N feeder): q, n as FP64.
__device__ __forceinline__ void emit_fx(const OperandPlanes& op, int i, int64_t col, double q, double nd, bool valid) {
    uint32_t X = 0, NA = 0;
    if (valid) {
        const double nm1 = nd - 1.0;
        fx_terms(q, 1.0 / ((nm1 > 1.0) ? nm1 : 1.0), X, NA);
    }
    const uint32_t dx = fx_digits(X), dn = fx_digits(NA);
    const int r = i % kTileRows, k = static_cast<int>(col % kTileK);
    const int64_t tile = static_cast<int64_t>(i / kTileRows) * op.n_ck + col / kTileK;
    uint8_t* img = static_cast<uint8_t*>(op.planes) + tile * kFxImageBytes + tile8_offset(r, k);
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        img[d * kTile8Bytes] = static_cast<uint8_t>(dx >> (8 * d));
        img[(4 + d) * kTile8Bytes] = static_cast<uint8_t>(dn >> (8 * d));
    }
    const uint8_t m = valid ? uint8_t(kFxM) : uint8_t(0);
    op.mplanes[tile * kTile8Bytes + tile8_offset(r, k)] = m;
}

// ---- canonical genotypes -------------------------------------------------------------------
//
// The decode runs in two passes over an intermediate "canonical" copy of the selected
// samples' genotypes, laid out in the padded column space of the operand planes. Columns
// are grouped in quads of 128 = four 32-column tiles; selected sample g owns one 32-byte
// sector per quad: canon[((quad * n_sel + g) * 4 + sub] holds tile 4*quad + sub, column
// 32*tile + 4k + j in byte k at bits (7-2j, 6-2j) (MSB-first, as in the .geno records).
// Padding columns hold code 3 (missing) and therefore decode to zero operands.

// 4x4 transpose of 2-bit elements packed MSB-first in a 32-bit word (row 0 in the top
// byte): two block-swap steps.
__device__ __forceinline__ uint32_t transpose4x4_2bit(uint32_t w) {
    uint32_t t = (w ^ (w >> 12)) & 0x0000F0F0u;
    w ^= t ^ (t << 12);
    t = (w ^ (w >> 6)) & 0x00CC00CCu;
    w ^= t ^ (t << 6);
    return w;
}

constexpr int kSliceWords = 64;                      // 1024 samples per staged slice
constexpr int kSliceBytes = kSliceWords * 4;
constexpr int kRowStride = kSliceWords + 4;          // words per staged record row (16-byte rows)
constexpr int kStagedWords = 4 * kTileCols * kRowStride + 32;
constexpr int kQuadRows = 4 * kTileCols;  // record rows of a quad
// Two staging buffers, then the quad's row offsets (int64 each).
constexpr size_t kTransSmemBytes = 2 * kStagedWords * sizeof(uint32_t) + kQuadRows * sizeof(int64_t);
static_assert((2 * kStagedWords * sizeof(uint32_t)) % 8 == 0, "row table alignment");
static_assert(kTransThreads >= kQuadRows && (kQuadRows * (kSliceBytes / 16)) % kTransThreads == 0, "staging split");

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}

// Byte offset of each of the quad's 128 record rows (row sub*32 + r: SNP r of tile 4q+sub,
// through the row map when rows are kept), or -1 for a row past its tile's SNPs or past the
// last tile. Computed once per CTA; every slice's staging reads it.
__device__ __forceinline__ void quad_rows(int64_t* rows, uint64_t pitch, const TileInfo* __restrict__ tiles,
                                          int64_t n_tiles, int64_t q, const int32_t* __restrict__ row_map) {
    const int row = threadIdx.x;
    if (row >= kQuadRows) return;
    const int sub = row / kTileCols, r = row % kTileCols;
    const int64_t t = 4 * q + sub;
    int64_t off = -1;
    if (t < n_tiles) {
        const TileInfo ti = tiles[t];
        if (r < ti.nvalid) {
            const int64_t snp = static_cast<int64_t>(ti.snp0) + r;
            off = static_cast<int64_t>(row_map ? __ldg(row_map + snp) : snp) * static_cast<int64_t>(pitch);
        }
    }
    rows[row] = off;
}

// Stages slice `slice` of the quad's 128 records into buf: row (sub, r) at word
// (sub*32 + r)*kRowStride + sub*8 (the sub*8 skew keeps the threads of one warp on
// distinct banks when they read it back); bytes past the record and rows without a record
// (rows[row] < 0) hold code 3 (missing). Thread t copies 16-byte column t % 16 of rows
// t / 16 + 16 i. kVec16: records and pitch are 16-byte aligned (16-byte copies); otherwise
// 4-byte aligned (4-byte copies, so a host panel keeps its own pitch on the device).
template <bool kVec16>
__device__ __forceinline__ void stage_slice(uint32_t* buf, const uint8_t* __restrict__ records, uint64_t pitch,
                                            const int64_t* rows, int64_t slice) {
    constexpr int kCols16 = kSliceBytes / 16;
    const int k = threadIdx.x % kCols16;
    const uint64_t b = static_cast<uint64_t>(slice) * kSliceBytes + static_cast<uint64_t>(k) * 16;
#pragma unroll
    for (int i = 0; i < kQuadRows * kCols16 / kTransThreads; ++i) {
        const int row = threadIdx.x / kCols16 + i * (kTransThreads / kCols16);
        uint32_t* d = buf + row * kRowStride + (row / kTileCols) * 8 + k * 4;
        const int64_t off = rows[row];
        if constexpr (kVec16) {
            if (off >= 0 && b < pitch) cp_async16(d, records + off + b);
            else *reinterpret_cast<uint4*>(d) = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
        } else {
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                if (off >= 0 && b + 4 * w < pitch) cp_async4(d + w, records + off + b + 4 * w);
                else d[w] = 0xFFFFFFFFu;
            }
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Pass 1: SNP-major records -> canonical quads, gathering the selected samples. One CTA per
// quad of 128 columns walks the record slices of 1024 samples, staging slice s+1 with
// cp.async while it transposes slice s: thread (word w, tile sub) transposes 16 samples x
// 32 columns with SWAR 4x4 transposes, and the four threads of a sample write its 32-byte
// sector together. The first slice also yields each column's centre c_s: the pooled
// frequency of the called genotypes among the record's first 256 samples, rounded to 1/256
// (f2 is exact for any per-SNP centre; this one only keeps the operand magnitudes small).
template <bool kVec16>
__global__ void __launch_bounds__(kTransThreads)
transpose_pa_kernel(const uint8_t* __restrict__ records, uint64_t pitch, int64_t n_ind,
                    const TileInfo* __restrict__ tiles, int64_t n_tiles, const int32_t* __restrict__ pos,
                    int64_t n_sel, int64_t n_slices, uint64_t* __restrict__ canon, double* __restrict__ center,
                    const int32_t* __restrict__ row_map) {
    extern __shared__ __align__(16) uint32_t srec_all[];
    const int64_t q = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t* rows = reinterpret_cast<int64_t*>(srec_all + 2 * kStagedWords);
    quad_rows(rows, pitch, tiles, n_tiles, q, row_map);
    __syncthreads();
    stage_slice<kVec16>(srec_all, records, pitch, rows, 0);
    for (int64_t slice = 0; slice < n_slices; ++slice) {
        uint32_t* srec = srec_all + (slice & 1) * kStagedWords;
        // One barrier per slice: after it every thread's copies of this slice have landed and
        // every thread is done with the previous slice, whose buffer the next slice refills.
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
        if (slice + 1 < n_slices)
            stage_slice<kVec16>(srec_all + ((slice + 1) & 1) * kStagedWords, records, pitch, rows, slice + 1);

        if (slice == 0 && warp < 4) {
            const int sub = warp;
            const int64_t t = 4 * q + sub;
            const int nvalid = t < n_tiles ? tiles[t].nvalid : 0;
            const int64_t rem = n_ind - static_cast<int64_t>(lane) * 16;
            const int nv = lane < 16 ? static_cast<int>(rem < 0 ? 0 : (rem < 16 ? rem : 16)) : 0;
            uint32_t vmask = 0;
            for (int m = 0; m < nv; ++m) vmask |= 3u << (8 * (m >> 2) + 6 - 2 * (m & 3));
            for (int r = 0; r < kTileCols; ++r) {
                const uint32_t x = (nv > 0 ? srec[(sub * kTileCols + r) * kRowStride + sub * 8 + lane] : 0u) & vmask;
                const uint32_t lo = x & 0x55555555u, hi = (x >> 1) & 0x55555555u;
                const uint32_t miss = lo & hi;
                const int cnt = __reduce_add_sync(0xffffffffu, __popc(vmask & 0x55555555u) - __popc(miss));
                const int sum = __reduce_add_sync(0xffffffffu, __popc(lo & ~miss) + 2 * __popc(hi & ~miss));
                if (lane == 0 && t < n_tiles)
                    center[t * kTileCols + r] =
                        (r < nvalid && cnt > 0) ? rint((static_cast<double>(sum) / (2.0 * cnt)) * 256.0) / 256.0 : 0.5;
            }
        }

        const int sub = threadIdx.x & 3;
        for (int wl = threadIdx.x >> 2; wl < kSliceWords; wl += blockDim.x >> 2) {
            const int64_t r0 = slice * (kSliceWords * 16) + static_cast<int64_t>(wl) * 16;
            const int64_t rem = n_ind - r0;
            if (rem <= 0) break;
            const int nv = static_cast<int>(rem < 16 ? rem : 16);
            const uint32_t* base = srec + sub * kTileCols * kRowStride + sub * 8 + wl;
            // y[rg][j]: the 4 x 4 block of SNPs 4rg.. x samples 4j.., transposed so that byte
            // 3 - m holds sample 4j + m's four codes.
            uint32_t y[kTileCols / 4][4];
#pragma unroll
            for (int rg = 0; rg < kTileCols / 4; ++rg) {
                uint32_t rw[4];
#pragma unroll
                for (int r = 0; r < 4; ++r) rw[r] = base[(4 * rg + r) * kRowStride];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const uint32_t sel = static_cast<uint32_t>(j) | (static_cast<uint32_t>(j + 4) << 4);
                    const uint32_t a = __byte_perm(rw[0], rw[1], sel);
                    const uint32_t b = __byte_perm(rw[2], rw[3], sel);
                    y[rg][j] = transpose4x4_2bit(__byte_perm(a, b, 0x0145));
                }
            }
            // Sample 4j + m's 32 SNPs: byte 3 - m of y[0..7][j], by 4 x 4 byte transposes.
            uint64_t out[16];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                uint32_t lo[4], hi[4];
                bytes4x4(y[0][j], y[1][j], y[2][j], y[3][j], lo);
                bytes4x4(y[4][j], y[5][j], y[6][j], y[7][j], hi);
#pragma unroll
                for (int m = 0; m < 4; ++m) out[4 * j + m] = (static_cast<uint64_t>(hi[3 - m]) << 32) | lo[3 - m];
            }
            int32_t g[16];
            if (nv == 16) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int4 v = __ldg(reinterpret_cast<const int4*>(pos + r0) + k);
                    g[4 * k] = v.x; g[4 * k + 1] = v.y; g[4 * k + 2] = v.z; g[4 * k + 3] = v.w;
                }
            } else {
#pragma unroll
                for (int m = 0; m < 16; ++m) g[m] = m < nv ? __ldg(pos + r0 + m) : -1;
            }
#pragma unroll
            for (int m = 0; m < 16; ++m)
                if (g[m] >= 0) canon[(q * n_sel + g[m]) * 4 + sub] = out[m];
        }
    }
}

// Pass 2: one CTA per (64 populations, quad of 4 column tiles), in two phases.
//
// Fold: a warp holds 8 populations x 4 tiles, lane = (population, tile), so the four lanes
// of a population read one 32-byte sector of the quad per sample. With a fold order the
// warps take the CTA's 64 populations largest first, so that the populations of one warp
// have similar sample counts (the counts land in the same shared slots either way). Each thread folds its
// population's samples into exact integer counts for its tile's 32 columns at once with
// SWAR bytes: PRMT maps four 2-bit codes, taken as selector nibbles straight from the
// masked code bits, to four count bytes through the sample's ploidy table (byte b of count
// word k holds column dec_col(k, b)). Four sample loads stay in flight per thread. Counts
// go to shared memory (byte lanes spill there every 60 samples).
//
// Emit: warp w takes its 8 populations again, now with lane = (population, 8-column chunk),
// and walks the 4 tiles, so every 16-byte store instruction of a plane fills 8 whole
// 64-byte rows (512 contiguous bytes) of one tile image.
constexpr int kDecPops = 64;                        // populations per decode CTA
constexpr int kDecUnroll = 4;                       // sample loads in flight per thread
constexpr int kDecFlush = 60 / kDecUnroll;          // iterations between byte-lane spills
constexpr int kCenterPitch = kTileCols + 1;         // doubles per tile of shared centres
// Shared counts (ac2 | n << 16) of (tile t, column c, population p) at word
// t * kCntTile + c * kCntCol + p: fold writes (fixed c; p, t vary) and emit reads (fixed
// t, c; p and the chunk vary) both touch 32 distinct banks.
constexpr int kCntCol = kDecPops + 1;
constexpr int kCntTile = kTileCols * kCntCol + 8;
constexpr size_t kDecSmemBytes = size_t(4) * kCntTile * 4;

// Column (0..31 within the tile) that byte b of count word k accumulates. Word k = 4h + s
// comes from half h of the 8 canonical bytes and selector s: s = 0 / 1 take the low 16 bits
// of lo = w & 0x33333333 / hi = (w >> 2) & 0x33333333, s = 2 / 3 their high 16 bits; byte
// k' of w holds columns 4k' .. 4k'+3 MSB-first, so lo's nibbles hold columns 4k'+3, 4k'+1
// and hi's 4k'+2, 4k'.
__host__ __device__ constexpr int dec_col(int k, int b) {
    return 16 * (k >> 2) + 8 * ((k >> 1) & 1) + 4 * (b >> 1) + 2 * (1 - (b & 1)) + (1 - (k & 1));
}

// Adds one sample's codes for 32 columns (x: 8 canonical bytes) to the byte-lane sums.
// pl is the sample's ploidy (1 pseudo-haploid, 2 diploid, 0 none); the tables map code
// 0/1/2/3 to ac2 = (0, 1, 2, 0) * pl and n = (1, 1, 1, 0) * pl (decode_af.hpp:58-65).
__device__ __forceinline__ void fold_sample(uint64_t x, uint32_t pl, uint32_t (&sa)[8], uint32_t (&sn)[8]) {
    const uint32_t la = 0x00020100u * pl, ln = 0x00010101u * pl;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint32_t w = static_cast<uint32_t>(x >> (32 * h));
        const uint32_t lo = w & 0x33333333u, hi = (w >> 2) & 0x33333333u;
        const uint32_t sel[4] = {lo, hi, lo >> 16, hi >> 16};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            sa[4 * h + s] += __byte_perm(la, 0, sel[s]);
            sn[4 * h + s] += __byte_perm(ln, 0, sel[s]);
        }
    }
}

// Moves the byte-lane sums into the shared counts (adding to what an earlier spill left).
__device__ __forceinline__ void spill_counts(uint32_t* cnt, bool add, uint32_t (&sa)[8], uint32_t (&sn)[8]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            // ac2 byte b -> bits 0-7, n byte b -> bits 16-23
            const uint32_t v = __byte_perm(sa[k], sn[k], b | ((4 + b) << 8)) & 0x00FF00FFu;
            uint32_t* d = cnt + dec_col(k, b) * kCntCol;
            *d = (add ? *d : 0u) + v;
        }
        sa[k] = sn[k] = 0;
    }
}

// Operand terms of 8 columns from their packed counts (ac2 | n << 16) and centres: in FP64
// (q from the exact counts), rounded once to FP32 for the planes; a2 -> double through the
// 2^52 trick (an FP64 add, no conversion unit).
__device__ __forceinline__ Terms8 terms8_from_counts(const uint32_t (&v)[8], const double* cen,
                                                     const double* __restrict__ rec_n,
                                                     const double* __restrict__ rec_nm1) {
    Terms8 tm;
    tm.mbits = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint32_t n = v[c] >> 16, a2 = v[c] & 0xFFFFu;
        double pt = 0.0, ah = 0.0;
        if (n > 0) {
            const double a2d = __hiloint2double(0x43300000, static_cast<int>(a2)) - 4503599627370496.0;
            const double qf = a2d * 0.5 * __ldg(rec_n + n);
            const double h = qf * (1.0 - qf) * __ldg(rec_nm1 + n);
            pt = qf - cen[c];
            ah = 0.5 * (pt * pt - h);
            tm.mbits |= 1u << c;
        }
        tm.pt[c] = static_cast<float>(pt);
        tm.ah[c] = static_cast<float>(ah);
    }
    return tm;
}

template <OpFmt F, bool kUnion>
__global__ void __launch_bounds__(kDecThreads2, 5)
decode_canon_kernel(const uint64_t* __restrict__ canon, int64_t n_tiles, int64_t n_sel,
                    const uint32_t* __restrict__ sel, const int32_t* __restrict__ pop_off, int P,
                    const double* __restrict__ center, const double* __restrict__ rec_n,
                    const double* __restrict__ rec_nm1, const int32_t* __restrict__ col_snp, int64_t col_base,
                    OperandPlanes op, int32_t* __restrict__ cnt_ac2, int32_t* __restrict__ cnt_n,
                    const int32_t* __restrict__ umap, const double* __restrict__ center_snp,
                    uint32_t* __restrict__ cnt_packed, int64_t cnt_ld, const int32_t* __restrict__ fold_order) {
    extern __shared__ uint32_t s_cnt[];
    __shared__ double s_center[4 * kCenterPitch];
    const int64_t q = blockIdx.x;
    for (int c = threadIdx.x; c < 4 * kTileCols; c += blockDim.x) {
        const int64_t col = q * 4 * kTileCols + c;
        double cv = 0.5;
        if (col < n_tiles * kTileCols) {
            if constexpr (kUnion) {
                const int32_t s = __ldg(col_snp + col);
                if (s >= 0) cv = __ldg(center_snp + s);
            } else {
                cv = __ldg(center + col);
            }
        }
        s_center[(c / kTileCols) * kCenterPitch + c % kTileCols] = cv;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    {
        const int sub = lane & 3;
        const int slot = warp * 8 + (lane >> 2);
        const int pl_ = fold_order ? __ldg(fold_order + blockIdx.y * kDecPops + slot) : slot;
        const int i = blockIdx.y * kDecPops + pl_;
        if (i < P && 4 * q + sub < n_tiles) {
            const int g0 = __ldg(pop_off + i), g1 = __ldg(pop_off + i + 1);
            uint32_t* cnt = s_cnt + sub * kCntTile + pl_;
            uint32_t sa[8], sn[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) sa[k] = sn[k] = 0;
            bool spilled = false;
            int it = 0;
            const uint64_t* col = canon + q * n_sel * 4 + sub;
            // Shared-canonical mode: selected sample gg is canonical sample umap[gg].
            auto load = [&](int gg) -> uint64_t {
                if constexpr (kUnion) return __ldg(col + static_cast<int64_t>(__ldg(umap + gg)) * 4);
                else return __ldg(col + static_cast<int64_t>(gg) * 4);
            };
            int g = g0;
            for (; g + kDecUnroll <= g1; g += kDecUnroll) {
                uint64_t x[kDecUnroll];
                uint32_t pl[kDecUnroll];
#pragma unroll
                for (int u = 0; u < kDecUnroll; ++u) {
                    x[u] = load(g + u);
                    pl[u] = __ldg(sel + g + u) & 3u;
                }
#pragma unroll
                for (int u = 0; u < kDecUnroll; ++u) fold_sample(x[u], pl[u], sa, sn);
                if (++it == kDecFlush) {  // byte lanes hold at most 63 samples x 4
                    spill_counts(cnt, spilled, sa, sn);
                    spilled = true;
                    it = 0;
                }
            }
            if (g < g1) {  // fewer than kDecUnroll samples left (at most 59 unspilled in all)
                uint64_t x[kDecUnroll - 1];
                uint32_t pl[kDecUnroll - 1];
#pragma unroll
                for (int u = 0; u < kDecUnroll - 1; ++u) {
                    const bool ok = g + u < g1;
                    x[u] = ok ? load(g + u) : ~0ull;
                    pl[u] = ok ? (__ldg(sel + g + u) & 3u) : 0u;
                }
#pragma unroll
                for (int u = 0; u < kDecUnroll - 1; ++u) fold_sample(x[u], pl[u], sa, sn);
            }
            spill_counts(cnt, spilled, sa, sn);
        }
    }
    __syncthreads();

    const int r = lane & 7, chunk = lane >> 3;
    const int pl_ = warp * 8 + r;
    const int i = blockIdx.y * kDecPops + pl_;
    if (i >= P) return;
#pragma unroll 1
    for (int sub = 0; sub < 4; ++sub) {
        const int64_t t = 4 * q + sub;
        if (t >= n_tiles) break;
        const int64_t col0 = t * kTileCols + 8 * chunk;
        const uint32_t* cnt = s_cnt + sub * kCntTile + (8 * chunk) * kCntCol + pl_;
        const double* cen = s_center + sub * kCenterPitch + 8 * chunk;
        if (cnt_ac2) {
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int32_t s = __ldg(col_snp + col0 + c);
                const uint32_t v = cnt[c * kCntCol];
                if (s >= 0) {
                    cnt_ac2[static_cast<int64_t>(i) + static_cast<int64_t>(P) * s] = static_cast<int32_t>(v & 0xFFFFu);
                    cnt_n[static_cast<int64_t>(i) + static_cast<int64_t>(P) * s] = static_cast<int32_t>(v >> 16);
                }
            }
        }
        if (cnt_packed) {
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int32_t s = __ldg(col_snp + col0 + c);
                if (s >= 0) cnt_packed[static_cast<int64_t>(i) * cnt_ld + s] = cnt[c * kCntCol];
            }
        }
        if (!op.planes) continue;
        uint32_t v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = cnt[c * kCntCol];
        if constexpr (F == OpFmt::FX)
            emit8_fx(op, i, col_base + col0, fx_terms8_from_counts(v, rec_n, rec_nm1, op.fx_table, op.fx_table_ld));
        else
            emit8<F>(op, i, col_base + col0, terms8_from_counts(v, cen, rec_n, rec_nm1));
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
    if constexpr (F == OpFmt::FX)
        emit_fx(op, i, snp_col[s], Q[o], N[o], V[o] != 0.0);
    else
        emit<F>(op, i, snp_col[s], make_terms(Q[o], N[o], V[o] != 0.0, center[s]));
}

}  // namespace

namespace {
// The same rule with one warp per 4-byte record word (16 samples): the lanes read the word
// from 32 records at a time (coalesced across the warps of neighbouring words) and OR
// their het masks (code 1: low bit set, high bit clear); lanes 0-15 then write the
// ploidy of the word's selected samples (pos: file row -> selected index, -1 if not).
__global__ void detect_ploidy_words_kernel(const uint8_t* __restrict__ records, uint64_t pitch, int64_t window,
                                           int64_t n_ind, const int32_t* __restrict__ pos, uint32_t* __restrict__ sel) {
    const int64_t w = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (16 * w >= n_ind) return;  // warp-uniform
    uint32_t het = 0;
    for (int64_t s = lane; s < window; s += 32) {
        const uint32_t x = __ldg(reinterpret_cast<const uint32_t*>(records + s * pitch) + w);
        het |= (x & 0x55555555u) & ~((x >> 1) & 0x55555555u);
    }
    het = __reduce_or_sync(0xffffffffu, het);
    const int64_t row = 16 * w + lane;
    if (lane < 16 && row < n_ind) {
        const int32_t g = __ldg(pos + row);
        if (g >= 0) {
            const bool h = (het >> (8 * (lane >> 2) + 6 - 2 * (lane & 3))) & 1u;
            sel[g] = (sel[g] & ~3u) | (h ? 2u : 1u);
        }
    }
}
}  // namespace

namespace {
// The canonical individual-major tile (record g: individual g's SNP codes, 4 per byte
// MSB-first) to SNP-major PACKEDANCESTRYMAP records (record s: individual g's code at byte
// g / 4, MSB-first). Thread (4 SNPs, 4 individuals): four tile bytes in, a 4x4 2-bit
// transpose, four record bytes out (consecutive threads write consecutive bytes of a record).
// Individuals past n_ind read as missing (code 3).
__global__ void canonical_to_records_kernel(const uint8_t* __restrict__ packed, uint64_t bpr, int64_t n_snp,
                                            int64_t n_ind, uint8_t* __restrict__ records, uint64_t pitch) {
    const int64_t g4 = static_cast<int64_t>(blockIdx.y) * blockDim.x + threadIdx.x;
    const int64_t s4 = static_cast<int64_t>(blockIdx.x) * blockDim.y + threadIdx.y;
    if (4 * g4 >= n_ind || 4 * s4 >= n_snp) return;
    uint32_t w = 0;  // byte j (row 0 in the top byte): individual 4*g4 + j's codes of SNPs 4*s4 .. +3
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t g = 4 * g4 + j;
        const uint32_t b = g < n_ind ? packed[g * static_cast<int64_t>(bpr) + s4] : 0xFFu;
        w |= b << (8 * (3 - j));
    }
    w = transpose4x4_2bit(w);  // byte k (top first): SNP 4*s4 + k's codes of the 4 individuals
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int64_t s = 4 * s4 + k;
        if (s < n_snp) records[s * static_cast<int64_t>(pitch) + g4] = static_cast<uint8_t>(w >> (8 * (3 - k)));
    }
}
}  // namespace

void launch_canonical_to_records(Ctx& c, const uint8_t* packed, uint64_t bpr, int64_t n_snp, int64_t n_ind,
                                 uint8_t* records, uint64_t pitch, cudaStream_t s) {
    if (n_snp <= 0 || n_ind <= 0) return;
    const dim3 block(64, 4);
    const dim3 grid(static_cast<unsigned>(((n_snp + 3) / 4 + 3) / 4), static_cast<unsigned>(((n_ind + 3) / 4 + 63) / 64));
    if (grid.y > 65535u) fail(STP_INVALID_ARGUMENT, "canonical tile: too many individuals for one transpose launch");
    canonical_to_records_kernel<<<grid, block, 0, s>>>(packed, bpr, n_snp, n_ind, records, pitch);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_detect_ploidy_words(Ctx& c, const uint8_t* records, uint64_t pitch, int64_t n_snp, int64_t n_ind,
                                const int32_t* pos, uint32_t* sel, cudaStream_t s) {
    if (n_ind <= 0 || n_snp <= 0) return;
    if (pitch % 4 != 0 || reinterpret_cast<uintptr_t>(records) % 4 != 0)
        fail(STP_INVALID_ARGUMENT, "word-wise ploidy detection needs 4-byte aligned records and pitch");
    const int64_t window = n_snp < kPloidyWindow ? n_snp : kPloidyWindow;
    const int64_t warps = (n_ind + 15) / 16;
    detect_ploidy_words_kernel<<<static_cast<unsigned>((warps + 7) / 8), 256, 0, s>>>(records, pitch, window, n_ind, pos, sel);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

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

void launch_transpose_pa(Ctx& c, const uint8_t* records, uint64_t pitch, int64_t n_ind, const TileInfo* tiles,
                         int64_t n_tiles, const int32_t* pos, int64_t n_sel, uint64_t* canon, double* center,
                         cudaStream_t s, const int32_t* row_map) {
    if (n_tiles <= 0) return;
    const uint64_t align = pitch | static_cast<uint64_t>(reinterpret_cast<uintptr_t>(records));
    if (align % 4 != 0) fail(STP_INVALID_ARGUMENT, "transpose: genotype records need a 4-byte aligned pitch");
    const bool vec16 = align % 16 == 0;
    const int64_t n_quads = (n_tiles + 3) / 4;
    const int64_t n_slices = std::max<int64_t>(1, (n_ind + kSliceWords * 16 - 1) / (kSliceWords * 16));
    static bool attr_set[2][64] = {};  // per form and device ordinal
    if (c.device < 0 || c.device >= 64 || !attr_set[vec16][c.device]) {
        STPF2_CUDA(cudaFuncSetAttribute(vec16 ? transpose_pa_kernel<true> : transpose_pa_kernel<false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kTransSmemBytes)));
        if (c.device >= 0 && c.device < 64) attr_set[vec16][c.device] = true;
    }
    if (vec16)
        transpose_pa_kernel<true><<<static_cast<unsigned>(n_quads), kTransThreads, kTransSmemBytes, s>>>(
            records, pitch, n_ind, tiles, n_tiles, pos, n_sel, n_slices, canon, center, row_map);
    else
        transpose_pa_kernel<false><<<static_cast<unsigned>(n_quads), kTransThreads, kTransSmemBytes, s>>>(
            records, pitch, n_ind, tiles, n_tiles, pos, n_sel, n_slices, canon, center, row_map);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

namespace {
// Operand images of one request from packed per-population counts (pop-major, row u at
// counts + u * cnt_ld, SNP s at column s): its population i reads row upop[i], its padded
// column c SNP col_snp[c]. Work unit = (8-row group, 32-column tile), one per warp from a
// flat range (row groups of one tile on neighbouring warps, so the tile's column maps are
// shared through L1), so every warp is busy whatever the population count; lane =
// (row, 8-column chunk), and each 16-byte store of a plane fills 8 whole 64-byte rows of
// the tile image. The terms are the decode's (terms8_from_counts).
template <OpFmt F>
__global__ void __launch_bounds__(256)
emit_counts_kernel(const uint32_t* __restrict__ counts, int64_t cnt_ld, bool vec, const int32_t* __restrict__ upop,
                   int P, int64_t n_tiles, const int32_t* __restrict__ col_snp, const double* __restrict__ center_snp,
                   const double* __restrict__ rec_n, const double* __restrict__ rec_nm1, OperandPlanes op) {
    const int lane = threadIdx.x & 31;
    const int r = lane & 7, chunk = lane >> 3;
    const int64_t n_rg = (P + 7) / 8;
    const int64_t n_units = n_rg * n_tiles;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t u = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); u < n_units; u += warps) {
        const int64_t t = u / n_rg;
        const int i = static_cast<int>(u - t * n_rg) * 8 + r;
        if (i >= P) continue;
        const uint32_t* row = counts + static_cast<int64_t>(__ldg(upop + i)) * cnt_ld;
        const int64_t col0 = t * kTileCols + 8 * chunk;
        // The chunk's eight SNPs (col_snp rows are 32-byte aligned, col0 a multiple of 8).
        const int4 ca = __ldg(reinterpret_cast<const int4*>(col_snp + col0));
        const int4 cb = __ldg(reinterpret_cast<const int4*>(col_snp + col0) + 1);
        const int32_t sc[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
        uint32_t v[8];
        if (vec && sc[0] >= 0 && sc[7] == sc[0] + 7) {
            // Eight consecutive SNPs (a chunk inside one block): three aligned 16-byte loads
            // from the word s0 rounds down to, then the eight words from offset s0 & 3.
            const uint4* rp = reinterpret_cast<const uint4*>(row + (sc[0] & ~3));
            const uint4 w0 = __ldg(rp), w1 = __ldg(rp + 1), w2 = __ldg(rp + 2);
            const uint32_t w[12] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w, w2.x, w2.y, w2.z, w2.w};
            switch (sc[0] & 3) {
                case 0:
#pragma unroll
                    for (int c = 0; c < 8; ++c) v[c] = w[c];
                    break;
                case 1:
#pragma unroll
                    for (int c = 0; c < 8; ++c) v[c] = w[c + 1];
                    break;
                case 2:
#pragma unroll
                    for (int c = 0; c < 8; ++c) v[c] = w[c + 2];
                    break;
                default:
#pragma unroll
                    for (int c = 0; c < 8; ++c) v[c] = w[c + 3];
                    break;
            }
        } else {
#pragma unroll
            for (int c = 0; c < 8; ++c) v[c] = sc[c] >= 0 ? __ldg(row + sc[c]) : 0u;
        }
        double cen[8];
        if constexpr (F != OpFmt::FX) {  // the fixed point needs no centre
#pragma unroll
            for (int c = 0; c < 8; ++c) cen[c] = sc[c] >= 0 ? __ldg(center_snp + sc[c]) : 0.5;
        }
        if constexpr (F == OpFmt::FX)
            emit8_fx(op, i, col0, fx_terms8_from_counts(v, rec_n, rec_nm1, op.fx_table, op.fx_table_ld));
        else
            emit8<F>(op, i, col0, terms8_from_counts(v, cen, rec_n, rec_nm1));
    }
}
}  // namespace

namespace {
__global__ void copy_union_ploidy_kernel(uint32_t* __restrict__ desc, const int32_t* __restrict__ umap, int64_t n_sel,
                                         const uint32_t* __restrict__ desc_u) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g < n_sel && (desc[g] & 3u) == 3u) desc[g] = (desc[g] & ~3u) | (desc_u[umap[g]] & 3u);
}
}  // namespace

namespace {
// Column c of the padded space belongs to the last block whose first column is <= c (empty
// blocks share their successor's first column and cover nothing).
__global__ void layout_tables_kernel(const BlockInfo* __restrict__ blocks, const int64_t* __restrict__ snp_begin,
                                     int n_block, int64_t ld, int32_t* __restrict__ col_snp,
                                     TileInfo* __restrict__ tiles) {
    const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= ld) return;
    int lo = 0, hi = n_block;  // first block with col > c
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (blocks[mid].col <= c) lo = mid + 1;
        else hi = mid;
    }
    const int b = lo - 1;
    int64_t off = -1, k = 0, s0 = 0;
    if (b >= 0) {
        off = c - blocks[b].col;
        k = blocks[b].k;
        s0 = snp_begin[b];
    }
    const bool real = b >= 0 && off < k;
    col_snp[c] = real ? static_cast<int32_t>(s0 + off) : -1;
    if ((c & 31) == 0)
        tiles[c >> 5] = real ? TileInfo{static_cast<int32_t>(s0 + off), static_cast<int32_t>(k - off < 32 ? k - off : 32)}
                             : TileInfo{0, 0};
}
}  // namespace

void launch_layout_tables(Ctx& c, const BlockInfo* blocks, const int64_t* snp_begin, int n_block, int64_t ld,
                          int32_t* col_snp, TileInfo* tiles, cudaStream_t s) {
    if (ld <= 0) return;
    layout_tables_kernel<<<static_cast<unsigned>((ld + 255) / 256), 256, 0, s>>>(blocks, snp_begin, n_block, ld, col_snp, tiles);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

namespace {
// Entry n * (2 n_max + 1) + a2 of the fixed-point term table: the digit words of X and -A
// for a population with n called alleles and doubled count a2, exactly as the emit
// computes them (zeros when n = 0 or a2 > 2n).
__global__ void fx_table_kernel(const double* __restrict__ rec_n, const double* __restrict__ rec_nm1, int64_t n_max,
                                uint2* __restrict__ out) {
    const int64_t ld = 2 * n_max + 1;
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= (n_max + 1) * ld) return;
    const int64_t n = k / ld, a2 = k - n * ld;
    uint32_t X = 0, NA = 0;
    if (n > 0 && a2 <= 2 * n) {
        const double a2d = __hiloint2double(0x43300000, static_cast<int>(a2)) - 4503599627370496.0;
        fx_terms(a2d * 0.5 * __ldg(rec_n + n), __ldg(rec_nm1 + n), X, NA);
    }
    out[k] = make_uint2(fx_digits(X), fx_digits(NA));
}
}  // namespace

int64_t fx_table_entries(int64_t n_max) {
    const int64_t e = (n_max + 1) * (2 * n_max + 1);
    return e <= (int64_t(1) << 20) ? e : 0;  // 8 MiB at most; larger populations compute the terms
}

void launch_fx_table(Ctx& c, const double* rec_n, const double* rec_nm1, int64_t n_max, uint2* out, cudaStream_t s) {
    const int64_t e = fx_table_entries(n_max);
    if (e <= 0) return;
    fx_table_kernel<<<static_cast<unsigned>((e + 255) / 256), 256, 0, s>>>(rec_n, rec_nm1, n_max, out);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_emit_counts(Ctx& c, const uint32_t* counts, int64_t cnt_ld, int64_t n_snp, const int32_t* upop, int P, int64_t n_tiles,
                        const int32_t* col_snp, const double* center_snp, const double* rec_n, const double* rec_nm1,
                        const OperandPlanes& op, cudaStream_t s) {
    if (P <= 0 || n_tiles <= 0) return;
    const int64_t units = (P + 7) / 8 * n_tiles;
    const int64_t cap = static_cast<int64_t>(c.sm_count) * 16;  // 16 CTAs of 8 warps per SM, grid-stride beyond
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((units + 7) / 8, cap)));
    if (reinterpret_cast<uintptr_t>(col_snp) % 32 != 0) fail(STP_RUNTIME_ERROR, "emission: column map not 32-byte aligned");
    const bool vec = cnt_ld % 4 == 0 && cnt_ld >= n_snp + 4 && reinterpret_cast<uintptr_t>(counts) % 16 == 0;
    switch (op.fmt) {
        case OpFmt::F32: emit_counts_kernel<OpFmt::F32><<<grid, 256, 0, s>>>(counts, cnt_ld, vec, upop, P, n_tiles, col_snp, center_snp, rec_n, rec_nm1, op); break;
        case OpFmt::BF16: emit_counts_kernel<OpFmt::BF16><<<grid, 256, 0, s>>>(counts, cnt_ld, vec, upop, P, n_tiles, col_snp, center_snp, rec_n, rec_nm1, op); break;
        case OpFmt::F16: emit_counts_kernel<OpFmt::F16><<<grid, 256, 0, s>>>(counts, cnt_ld, vec, upop, P, n_tiles, col_snp, center_snp, rec_n, rec_nm1, op); break;
        case OpFmt::FX: emit_counts_kernel<OpFmt::FX><<<grid, 256, 0, s>>>(counts, cnt_ld, vec, upop, P, n_tiles, col_snp, center_snp, rec_n, rec_nm1, op); break;
    }
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_copy_union_ploidy(Ctx& c, uint32_t* desc, const int32_t* umap, int64_t n_sel, const uint32_t* desc_u,
                              cudaStream_t s) {
    if (n_sel <= 0) return;
    copy_union_ploidy_kernel<<<static_cast<unsigned>((n_sel + 255) / 256), 256, 0, s>>>(desc, umap, n_sel, desc_u);
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
}

void launch_decode_canon(Ctx& c, const CanonDecodeArgs& a, cudaStream_t s) {
    if (a.P <= 0 || a.n_tiles <= 0) return;
    const dim3 grid(static_cast<unsigned>((a.n_tiles + 3) / 4), static_cast<unsigned>((a.P + kDecPops - 1) / kDecPops));
#define STPF2_DECODE_ARGS a.canon, a.n_tiles, a.n_sel, a.sel, a.pop_off, a.P, a.center, a.rec_n, a.rec_nm1, a.col_snp, \
                          a.col_base, a.op, a.cnt_ac2, a.cnt_n, a.umap, a.center_snp, a.cnt_packed, a.cnt_ld, a.fold_order
#define STPF2_DECODE_LAUNCH(F)                                                                      \
    (a.umap ? decode_canon_kernel<F, true><<<grid, kDecThreads2, kDecSmemBytes, s>>>(STPF2_DECODE_ARGS) \
            : decode_canon_kernel<F, false><<<grid, kDecThreads2, kDecSmemBytes, s>>>(STPF2_DECODE_ARGS))
    if (a.umap && !a.center_snp) fail(STP_INVALID_ARGUMENT, "shared-canonical decode needs per-SNP centres");
    switch (a.op.fmt) {
        case OpFmt::F32: STPF2_DECODE_LAUNCH(OpFmt::F32); break;
        case OpFmt::BF16: STPF2_DECODE_LAUNCH(OpFmt::BF16); break;
        case OpFmt::F16: STPF2_DECODE_LAUNCH(OpFmt::F16); break;
        case OpFmt::FX: STPF2_DECODE_LAUNCH(OpFmt::FX); break;
    }
#undef STPF2_DECODE_LAUNCH
#undef STPF2_DECODE_ARGS
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
        case OpFmt::FX: feed_qvn_kernel<OpFmt::FX><<<grid, block, 0, s>>>(Q, V, N, P, M, snp_col, center, op); break;
    }
    STPF2_CUDA(cudaGetLastError());
    c.launches++;
    STPF2_CUDA(cudaFreeAsync(center, s));
}


}  // namespace stpf2
