// Persistent, warp-specialised SHGEMM tile kernel for sm_100a.
//
// C = alpha * op(A) * op(B) + beta * C, A FP32, B binary16, column-major.
// The error-corrected method of the reference (src/wmmae_shgemm.hpp:11-125):
// the FP32 operand is split on the fly into hi = T(a) and lo = T(2^11 (a - hi))
// with T = binary16 or TF32, and hi*B and lo*B are issued as tensor-core MMAs.
// The reference forms every k-fragment's hi product in a zeroed accumulator and
// adds it to its FP32 running sum with a round-to-nearest add, avoiding the
// tensor core's truncating accumulation; lo accumulates on the tensor core and
// is folded in as hi + lo * 2^-11 (tcec store_matrix_sync, src/shgemm.cu:87-99).
//
// Here every k-step (one 128-byte swizzle row: 64 binary16 / 32 TF32 values of
// k, four UMMA instructions per operand) is one drain chunk:
//   D  = sum lo*B            (4 UMMAs into a fresh TMEM accumulator)
//   D  = hi_0*B + D * 2^-11  (UMMA with scale-input-d = 11)
//   D += hi_k*B              (3 more UMMAs)
// so D holds the chunk's hi product plus its 2^-11-scaled lo product; the
// epilogue warps drain D from TMEM every chunk and add it to FP32 registers
// with round-to-nearest adds. D is double-buffered in TMEM (2 x BN columns),
// so the next chunk's MMAs overlap the drain. The epilogue applies alpha/beta
// like src/dmem_accessor.hpp:187-356 (C is not read when beta == 0) or, for
// split-K, writes the slice's partial to a workspace that a separate kernel
// reduces in fixed slice order.
//
// Warp roles (512 threads, one CTA per SM, registers rebalanced per warpgroup):
//   warp 0       TMA producer: raw FP32 A tile and binary16 B tile per k-step
//   warp 1       TMEM allocator + single-thread UMMA issuer
//   warps 2-7    split: turn the raw FP32 tile, in place, into 128B-swizzled
//                hi/lo UMMA tiles (K-major when A is K-contiguous, MN-major for
//                binary16 when it is M-contiguous) and, for TF32, widen B in place
//   warps 8-15   epilogue: TMEM lane quadrant (warp % 4) x column half
// Rings: A stages (TMA -> split in place -> MMA), B stages (TMA -> MMA; for TF32
// TMA -> widen in place -> MMA), D (MMA <-> epilogue). A stage is 32 KB: the raw
// FP32 tile and the hi + lo tiles have the same size (binary16) or fit in it
// (TF32), so the split reads its whole share into registers, waits until every
// split thread has done so, then overwrites the stage. Every wait is bounded; on
// timeout the kernel records an error code, drains its own in-flight copies and
// MMAs, frees TMEM and exits.
#pragma once
#include "ptx.cuh"

namespace shgemm_b200 {

enum : int { kOpN = 0, kOpT = 1 };
enum : int { kFP16 = 0, kTF32 = 1 };

enum : int {
    kErrNone = 0,
    kErrProducerTimeout = 1,
    kErrMmaTimeout = 2,
    kErrSplitTimeout = 3,
    kErrEpilogueTimeout = 4,
    kErrDrainTimeout = 5,
};

struct alignas(64) TileGemmParams {
    CUtensorMap tmap_a;  // FP32 operand
    CUtensorMap tmap_b;  // binary16 operand
    float* c;
    uint64_t ldc;
    float* workspace;  // split-K partials: [slice][n][m] (ld = m)
    int* error_flag;
    uint64_t wait_limit_ns;
    int m, n, k;
    int op_c;
    float alpha, beta;
    // Device-resident scalars (both null: alpha and beta above). Read when a tile's epilogue
    // starts, so a captured launch picks up whatever the caller stored there since.
    const float* alpha_dev;
    const float* beta_dev;
    int tiles_m, tiles_n;
    int num_slices;       // split-K slices (1: the epilogue writes C)
    int steps_per_slice;  // k-steps per slice
    int num_units;        // tiles_m * tiles_n * num_slices
    int group_m;          // rasterisation group along m
    // Tensor-memory kernel, K-major FP32 operand: tmap_a is a 3-D view {32 floats, k / 32, m}
    // whose box {32, 2, 128} lands each row's 64 floats of a k-step in two adjacent 128-byte
    // segments (row r, k-half h at segment 2 r + h). 0: two 2-D boxes {32, 128}, one per
    // k-half (segment 128 h + r).
    int a_rows_paired;
    // Tensor-memory kernel: every FP32 tile is read by one unit only (a single tile column),
    // so its loads carry an evict-first L2 hint and leave L2 to the shared binary16 tiles.
    int a_read_once;
    // tmap_b is a 3-D view {BK, n, k / BK} of B re-laid out as contiguous k-blocks (the
    // binary16 operand for the tensor-memory kernel, BK = 64; the widened FP32 operand for
    // the widened-B TF32 kernel, BK = 32); a step loads box (0, bn tn, step).
    int b_blocked;
};

// B_WIDE (TF32 compute only): the binary16 operand arrives already widened to FP32
// (K-major), so it is loaded straight into the TF32 tile layout and the split warps
// handle the FP32 operand alone.
template <int TC, int BN_, bool A_KMAJOR, bool B_KMAJOR, bool B_WIDE = false>
struct TileCfg {
    static constexpr int BM = 128;
    static constexpr int BN = BN_;
    static constexpr bool kTf32 = (TC == kTF32);
    static constexpr bool kBWide = B_WIDE;
    // split warps work on independent items, each converted in place by one warp
    static constexpr bool kItemSplit = !kTf32 || kBWide;
    static constexpr int BK = kTf32 ? 32 : 64;  // one 128-byte swizzle row of the compute type
    static constexpr int UMMA_K = kTf32 ? 8 : 16;
    static constexpr int KSUB = BK / UMMA_K;  // UMMAs per operand per k-step
    static constexpr int A_RAW = BM * BK * 4;
    static constexpr int B_RAW = BN * BK * (kBWide ? 4 : 2);
    static constexpr int HI_BYTES = BM * 128;  // BM rows of 128 bytes (both modes)
    static constexpr int A_STAGE = 2 * HI_BYTES;  // raw FP32 tile, then hi + lo tiles
    static constexpr int B_STAGE = BN * 128;      // binary16 tile; TF32: widened tile
    // Split items per stage. binary16: 8 rows x 64 k of a K-major tile, or 8 k x 64 m of an
    // M-major one. TF32 (B_WIDE): 8 rows x 32 k of a K-major tile, or one [32 k][32 m] box of
    // an M-major one.
    static constexpr int SPLIT_ITEMS = (kTf32 && !A_KMAJOR) ? 4 : 16;
    // M-major raw A (binary16 compute): two [BK][64 m] boxes; hi/lo atoms of item
    // (k group g, m half h) at h * MN_HALF_BYTES + g * 2048 (+1024 for lo).
    static constexpr int MN_HALF_BYTES = BK * 64 * 4;
    // M-major raw A (TF32, B_WIDE): four [32 k][32 m] boxes of MN_BOX_BYTES.
    static constexpr int MN_BOX_BYTES = BK * 32 * 4;
    static constexpr int SMEM_BUDGET = 224 * 1024;
    static constexpr int SA = 4;
    static constexpr int SB_FIT = (SMEM_BUDGET - SA * A_STAGE) / B_STAGE;
    static constexpr int SB = SB_FIT > 6 ? 6 : SB_FIT;
    static_assert(SB >= 3, "shared memory budget");
    static constexpr int NUM_THREADS = 512;
    static constexpr int SPLIT_WARPS = 6;
    static constexpr int SPLIT_THREADS = 32 * SPLIT_WARPS;
    static constexpr int EPI_WARP0 = 8;
    static constexpr int TMEM_COLS = 2 * BN < 32 ? 32 : 2 * BN;  // D ping-pong
    static constexpr int HALF_N = BN / 2;                        // columns per epilogue warp
    // Per-thread registers after setmaxnreg: warpgroups 0-1 (producer, MMA, split) and
    // 2-3 (epilogue, which holds HALF_N running sums); 256 x (SPLIT_REGS + EPI_REGS) = 65536.
    static constexpr int SPLIT_REGS = BN == 256 ? 80 : 112;
    static constexpr int EPI_REGS = 256 - SPLIT_REGS;
    static constexpr int BAR_BYTES = 1024;
    static constexpr int SMEM_BYTES = SA * A_STAGE + SB * B_STAGE + BAR_BYTES + 1024;
    static_assert(BN == 64 || BN == 128 || (BN == 256 && (!kTf32 || kBWide)), "tile N");
    static_assert(!kBWide || (kTf32 && B_KMAJOR), "widened B: TF32 compute, K-major");
    static_assert(A_STAGE % 1024 == 0 && B_STAGE % 1024 == 0 && A_RAW <= A_STAGE, "1024B-aligned stages");
    static_assert(SMEM_BYTES <= 232448, "dynamic shared memory limit");
};

__device__ __forceinline__ void decode_unit(const TileGemmParams& p, int u, int& tm, int& tn, int& slice) {
    const int tiles = p.tiles_m * p.tiles_n;
    slice = u / tiles;
    const int r = u - slice * tiles;
    const int group_size = p.group_m * p.tiles_n;
    const int g = r / group_size;
    const int first_m = g * p.group_m;
    const int gm = min(p.tiles_m - first_m, p.group_m);
    const int rr = r - g * group_size;
    tm = first_m + rr % gm;
    tn = rr / gm;
}

__device__ __forceinline__ void step_range(const TileGemmParams& p, int slice, int total_steps, int& s0, int& s1) {
    s0 = slice * p.steps_per_slice;
    s1 = min(s0 + p.steps_per_slice, total_steps);
}

// One grouped problem: C (m x n) = alpha * op(A) * op(B) + beta * C, with its TMA
// descriptors; built on the host and copied to device memory before the launch.
struct alignas(64) GroupedProblem {
    CUtensorMap tmap_a;
    CUtensorMap tmap_b;
    float* c;
    uint64_t ldc;
    int m, n, k;
    int bn;     // tile N of this problem (<= the kernel's BN; 16-multiple)
    int steps;  // k-steps
    float alpha, beta;
    int b_gen;          // 1: B is the block-sign Rademacher operand of gen_seed (entries +-1), written
    int pad0;           //    by the split warps instead of loaded (binary16 compute); tmap_b unused
    uint64_t gen_seed;
};
static_assert(sizeof(GroupedProblem) % 64 == 0, "GroupedProblem alignment");

struct alignas(64) GroupedParams {
    const GroupedProblem* problems;
    const int2* units;      // {problem, tm | tn << 16}, longest first
    const int* num_units;   // in device memory: a captured graph relaunches with new tables
    int* error_flag;
    uint64_t wait_limit_ns;
    int op_c;
    // Device-resident scalars for every problem of the launch (both null: each problem's
    // alpha and beta), read once by each epilogue warp when the kernel starts.
    const float* alpha_dev;
    const float* beta_dev;
    // The next unit to hand out after each CTA's first (blockIdx.x): a counter in device
    // memory, zeroed by the table copy that precedes every launch (and every graph replay).
    int* next_unit;
};

// What one work unit (a 128 x bn tile of one problem over a range of k-steps) needs.
struct UnitDesc {
    const CUtensorMap* tmap_a;
    const CUtensorMap* tmap_b;
    float* c;
    uint64_t ldc;
    float* partial;  // split-K: this slice's partial buffer [n][m]; null: write C
    int m, n, k;
    int tm, tn;
    int s0, s1;  // k-step range
    int bn;      // tile N
    float alpha, beta;
    bool maps_in_global;  // descriptors written by a copy before the launch
    bool b_gen;           // B generated by the producer (block-sign Rademacher, gen_seed)
    uint64_t gen_seed;
};

// Device-resident alpha and beta of a launch, read once per epilogue warp; `on` false when
// the launch passes host scalars (each unit's alpha and beta then apply).
struct DevScalarValues {
    bool on;
    float alpha, beta;
};
template <class Params>
__device__ __forceinline__ DevScalarValues load_dev_scalars(const Params& p) {
    DevScalarValues v{p.alpha_dev != nullptr, 0.0f, 0.0f};
    if (v.on) {
        v.alpha = *p.alpha_dev;
        v.beta = *p.beta_dev;
    }
    return v;
}

template <class Cfg>
__device__ __forceinline__ void get_unit(const TileGemmParams& p, int u, UnitDesc& d) {
    int tm, tn, slice, s0, s1;
    decode_unit(p, u, tm, tn, slice);
    step_range(p, slice, (p.k + Cfg::BK - 1) / Cfg::BK, s0, s1);
    d.tmap_a = &p.tmap_a;
    d.tmap_b = &p.tmap_b;
    d.c = p.c;
    d.ldc = p.ldc;
    d.partial = p.num_slices > 1 ? p.workspace + static_cast<size_t>(slice) * p.n * p.m : nullptr;
    d.m = p.m;
    d.n = p.n;
    d.k = p.k;
    d.b_gen = false;
    d.gen_seed = 0;
    d.tm = tm;
    d.tn = tn;
    d.s0 = s0;
    d.s1 = s1;
    d.bn = Cfg::BN;
    d.alpha = p.alpha;
    d.beta = p.beta;
    d.maps_in_global = false;
}

template <class Cfg>
__device__ __forceinline__ void get_unit(const GroupedParams& p, int u, UnitDesc& d) {
    const int2 e = p.units[u];
    const GroupedProblem& q = p.problems[e.x];
    d.tmap_a = &q.tmap_a;
    d.tmap_b = &q.tmap_b;
    d.c = q.c;
    d.ldc = q.ldc;
    d.partial = nullptr;
    d.m = q.m;
    d.n = q.n;
    d.k = q.k;
    d.b_gen = q.b_gen != 0;
    d.gen_seed = q.gen_seed;
    d.tm = e.y & 0xFFFF;
    d.tn = e.y >> 16;
    d.s0 = 0;
    d.s1 = q.steps;
    d.bn = q.bn;
    d.alpha = q.alpha;
    d.beta = q.beta;
    d.maps_in_global = true;
}

__device__ __forceinline__ int unit_count(const TileGemmParams& p) { return p.num_units; }
__device__ __forceinline__ int unit_count(const GroupedParams& p) { return *p.num_units; }

// The k-th unit (k = 0, 1, ...) a CTA works on, or -1 when none is left. A single problem's
// units are uniform: CTA b takes b, b + gridDim.x, ... Grouped units are uneven (their k and
// tile N differ): after its first unit a CTA takes the next one from a device counter when
// its producer is ready for it, so the units balance by their actual time rather than by an
// estimate (the list is still longest first).
__device__ __forceinline__ int claim_unit(const TileGemmParams& p, int k) {
    const long long u = blockIdx.x + static_cast<long long>(k) * gridDim.x;
    return u < p.num_units ? static_cast<int>(u) : -1;
}
__device__ __forceinline__ int claim_unit(const GroupedParams& p, int k) {
    const int u = k == 0 ? static_cast<int>(blockIdx.x) : static_cast<int>(gridDim.x) + atomicAdd(p.next_unit, 1);
    return u < *p.num_units ? u : -1;
}
__device__ __forceinline__ int output_op(const TileGemmParams& p) { return p.op_c; }
__device__ __forceinline__ bool b_blocked(const TileGemmParams& p) { return p.b_blocked != 0; }
__device__ __forceinline__ bool b_blocked(const GroupedParams&) { return false; }
__device__ __forceinline__ int output_op(const GroupedParams& p) { return p.op_c; }
__device__ __forceinline__ void prefetch_params_maps(const TileGemmParams& p) {
    ptx::tma_prefetch_desc(&p.tmap_a);
    ptx::tma_prefetch_desc(&p.tmap_b);
}
__device__ __forceinline__ void prefetch_params_maps(const GroupedParams&) {}

// ---------------------------------------------------------------------------
// Counter hash for generated sketch operands: splitmix64's finaliser (Steele, Lea and Flood,
// "Fast splittable pseudorandom number generators", OOPSLA 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// 64 sign bits of a block-sign Rademacher operand: entries 64 b .. 64 b + 63 of column c of a
// k x n operand, block index c * ceil(k / 64) + b; entry 64 b + r is negative when bit
// block_sign_bit(r) is set.
__device__ __forceinline__ uint64_t rademacher_block_bits(uint64_t seed, uint64_t block) {
    return mix64(seed * 0x9E3779B97F4A7C15ull + block + 1);
}

// The bit of a block's hash that gives the sign of entry r (0..63) of the block: entries 2p
// and 2p + 1 take bits (p mod 16) and (p mod 16) + 16 of 32-bit half p / 16, so the two
// binary16 values of a 32-bit word come from bits 16 apart (one shift and one mask a word).
__host__ __device__ __forceinline__ int block_sign_bit(int r) {
    return 32 * (r >> 5) + ((r >> 1) & 15) + 16 * (r & 1);
}

// ---------------------------------------------------------------------------
// Epilogue helpers.
// Element (row, col) of C: column-major (op_c = N) or stored transposed (op_c = T).
__device__ __forceinline__ float* c_elem(float* c, uint64_t ldc, int op_c, int row, int col) {
    return op_c == kOpN ? c + row + static_cast<size_t>(col) * ldc : c + static_cast<size_t>(row) * ldc + col;
}

// C(row, col0 .. col0 + NC - 1) = alpha * acc(j) + beta * C (C not read when beta == 0);
// columns at or past n are skipped. With beta != 0 the C values of 4 columns are loaded
// before any of them is written, so the loads' latencies overlap instead of adding up.
template <int NC, class AccFn>
__device__ __forceinline__ void store_row(float* c, uint64_t ldc, int op_c, int row, int col0, int n, float alpha,
                                          float beta, AccFn&& acc) {
    const size_t stride = op_c == kOpN ? ldc : 1;
    float* p = c_elem(c, ldc, op_c, row, col0);
    if (beta == 0.0f) {
#pragma unroll
        for (int j = 0; j < NC; ++j)
            if (col0 + j < n) p[j * stride] = __fmul_rn(acc(j), alpha);
        return;
    }
#pragma unroll
    for (int jb = 0; jb < NC; jb += 4) {
        float cv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) cv[j] = (col0 + jb + j < n) ? p[(jb + j) * stride] : 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (col0 + jb + j < n) p[(jb + j) * stride] = __fmaf_rn(acc(jb + j), alpha, __fmul_rn(beta, cv[j]));
    }
}

// Asks L2 to fetch and keep the lines of C(row, col0 .. col0 + NC - 1) ahead of a
// beta != 0 epilogue.
template <int NC>
__device__ __forceinline__ void prefetch_row(float* c, uint64_t ldc, int op_c, int row, int col0, int n) {
    // op_c = N: a warp's 32 consecutive rows share each column's line; T: a row's columns
    // are contiguous, one line per 32 columns
    const int step = op_c == kOpN ? 1 : 32;
#pragma unroll 1
    for (int j = 0; j < NC; j += step)
        if (col0 + j < n) ptx::prefetch_l2_evict_last(c_elem(c, ldc, op_c, row, col0 + j));
}

// ---------------------------------------------------------------------------
// Split helpers. hi = T(v), lo = T(2^11 (v - hi)), T = binary16 round-to-nearest-
// even or TF32 round-to-nearest-away: the reference's split (src/wmmae_shgemm.hpp:30-31).
__device__ __forceinline__ void split8_f16(const float (&v)[8], uint4& hi, uint4& lo) {
    const uint64_t scale = ptx::f2_pack(2048.0f, 2048.0f);
    uint32_t h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const __half2 hh = __floats2half2_rn(v[2 * e], v[2 * e + 1]);
        const float2 hf = __half22float2(hh);
        // (v - hi) is exact and the 2^11 scaling is exact: lo = T(2^11 (v - hi))
        const uint64_t d = ptx::f2_mul(ptx::f2_sub(ptx::f2_pack(v[2 * e], v[2 * e + 1]), ptx::f2_pack(hf.x, hf.y)),
                                       scale);
        const __half2 ll = __floats2half2_rn(ptx::f2_lo(d), ptx::f2_hi(d));
        h[e] = *reinterpret_cast<const uint32_t*>(&hh);
        l[e] = *reinterpret_cast<const uint32_t*>(&ll);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

__device__ __forceinline__ void split4_tf32(const float4 x, float4& hi, float4& lo) {
    hi.x = ptx::to_tf32_rna(x.x);
    hi.y = ptx::to_tf32_rna(x.y);
    hi.z = ptx::to_tf32_rna(x.z);
    hi.w = ptx::to_tf32_rna(x.w);
    const uint64_t scale = ptx::f2_pack(2048.0f, 2048.0f);
    const uint64_t d0 = ptx::f2_mul(ptx::f2_sub(ptx::f2_pack(x.x, x.y), ptx::f2_pack(hi.x, hi.y)), scale);
    const uint64_t d1 = ptx::f2_mul(ptx::f2_sub(ptx::f2_pack(x.z, x.w), ptx::f2_pack(hi.z, hi.w)), scale);
    lo.x = ptx::to_tf32_rna(ptx::f2_lo(d0));
    lo.y = ptx::to_tf32_rna(ptx::f2_hi(d0));
    lo.z = ptx::to_tf32_rna(ptx::f2_lo(d1));
    lo.w = ptx::to_tf32_rna(ptx::f2_hi(d1));
}

// binary16 compute: one split item, converted in place by one warp.
// K-major A (item = rows 8i .. 8i+7): the raw tile is two [128 rows][32 floats] 128B-swizzled
// sub-tiles (k 0-31, 32-63); hi row r replaces raw row r of the first, lo row r that of the
// second, both [64 halves] K-major with a 128-byte swizzle.
// M-major A (item = k group g = i & 7 of m half h = i >> 3): the raw tile is two [64 k][64 m]
// boxes (256-byte rows); the item's 8 raw rows (2 KB) become its hi atom (8 k x 64 m halves,
// 128B swizzle) and, 1 KB above it, its lo atom.
// Lane l covers output chunks (16 bytes, 8 values) chosen so that each group of 8 lanes
// touches 8 distinct 16-byte bank groups on every load and store.
template <class Cfg, bool A_KMAJOR>
__device__ __forceinline__ void split_item_load(const uint8_t* st, int item, int lane, float4 (&x)[4]) {
    if constexpr (A_KMAJOR) {
        const int row = item * 8 + (lane & 7), cb = lane >> 3, sw = lane & 7;
        const uint8_t* r0 = st + row * 128;
        const uint8_t* r1 = r0 + Cfg::BM * 128;
        x[0] = *reinterpret_cast<const float4*>(r0 + (((2 * cb) ^ sw) << 4));
        x[1] = *reinterpret_cast<const float4*>(r0 + (((2 * cb + 1) ^ sw) << 4));
        x[2] = *reinterpret_cast<const float4*>(r1 + (((2 * cb) ^ sw) << 4));
        x[3] = *reinterpret_cast<const float4*>(r1 + (((2 * cb + 1) ^ sw) << 4));
    } else {
        const uint8_t* base = st + (item >> 3) * Cfg::MN_HALF_BYTES + (item & 7) * 2048;
        const int c = lane & 7, first = (c >> 2) & 1;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint8_t* rp = base + ((lane >> 3) + 4 * h) * 256 + c * 32;
            const float4 xa = *reinterpret_cast<const float4*>(rp + 16 * first);
            const float4 xb = *reinterpret_cast<const float4*>(rp + 16 * (1 - first));
            x[2 * h] = first ? xb : xa;
            x[2 * h + 1] = first ? xa : xb;
        }
    }
}

template <class Cfg, bool A_KMAJOR>
__device__ __forceinline__ void split_item_store(uint8_t* st, int item, int lane, const float4 (&x)[4]) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const float v[8] = {x[2 * h].x, x[2 * h].y, x[2 * h].z, x[2 * h].w,
                            x[2 * h + 1].x, x[2 * h + 1].y, x[2 * h + 1].z, x[2 * h + 1].w};
        uint4 hv, lv;
        split8_f16(v, hv, lv);
        uint8_t* hp;
        uint8_t* lp;
        if constexpr (A_KMAJOR) {
            const int row = item * 8 + (lane & 7), c = (lane >> 3) + 4 * h, sw = lane & 7;
            hp = st + row * 128 + ((c ^ sw) << 4);
            lp = hp + Cfg::BM * 128;
        } else {
            const int r = (lane >> 3) + 4 * h, c = lane & 7;
            hp = st + (item >> 3) * Cfg::MN_HALF_BYTES + (item & 7) * 2048 + r * 128 + ((c ^ r) << 4);
            lp = hp + 1024;
        }
        *reinterpret_cast<uint4*>(hp) = hv;
        *reinterpret_cast<uint4*>(lp) = lv;
    }
}

// The items i = first, first + SPLIT_WARPS, ... of one stage (binary16 compute). An item's
// outputs overwrite only its own raw bytes, so a warp needs no other warp to have read the
// stage: __syncwarp orders its lanes' loads before their stores. The next item's loads are
// issued before the current item's conversion.
template <class Cfg, bool A_KMAJOR>
__device__ __forceinline__ void split_stage_f16(uint8_t* st, int first, int lane) {
    float4 cur[4];
    split_item_load<Cfg, A_KMAJOR>(st, first, lane, cur);
    for (int it = first; it < Cfg::SPLIT_ITEMS; it += Cfg::SPLIT_WARPS) {
        float4 nxt[4];
        const bool more = it + Cfg::SPLIT_WARPS < Cfg::SPLIT_ITEMS;
        if (more) split_item_load<Cfg, A_KMAJOR>(st, it + Cfg::SPLIT_WARPS, lane, nxt);
        __syncwarp();
        split_item_store<Cfg, A_KMAJOR>(st, it, lane, cur);
        if (more) {
#pragma unroll
            for (int e = 0; e < 4; ++e) cur[e] = nxt[e];
        }
    }
}

// TF32 compute with a widened B: the items of one stage.
// K-major A (item = rows 8i .. 8i+7 of the [128 rows][32 floats] 128B-swizzled raw tile):
// each lane converts two 16-byte chunks in place (hi) and writes lo at the same offset
// HI_BYTES above; no lane reads what another writes.
// M-major A (item = box i, [32 k][32 m] floats with 128-byte rows at i * MN_BOX_BYTES):
// lane l gathers column m = 32 i + l, then (after __syncwarp) writes hi row m over the
// box, [32 TF32] K-major with a 128-byte swizzle, and lo row m HI_BYTES above.
template <class Cfg, bool A_KMAJOR>
__device__ __forceinline__ void split_stage_tf32w(uint8_t* st, int first, int lane) {
    for (int it = first; it < Cfg::SPLIT_ITEMS; it += Cfg::SPLIT_WARPS) {
        if constexpr (A_KMAJOR) {
            const int row = it * 8 + (lane & 7), sw = lane & 7;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint8_t* p = st + row * 128 + ((((lane >> 3) + 4 * h) ^ sw) << 4);
                float4 hv, lv;
                split4_tf32(*reinterpret_cast<const float4*>(p), hv, lv);
                *reinterpret_cast<float4*>(p) = hv;
                *reinterpret_cast<float4*>(p + Cfg::HI_BYTES) = lv;
            }
        } else {
            uint8_t* box = st + it * Cfg::MN_BOX_BYTES;
            float v[32];
#pragma unroll
            for (int k = 0; k < 32; ++k) v[k] = *reinterpret_cast<const float*>(box + k * 128 + lane * 4);
            __syncwarp();
            const int m = it * 32 + lane;
            uint8_t* hp = st + m * 128;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float4 hv, lv;
                split4_tf32(make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]), hv, lv);
                const int off = (j ^ (m & 7)) << 4;
                *reinterpret_cast<float4*>(hp + off) = hv;
                *reinterpret_cast<float4*>(hp + Cfg::HI_BYTES + off) = lv;
            }
        }
    }
}

// TF32 compute: one k-step of the split warps (thread sidx of SPLIT_THREADS), in place:
// phase 1 reads this thread's share of the raw tiles into registers;
// `all_read()` returns once every split thread has done so (false on timeout);
// phase 2 converts and overwrites the stages with the UMMA tiles:
//   A stage: hi at [0, HI_BYTES), lo at [HI_BYTES, 2 HI_BYTES)
//   B stage: the widened [BN][32] TF32 tile.
template <class Cfg, bool A_KMAJOR, bool B_KMAJOR, class AllRead>
__device__ __forceinline__ bool split_step_tf32(uint8_t* a_st, uint8_t* b_st, int sidx, AllRead&& all_read) {
    constexpr int NT = Cfg::SPLIT_THREADS;
    uint8_t* hi_t = a_st;
    uint8_t* lo_t = a_st + Cfg::HI_BYTES;
    constexpr int BN = Cfg::BN;
    // ---- phase 1: A
    constexpr int UA = A_KMAJOR ? (1024 + NT - 1) / NT : (256 + NT - 1) / NT;
    float4 xa[UA][A_KMAJOR ? 1 : 4];
#pragma unroll
    for (int j = 0; j < UA; ++j) {
        const int u = sidx + j * NT;
        if constexpr (A_KMAJOR) {
            // raw: [128 rows][32 floats] 128B-swizzled. Unit: (row, 16-byte chunk c).
            if (u < 1024) {
                const int row = u & 127, c = u >> 7;
                xa[j][0] = *reinterpret_cast<const float4*>(a_st + row * 128 + ((c ^ (row & 7)) << 4));
            }
        } else {
            // raw: [32 k][128 m] floats. Unit: (m group g of 4, k group kq of 4).
            if (u < 256) {
                const int g = u & 31, kq = u >> 5;
#pragma unroll
                for (int r = 0; r < 4; ++r)
                    xa[j][r] = *reinterpret_cast<const float4*>(a_st + (kq * 4 + r) * 512 + g * 16);
            }
        }
    }
    // ---- phase 1: B (binary16, exact in TF32)
    constexpr int UB = B_KMAJOR ? (BN * 4 + NT - 1) / NT : (BN * 8 + NT - 1) / NT;
    uint4 xb_k[B_KMAJOR ? UB : 1];
    uint2 xb_m[B_KMAJOR ? 1 : UB];
#pragma unroll
    for (int j = 0; j < UB; ++j) {
        const int u = sidx + j * NT;
        if constexpr (B_KMAJOR) {
            // raw: [BN][32] binary16, 64-byte rows, 64B swizzle. Unit: (row n, raw chunk rc).
            if (u < BN * 4) {
                const int n = u % BN, rc = u / BN;
                xb_k[j] = *reinterpret_cast<const uint4*>(b_st + n * 64 + ((rc ^ ((n >> 1) & 3)) << 4));
            }
        } else {
            // raw: [32 k][BN] binary16. Unit: (column n, output chunk c = k 4c .. 4c+3).
            if (u < BN * 8) {
                const int n = u % BN, c = u / BN;
                const uint16_t* bh = reinterpret_cast<const uint16_t*>(b_st);
                xb_m[j].x = uint32_t(bh[(c * 4 + 0) * BN + n]) | (uint32_t(bh[(c * 4 + 1) * BN + n]) << 16);
                xb_m[j].y = uint32_t(bh[(c * 4 + 2) * BN + n]) | (uint32_t(bh[(c * 4 + 3) * BN + n]) << 16);
            }
        }
    }
    if (!all_read()) return false;
    // ---- phase 2: A -> hi/lo [128 rows][32] TF32, K-major, 128B swizzle
#pragma unroll
    for (int j = 0; j < UA; ++j) {
        const int u = sidx + j * NT;
        if constexpr (A_KMAJOR) {
            if (u < 1024) {
                const int row = u & 127, c = u >> 7;
                const int off = row * 128 + ((c ^ (row & 7)) << 4);
                float4 h, l;
                split4_tf32(xa[j][0], h, l);
                *reinterpret_cast<float4*>(hi_t + off) = h;
                *reinterpret_cast<float4*>(lo_t + off) = l;
            }
        } else {
            if (u < 256) {
                const int g = u & 31, kq = u >> 5;
                float4 h[4], l[4];  // h[r]: k = 4kq + r, m = 4g .. 4g+3
#pragma unroll
                for (int r = 0; r < 4; ++r) split4_tf32(xa[j][r], h[r], l[r]);
                // transpose 4 x 4; rotate the row order so 8-thread store phases
                // hit distinct 16-byte bank groups
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int rr = (r + (g >> 1)) & 3;
                    const int row = 4 * g + rr;
                    const float4 hv = rr == 0   ? make_float4(h[0].x, h[1].x, h[2].x, h[3].x)
                                      : rr == 1 ? make_float4(h[0].y, h[1].y, h[2].y, h[3].y)
                                      : rr == 2 ? make_float4(h[0].z, h[1].z, h[2].z, h[3].z)
                                                : make_float4(h[0].w, h[1].w, h[2].w, h[3].w);
                    const float4 lv = rr == 0   ? make_float4(l[0].x, l[1].x, l[2].x, l[3].x)
                                      : rr == 1 ? make_float4(l[0].y, l[1].y, l[2].y, l[3].y)
                                      : rr == 2 ? make_float4(l[0].z, l[1].z, l[2].z, l[3].z)
                                                : make_float4(l[0].w, l[1].w, l[2].w, l[3].w);
                    const int off = row * 128 + ((kq ^ (row & 7)) << 4);
                    *reinterpret_cast<float4*>(hi_t + off) = hv;
                    *reinterpret_cast<float4*>(lo_t + off) = lv;
                }
            }
        }
    }
    // ---- phase 2: B -> [BN][32] TF32, K-major, 128B swizzle
#pragma unroll
    for (int j = 0; j < UB; ++j) {
        const int u = sidx + j * NT;
        if constexpr (B_KMAJOR) {
            if (u < BN * 4) {
                const int n = u % BN, rc = u / BN, sw = n & 7;
                const __half2* hp = reinterpret_cast<const __half2*>(&xb_k[j]);
                const float2 f0 = __half22float2(hp[0]);
                const float2 f1 = __half22float2(hp[1]);
                const float2 f2 = __half22float2(hp[2]);
                const float2 f3 = __half22float2(hp[3]);
                *reinterpret_cast<float4*>(b_st + n * 128 + (((2 * rc) ^ sw) << 4)) =
                    make_float4(f0.x, f0.y, f1.x, f1.y);
                *reinterpret_cast<float4*>(b_st + n * 128 + (((2 * rc + 1) ^ sw) << 4)) =
                    make_float4(f2.x, f2.y, f3.x, f3.y);
            }
        } else {
            if (u < BN * 8) {
                const int n = u % BN, c = u / BN;
                const __half2* hp = reinterpret_cast<const __half2*>(&xb_m[j]);
                const float2 f0 = __half22float2(hp[0]);
                const float2 f1 = __half22float2(hp[1]);
                *reinterpret_cast<float4*>(b_st + n * 128 + ((c ^ (n & 7)) << 4)) =
                    make_float4(f0.x, f0.y, f1.x, f1.y);
            }
        }
    }
    return true;
}

// Two binary16 values +1 / -1 (0x3C00 / 0xBC00) as one 32-bit word: the sign of the low
// half is bit i of h, the sign of the high half bit i + 16 (i < 16). One shift and one masked
// OR per word: this pairing of bits 16 apart is why the block-sign stream orders its bits as
// block_sign_bit says.
__device__ __forceinline__ uint32_t sign_pair_word(uint32_t h, int i) {
    return ((h << (15 - i)) & 0x80008000u) | 0x3C003C00u;
}

// What the generator needs of a unit: its first B column, tile N, n, k and seed.
struct GenB {
    uint64_t seed;
    int c0, bn, n, k;
};

// One k-step (64 k) of a generated B stage, rows j = t0, t0 + nthreads, ... < bn (columns
// c0 + j of the k x n block-sign operand): each row 64 binary16 values K-major in the
// 128-byte-swizzled layout the TMA would have written (16-byte chunk q of row j at chunk
// q ^ (j & 7)). Entries past n or past k are zero, as the TMA's out-of-range fill. Entry r of
// the row is word r / 2 of the chunk sequence; word p = 4 q + e takes bits (p mod 16) and
// (p mod 16) + 16 of 32-bit half p / 16 of the block's hash (block_sign_bit).
__device__ __forceinline__ void gen_b_rows(uint8_t* stage, const GenB& ud, int st, int t0, int nthreads) {
    const int c0 = ud.c0;
    const int kvalid = ud.k - st * 64;  // >= 1 on every step of the range
    const uint64_t kblocks = static_cast<uint64_t>((ud.k + 63) / 64);
    for (int j = t0; j < ud.bn; j += nthreads) {
        const int c = c0 + j;
        uint8_t* row = stage + j * 128;
        const int sw = j & 7;
        uint32_t h0 = 0, h1 = 0, on = 0;
        if (c < ud.n) {
            const uint64_t bits = rademacher_block_bits(ud.seed, static_cast<uint64_t>(c) * kblocks + st);
            h0 = static_cast<uint32_t>(bits);
            h1 = static_cast<uint32_t>(bits >> 32);
            on = ~0u;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t h = q < 4 ? h0 : h1;
            const int i = 4 * (q & 3);
            *reinterpret_cast<uint4*>(row + ((q ^ sw) << 4)) =
                make_uint4(sign_pair_word(h, i) & on, sign_pair_word(h, i + 1) & on, sign_pair_word(h, i + 2) & on,
                           sign_pair_word(h, i + 3) & on);
        }
        // the last k-step's ragged edge: entries r >= kvalid are zero
        for (int r = kvalid; r < 64; ++r)
            *reinterpret_cast<uint16_t*>(row + (((r >> 3) ^ sw) << 4) + (r & 7) * 2) = 0;
    }
}

// GEN_B (grouped binary16 launches with a K-major B): problems may ask for their B to be
// generated (block-sign Rademacher) instead of loaded. The split warps write those B stages,
// spread over their 192 threads, before they wait for the same k-step's A; the TMA producer
// skips them. A B stage then completes on the split warps' arrivals (one per warp) or on the
// producer's TMA (expect_tx plus the same number of arrivals).
template <int TC, int BN, bool A_KMAJOR, bool B_KMAJOR, bool B_WIDE, bool GEN_B, class Params>
__device__ __forceinline__ void tile_kernel_body(const Params& p) {
    using Cfg = TileCfg<TC, BN, A_KMAJOR, B_KMAJOR, B_WIDE>;
    static_assert(!GEN_B || (TC == kFP16 && B_KMAJOR), "generated B: binary16 compute, K-major B");
    constexpr int SA = Cfg::SA;
    constexpr int SB = Cfg::SB;
    constexpr bool kTf32 = Cfg::kTf32;
    constexpr int NSPLIT = Cfg::SPLIT_WARPS;

    extern __shared__ uint8_t smem_raw[];
    // 1024-byte alignment of the tile region (128B-swizzle atoms repeat every 1024 bytes).
    const uint32_t raw_s = ptx::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
    uint8_t* a_base = smem;
    uint8_t* b_base = a_base + SA * Cfg::A_STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(b_base + SB * Cfg::B_STAGE);
    uint64_t* a_full = bars;           // TMA landed the raw A tile
    uint64_t* a_read = a_full + SA;    // TF32: every split warp holds its share in registers
    uint64_t* a_split = a_read + SA;   // hi/lo tiles written (and, for TF32, B widened)
    uint64_t* a_empty = a_split + SA;  // MMAs reading the stage completed
    uint64_t* b_full = a_empty + SA;
    uint64_t* b_empty = b_full + SB;
    uint64_t* d_full = b_empty + SB;
    uint64_t* d_empty = d_full + 2;
    uint64_t* drain_bar = d_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    // per split warp: the current unit's generator parameters, past the barriers
    GenB* gen_slots = reinterpret_cast<GenB*>(reinterpret_cast<uint8_t*>(bars) + 512);
    // the producer claims each unit and hands it to the other roles through a 4-slot ring
    int* unit_ring = reinterpret_cast<int*>(reinterpret_cast<uint8_t*>(bars) + 768);
    uint64_t* unit_full = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(bars) + 800);
    uint64_t* unit_empty = unit_full + 4;
    constexpr uint32_t kUnitReaders = 1 + NSPLIT + 8;  // MMA issuer, split warps, epilogue warps
    static_assert((4 * SA + 2 * SB + 5) * 8 + 8 <= 512 && 512 + 8 * sizeof(GenB) <= 768 &&
                      800 + 8 * 8 <= Cfg::BAR_BYTES,
                  "barrier region");
    constexpr uint32_t kBFullCount = GEN_B ? NSPLIT : 1;

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < SA; ++s) {
            ptx::mbar_init(&a_full[s], 1);
            ptx::mbar_init(&a_read[s], NSPLIT);
            ptx::mbar_init(&a_split[s], NSPLIT);
            ptx::mbar_init(&a_empty[s], 1);
        }
        for (int s = 0; s < SB; ++s) {
            ptx::mbar_init(&b_full[s], kBFullCount);
            ptx::mbar_init(&b_empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            ptx::mbar_init(&d_full[b], 1);
            ptx::mbar_init(&d_empty[b], 8);
        }
        ptx::mbar_init(drain_bar, 1);
        for (int r = 0; r < 4; ++r) {
            ptx::mbar_init(&unit_full[r], 1);
            ptx::mbar_init(&unit_empty[r], kUnitReaders);
        }
        *abort_flag = 0;
        ptx::fence_mbarrier_init();
    }
    if (warp == 0 && lane == 0) prefetch_params_maps(p);
    if (warp == 1) {
        ptx::tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const uint64_t limit = p.wait_limit_ns;

    auto fail = [&](int code) {
        *abort_flag = 1;
        atomicCAS(p.error_flag, 0, code);
    };
    // the k-th unit from the producer's ring (false: the wait ran out); the caller then
    // releases the slot (one arrival per reading warp)
    auto take_unit = [&](int k, int& u) -> bool {
        if (!ptx::mbar_wait(&unit_full[k & 3], (k >> 2) & 1, abort_flag, limit)) return false;
        u = unit_ring[k & 3];
        return true;
    };

    // Warpgroups 0-1 (producer, MMA, split) give registers to warpgroups 2-3 (epilogue).
    if (warp < Cfg::EPI_WARP0) {
    ptx::setmaxnreg_dec<Cfg::SPLIT_REGS>();
    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            int as = 0, bs = 0;
            uint32_t aph = 0, bph = 0;
            uint32_t a_issued = 0, a_par = 0, b_issued = 0, b_par = 0;  // per stage: load in flight, its parity
            for (int uk = 0;; ++uk) {
                // claim the next unit and hand it to the other roles
                if (!ptx::mbar_wait(&unit_empty[uk & 3], ((uk >> 2) & 1) ^ 1u, abort_flag, limit)) {
                    fail(kErrProducerTimeout);
                    goto producer_done;
                }
                const int u = claim_unit(p, uk);
                unit_ring[uk & 3] = u;
                ptx::mbar_arrive(&unit_full[uk & 3]);
                if (u < 0) break;
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                const int tm = ud.tm, tn = ud.tn, s0 = ud.s0, s1 = ud.s1;
                if (ud.maps_in_global) {
                    ptx::fence_tensormap_acquire(ud.tmap_a);
                    if (!ud.b_gen) ptx::fence_tensormap_acquire(ud.tmap_b);
                }
                for (int st = s0; st < s1; ++st) {
                    const int kc = st * Cfg::BK;
                    {
                        if (!ptx::mbar_wait(&a_empty[as], aph ^ 1u, abort_flag, limit)) {
                            fail(kErrProducerTimeout);
                            goto producer_done;
                        }
                        {
                            uint8_t* a_dst = a_base + as * Cfg::A_STAGE;
                            ptx::mbar_arrive_expect_tx(&a_full[as], Cfg::A_RAW);
                            if constexpr (A_KMAJOR) {
#pragma unroll
                                for (int sub = 0; sub < Cfg::BK / 32; ++sub)
                                    ptx::tma_load_2d(a_dst + sub * (Cfg::BM * 128), ud.tmap_a, &a_full[as],
                                                     kc + 32 * sub, tm * Cfg::BM);
                            } else if constexpr (!kTf32) {
#pragma unroll
                                for (int h = 0; h < 2; ++h)
                                    ptx::tma_load_2d(a_dst + h * Cfg::MN_HALF_BYTES, ud.tmap_a, &a_full[as],
                                                     tm * Cfg::BM + 64 * h, kc);
                            } else if constexpr (B_WIDE) {
#pragma unroll
                                for (int b = 0; b < 4; ++b)
                                    ptx::tma_load_2d(a_dst + b * Cfg::MN_BOX_BYTES, ud.tmap_a, &a_full[as],
                                                     tm * Cfg::BM + 32 * b, kc);
                            } else {
                                ptx::tma_load_2d(a_dst, ud.tmap_a, &a_full[as], tm * Cfg::BM, kc);
                            }
                            a_issued |= 1u << as;
                            a_par = (a_par & ~(1u << as)) | (aph << as);
                        }
                    }
                    if (++as == SA) {
                        as = 0;
                        aph ^= 1u;
                    }
                    if (!ptx::mbar_wait(&b_empty[bs], bph ^ 1u, abort_flag, limit)) {
                        fail(kErrProducerTimeout);
                        goto producer_done;
                    }
                    if (GEN_B && ud.b_gen) {
                        // the split warps write this stage; the slot's earlier load has been
                        // consumed, so none of it is in flight
                        b_issued &= ~(1u << bs);
                    } else {
                        uint8_t* b_dst = b_base + bs * Cfg::B_STAGE;
                        ptx::mbar_arrive_expect_tx(&b_full[bs], ud.bn * Cfg::BK * (B_WIDE ? 4 : 2));
                        if constexpr (GEN_B) ptx::mbar_arrive_n(&b_full[bs], kBFullCount - 1);
                        if constexpr (B_KMAJOR) {
                            if (b_blocked(p))  // k-blocks: {k within the block, column, block}
                                ptx::tma_load_3d(b_dst, ud.tmap_b, &b_full[bs], 0, tn * ud.bn, st);
                            else
                                ptx::tma_load_2d(b_dst, ud.tmap_b, &b_full[bs], kc, tn * ud.bn);
                        } else if constexpr (!kTf32) {
#pragma unroll
                            for (int sub = 0; sub < BN / 64; ++sub)
                                ptx::tma_load_2d(b_dst + sub * (Cfg::BK * 128), ud.tmap_b, &b_full[bs],
                                                 tn * BN + 64 * sub, kc);
                        } else {
                            ptx::tma_load_2d(b_dst, ud.tmap_b, &b_full[bs], tn * BN, kc);
                        }
                        b_issued |= 1u << bs;
                        b_par = (b_par & ~(1u << bs)) | (bph << bs);
                    }
                    if (++bs == SB) {
                        bs = 0;
                        bph ^= 1u;
                    }
                }
            }
        producer_done:
            // Never leave with bulk copies in flight into this CTA's shared memory.
            if (lane == 0) {
                for (int s = 0; s < SA + SB; ++s) {
                    const bool is_a = s < SA;
                    const int st = is_a ? s : s - SA;
                    if (!((is_a ? a_issued : b_issued) & (1u << st))) continue;
                    uint64_t* bar = is_a ? &a_full[st] : &b_full[st];
                    const uint32_t par = ((is_a ? a_par : b_par) >> st) & 1u;
                    const uint64_t t0 = ptx::globaltimer_ns();
                    while (!ptx::mbar_try_wait(bar, par)) {
                        if (ptx::globaltimer_ns() - t0 > limit) {
                            fail(kErrDrainTimeout);
                            break;
                        }
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ UMMA issuer
        if (lane == 0) {
            int as = 0, bs = 0;
            uint32_t aph = 0, bph = 0, gc = 0;
            bool issued_any = false;
            for (int uk = 0;; ++uk) {
                int u;
                if (!take_unit(uk, u)) {
                    fail(kErrMmaTimeout);
                    goto mma_done;
                }
                ptx::mbar_arrive(&unit_empty[uk & 3]);
                if (u < 0) break;
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                const int nsteps = ud.s1 - ud.s0;
                const uint32_t idesc = ptx::make_idesc(kTf32, !A_KMAJOR && !kTf32, !kTf32 && !B_KMAJOR, Cfg::BM, ud.bn);
                for (int i = 0; i < nsteps; ++i) {
                    const uint32_t db = gc & 1u;
                    if (!ptx::mbar_wait(&d_empty[db], ((gc >> 1) & 1u) ^ 1u, abort_flag, limit)) {
                        fail(kErrMmaTimeout);
                        goto mma_done;
                    }
                    if constexpr (!kTf32 || B_WIDE) {
                        if (!ptx::mbar_wait(&b_full[bs], bph, abort_flag, limit)) {
                            fail(kErrMmaTimeout);
                            goto mma_done;
                        }
                    }
                    if (!ptx::mbar_wait(&a_split[as], aph, abort_flag, limit)) {
                        fail(kErrMmaTimeout);
                        goto mma_done;
                    }
                    ptx::tc_fence_after();
                    {
                        const uint32_t d = tmem_base + db * BN;
                        const uint32_t hi_s = ptx::smem_u32(a_base + as * Cfg::A_STAGE);
                        const uint32_t lo_s = hi_s + ((A_KMAJOR || kTf32) ? Cfg::HI_BYTES : 1024);
                        const uint32_t b_s = ptx::smem_u32(b_base + bs * Cfg::B_STAGE);
                        auto a_desc = [&](uint32_t base, int kk) -> uint64_t {
                            if constexpr (A_KMAJOR || kTf32) {
                                return ptx::make_smem_desc(base + kk * 32, 16, 1024, ptx::kLayoutSW128);
                            } else {
                                // MN-major: 64-wide m atoms MN_HALF_BYTES apart, 8-row k groups 2048
                                // bytes apart (hi and lo atoms interleaved); one UMMA_K = 16 step is
                                // two k groups.
                                return ptx::make_smem_desc(base + kk * 4096, Cfg::MN_HALF_BYTES, 2048,
                                                           ptx::kLayoutSW128);
                            }
                        };
                        auto b_desc = [&](int kk) -> uint64_t {
                            if constexpr (kTf32 || B_KMAJOR) {
                                return ptx::make_smem_desc(b_s + kk * 32, 16, 1024, ptx::kLayoutSW128);
                            } else {
                                return ptx::make_smem_desc(b_s + kk * 2048, Cfg::BK * 128, 1024, ptx::kLayoutSW128);
                            }
                        };
                        // lo products into a fresh accumulator ...
#pragma unroll
                        for (int kk = 0; kk < Cfg::KSUB; ++kk) {
                            if constexpr (kTf32)
                                ptx::umma_tf32_ss(d, a_desc(lo_s, kk), b_desc(kk), idesc, kk > 0 ? 1u : 0u);
                            else
                                ptx::umma_f16_ss(d, a_desc(lo_s, kk), b_desc(kk), idesc, kk > 0 ? 1u : 0u);
                        }
                        // ... scaled by 2^-11 under the first hi product, then the other hi products.
                        if constexpr (kTf32)
                            ptx::umma_tf32_ss_scale11(d, a_desc(hi_s, 0), b_desc(0), idesc);
                        else
                            ptx::umma_f16_ss_scale11(d, a_desc(hi_s, 0), b_desc(0), idesc);
#pragma unroll
                        for (int kk = 1; kk < Cfg::KSUB; ++kk) {
                            if constexpr (kTf32)
                                ptx::umma_tf32_ss(d, a_desc(hi_s, kk), b_desc(kk), idesc, 1u);
                            else
                                ptx::umma_f16_ss(d, a_desc(hi_s, kk), b_desc(kk), idesc, 1u);
                        }
                    }
                    issued_any = true;
                    ptx::umma_commit(&a_empty[as]);
                    ptx::umma_commit(&b_empty[bs]);
                    if (++as == SA) {
                        as = 0;
                        aph ^= 1u;
                    }
                    if (++bs == SB) {
                        bs = 0;
                        bph ^= 1u;
                    }
                    ptx::umma_commit(&d_full[db]);
                    ++gc;
                }
            }
        mma_done:
            // Wait for every MMA this thread issued before TMEM is released.
            if (issued_any) {
                ptx::umma_commit(drain_bar);
                const uint64_t t0 = ptx::globaltimer_ns();
                while (!ptx::mbar_try_wait(drain_bar, 0)) {
                    if (ptx::globaltimer_ns() - t0 > limit) {
                        fail(kErrDrainTimeout);
                        break;
                    }
                }
            }
        }
    } else if (warp < Cfg::EPI_WARP0) {
        // ------------------------------------------------------------ split warps
        const int sidx = (warp - 2) * 32 + lane;
        int as = 0, bs = 0;
        uint32_t aph = 0, bph = 0;
        // binary16: global item g of this CTA's item sequence goes to split warp g % SPLIT_WARPS;
        // `first` is this warp's first item of the current stage.
        int first = warp - 2;
        for (int uk = 0;; ++uk) {
            int u;
            if (!take_unit(uk, u)) {
                fail(kErrSplitTimeout);
                goto split_done;
            }
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&unit_empty[uk & 3]);
            if (u < 0) break;
            UnitDesc ud;
            get_unit<Cfg>(p, u, ud);
            if constexpr (GEN_B) {
                // the generator's view of the unit, kept in this warp's shared slot rather than
                // in registers the A split needs
                if (ud.b_gen && lane == 0)
                    gen_slots[warp - 2] = GenB{ud.gen_seed, ud.tn * ud.bn, ud.bn, ud.n, ud.k};
                __syncwarp();
            }
            for (int st = ud.s0; st < ud.s1; ++st) {
                if constexpr (GEN_B) {
                    if (ud.b_gen) {
                        // this stage's generated B, rows spread over all split threads, written
                        // while the stage's A is still in flight (its slot was freed by the MMAs
                        // of SB stages back)
                        if (!ptx::mbar_wait(&b_empty[bs], bph ^ 1u, abort_flag, limit)) {
                            fail(kErrSplitTimeout);
                            goto split_done;
                        }
                        gen_b_rows(b_base + bs * Cfg::B_STAGE, gen_slots[warp - 2], st, sidx, Cfg::SPLIT_THREADS);
                        ptx::fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0) ptx::mbar_arrive(&b_full[bs]);
                    }
                }
                if (!ptx::mbar_wait(&a_full[as], aph, abort_flag, limit) ||
                    (kTf32 && !B_WIDE && !ptx::mbar_wait(&b_full[bs], bph, abort_flag, limit))) {
                    fail(kErrSplitTimeout);
                    goto split_done;
                }
                if constexpr (Cfg::kItemSplit) {
                    if constexpr (kTf32)
                        split_stage_tf32w<Cfg, A_KMAJOR>(a_base + as * Cfg::A_STAGE, first, lane);
                    else
                        split_stage_f16<Cfg, A_KMAJOR>(a_base + as * Cfg::A_STAGE, first, lane);
                    first -= Cfg::SPLIT_ITEMS % NSPLIT;
                    if (first < 0) first += NSPLIT;
                } else {
                    auto all_read = [&]() -> bool {
                        __syncwarp();
                        if (lane == 0) ptx::mbar_arrive(&a_read[as]);
                        return ptx::mbar_wait(&a_read[as], aph, abort_flag, limit);
                    };
                    if (!split_step_tf32<Cfg, A_KMAJOR, B_KMAJOR>(a_base + as * Cfg::A_STAGE,
                                                                   b_base + bs * Cfg::B_STAGE, sidx, all_read)) {
                        fail(kErrSplitTimeout);
                        goto split_done;
                    }
                }
                // Make the generic-proxy stores visible to the tensor core (async proxy).
                ptx::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&a_split[as]);
                if (++as == SA) {
                    as = 0;
                    aph ^= 1u;
                }
                if constexpr ((kTf32 && !B_WIDE) || GEN_B) {
                    if (++bs == SB) {
                        bs = 0;
                        bph ^= 1u;
                    }
                }
            }
        }
    split_done:;
    }
    } else {
        // ------------------------------------------------------------ epilogue
        ptx::setmaxnreg_inc<Cfg::EPI_REGS>();
        const DevScalarValues dsc = load_dev_scalars(p);
        constexpr int HN = Cfg::HALF_N;
        const int q = warp & 3;                         // TMEM lane quadrant this warp may access
        const int half = (warp - Cfg::EPI_WARP0) >> 2;  // column half of the tile
        const int row_in_tile = q * 32 + lane;
        const uint32_t lane_addr = static_cast<uint32_t>(q * 32) << 16;
        uint32_t gc = 0;
        for (int uk = 0;; ++uk) {
            int u;
            if (!take_unit(uk, u)) {
                fail(kErrEpilogueTimeout);
                goto epi_done;
            }
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&unit_empty[uk & 3]);
            if (u < 0) break;
            int nsteps, hn;
            {
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                nsteps = ud.s1 - ud.s0;
                hn = ud.bn / 2;  // columns of this warp's half (<= HN)
                // beta != 0: C of this thread's row into L2 (kept there) while the tile's k-steps run
                const int row = ud.tm * Cfg::BM + row_in_tile;
                const int col0 = ud.tn * ud.bn + half * hn;
                if ((dsc.on ? dsc.beta : ud.beta) != 0.0f && !ud.partial && row < ud.m)
                    prefetch_row<HN>(ud.c, ud.ldc, output_op(p), row, col0, ud.n < col0 + hn ? ud.n : col0 + hn);
            }
            uint64_t acc2[HN / 2];  // running sums, packed in pairs of columns
#pragma unroll
            for (int j = 0; j < HN / 2; ++j) acc2[j] = 0ull;
            for (int i = 0; i < nsteps; ++i) {
                const uint32_t db = gc & 1u;
                if (!ptx::mbar_wait(&d_full[db], (gc >> 1) & 1u, abort_flag, limit)) {
                    fail(kErrEpilogueTimeout);
                    goto epi_done;
                }
                ptx::tc_fence_after();
#pragma unroll
                for (int j0 = 0; j0 < HN; j0 += 32) {
                    if (j0 >= hn) break;
                    uint32_t r0[16], r1[16];
                    const uint32_t ta = tmem_base + lane_addr + db * BN + half * hn + j0;
                    ptx::tmem_ld_32x32b_x16(ta, r0);
                    ptx::tmem_ld_32x32b_x16(ta + 16, r1);
                    ptx::tmem_ld_wait();
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        acc2[j0 / 2 + e] = ptx::f2_add(acc2[j0 / 2 + e],
                                                       (static_cast<uint64_t>(r0[2 * e + 1]) << 32) | r0[2 * e]);
                        acc2[j0 / 2 + 8 + e] = ptx::f2_add(acc2[j0 / 2 + 8 + e],
                                                           (static_cast<uint64_t>(r1[2 * e + 1]) << 32) | r1[2 * e]);
                    }
                }
                ptx::tc_fence_before();
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&d_empty[db]);
                ++gc;
            }
            {
                auto acc = [&](int j) -> float { return (j & 1) ? ptx::f2_hi(acc2[j >> 1]) : ptx::f2_lo(acc2[j >> 1]); };
                // the unit's output fields, read again here so they are not live during the drain
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                const int tm = ud.tm, tn = ud.tn;
                const int row = tm * Cfg::BM + row_in_tile;
                const int col0 = tn * ud.bn + half * hn;
                if (row < ud.m) {
                    if (ud.partial) {
                        float* w = ud.partial + row;
#pragma unroll
                        for (int j = 0; j < HN; ++j) {
                            const int col = col0 + j;
                            if (j < hn && col < ud.n) w[static_cast<size_t>(col) * ud.m] = acc(j);
                        }
                    } else {
                        // columns of this warp's half only (a grouped problem's tile may be narrower)
                        const int n_end = ud.n < col0 + hn ? ud.n : col0 + hn;
                        store_row<HN>(ud.c, ud.ldc, output_op(p), row, col0, n_end, dsc.on ? dsc.alpha : ud.alpha,
                                      dsc.on ? dsc.beta : ud.beta, acc);
                    }
                }
            }
        }
    epi_done:;
    }

    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 1) {
        ptx::tmem_dealloc(tmem_base, Cfg::TMEM_COLS);
    }
}

// Single problem (optionally split-K): descriptors in the kernel's parameter space.
template <int TC, int BN, bool A_KMAJOR, bool B_KMAJOR>
__global__ void __launch_bounds__(512, 1) shgemm_tile_kernel(const __grid_constant__ TileGemmParams p) {
    tile_kernel_body<TC, BN, A_KMAJOR, B_KMAJOR, false, false>(p);
}

// Single TF32 problem whose binary16 B was widened to FP32 beforehand (128 x BN tiles, BN 256
// or 128, B K-major): loaded straight into the TF32 tile layout, split-K as the other tile
// kernels.
template <int BN, bool A_KMAJOR>
__global__ void __launch_bounds__(512, 1) shgemm_tile_wide_kernel(const __grid_constant__ TileGemmParams p) {
    tile_kernel_body<kTF32, BN, A_KMAJOR, true, true, false>(p);
}

// Many problems in one launch: per-problem descriptors and a unit list in device memory.
// Binary16 launches can generate a problem's B (block-sign Rademacher) in the producer.
template <int TC, int BN, bool A_KMAJOR, bool B_KMAJOR, bool B_WIDE>
__global__ void __launch_bounds__(512, 1) shgemm_grouped_kernel(const __grid_constant__ GroupedParams p) {
    tile_kernel_body<TC, BN, A_KMAJOR, B_KMAJOR, B_WIDE, TC == kFP16 && B_KMAJOR>(p);
}

}  // namespace shgemm_b200
