// Host side of the C ABI (include/shgemm_b200.h): handle, dispatch, TMA
// descriptors and launches of the sm_100a kernels, plus the split-K reduction,
// the k == 0 scaling kernel, the bounded-wait self test and the FP64 evaluation
// kernels used to measure error.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "shgemm_b200.h"
#include "shgemm_kernel.cuh"
#include "shgemm_kernel_tm.cuh"
#include "shgemm_kernel_tm2.cuh"

using namespace shgemm_b200;

// The tables of a grouped launch: the device copy the kernel reads and its pinned host
// staging, each holding the problems, then the unit list, then the unit count at fixed
// offsets, so that a captured graph's copy replays whatever the staging holds.
struct GroupedTable {
    void* dev = nullptr;
    void* host = nullptr;
    cudaEvent_t copied = nullptr;  // the last eager copy out of the staging
    int max_problems = 0;
    size_t units_off = 0, count_off = 0, bytes = 0;
    int tc = -1, op_a = -1, op_b = -1, op_c = -1, b32 = -1;  // variant of the staged batch
    int units = 0;
    int copied_count = 0;  // problem slots the last enqueued copy covers
};

struct shgemm_b200_handle {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    unsigned debug_mode = 0;
    int fixed_level = SHGEMM_LEVEL_AUTO;
    long long split_k = 0;
    long long wait_limit_ms = 2000;
    long long group_m = 8;
    float* workspace = nullptr;
    size_t workspace_bytes = 0;
    int* error_word = nullptr;
    std::atomic<long long> launches{0};
    // grouped launches: the caller's batches (which captured graphs replay) and, apart from
    // them, the one-problem table of eager TF32 calls that take the widened-B route
    GroupedTable grouped;
    GroupedTable single;
    int grouped_b_fp32 = 0;  // SHGEMM_CFG_GROUPED_B_FP32
    // autotuner: best (tile N, split-K slices, rasterisation group) per shape bucket
    int autotune_mode = 1;  // SHGEMM_CFG_AUTOTUNE
    int tile_kernel = 0;    // SHGEMM_CFG_TILE_KERNEL
    int k_chunk = 64;       // SHGEMM_CFG_K_CHUNK
    int tm_stages = 0;      // SHGEMM_CFG_TM_STAGES
    int pair_tiles = 0;     // SHGEMM_CFG_PAIR_TILES
    int max_pairs = 74;     // clusters of 2 of the pair kernel resident at once
    std::mutex tune_mu;
    std::map<uint64_t, shgemm_b200_tuned_config> tuned;
    // host-buffer entry: device staging (A and three column-block slots of B and C), one
    // stream per copy direction, events start / in[3] / computed[3] / out[3]
    void* host_stage = nullptr;
    size_t host_stage_bytes = 0;
    cudaStream_t host_in = nullptr, host_out = nullptr;
    cudaEvent_t host_ev[10] = {};
    long long host_block_cols = 0;  // SHGEMM_CFG_HOST_BLOCK_COLS
};

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<EncodeTiledFn>(p);
        }
    });
    return fn;
}

// 2-D tiled tensor map: dim0 contiguous (`d0` elements), dim1 with a stride of
// `stride1_bytes`; box {b0, b1}. Out-of-range elements read as zero.
bool make_tmap(CUtensorMap* map, CUtensorMapDataType dtype, const void* base, uint64_t d0, uint64_t d1,
               uint64_t stride1_bytes, uint32_t b0, uint32_t b1, CUtensorMapSwizzle swz) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {d0, d1};
    cuuint64_t strides[1] = {stride1_bytes};
    cuuint32_t box[2] = {b0, b1};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// 3-D tiled tensor map: dim0 contiguous, dims 1 and 2 with byte strides s1, s2; box {b0, b1, b2}.
bool make_tmap_3d(CUtensorMap* map, CUtensorMapDataType dtype, const void* base, uint64_t d0, uint64_t d1,
                  uint64_t d2, uint64_t s1, uint64_t s2, uint32_t b0, uint32_t b1, uint32_t b2, CUtensorMapSwizzle swz) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {d0, d1, d2};
    cuuint64_t strides[2] = {s1, s2};
    cuuint32_t box[3] = {b0, b1, b2};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, dtype, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// K-major FP32 operand (k x m, column stride `ld_bytes`) as a 3-D view {32 floats, k / 32,
// m} with box {32, 2, 128} and a 128-byte swizzle: one load brings 128 rows x 64 floats, each
// row's two 128-byte halves adjacent in shared memory. k must be a multiple of 32 so that the
// view never reaches past a row into the next one.
bool make_tmap_a_paired(CUtensorMap* map, const float* base, uint64_t k, uint64_t m, uint64_t ld_bytes) {
    if (k % 32 != 0) return false;
    return make_tmap_3d(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, base, 32, k / 32, m, 128, ld_bytes, 32, 2, 128,
                        CU_TENSOR_MAP_SWIZZLE_128B);
}

// Width (m) of one TMA box of an M-major FP32 operand: the binary16 kernels load a 128-row
// tile as two 64-wide boxes (one per half of the split's items), the TF32 kernels with a
// widened B as four 32-wide boxes (one per item), the other TF32 kernels as one.
constexpr uint32_t a_mmajor_box(int tc, bool b_wide = false) { return tc == kFP16 ? 64 : (b_wide ? 32 : 128); }

using TileKernelFn = void (*)(TileGemmParams);

// Column pitch of a K-major binary16 operand from which it is re-laid out as k-blocks.
constexpr size_t kBlockBMinPitchBytes = size_t(1) << 20;

template <int TC, int BN, bool AK, bool BK>
void* tile_kernel_ptr() {
    return reinterpret_cast<void*>(&shgemm_tile_kernel<TC, BN, AK, BK>);
}

template <int TC, int BN, bool AK, bool BK>
int tile_smem() {
    return TileCfg<TC, BN, AK, BK>::SMEM_BYTES;
}

struct KernelEntry {
    void* fn;
    int smem;
};

// Instantiated tile kernels: binary16 compute with tile N 64 / 128 / 256, TF32 with 64 / 128.
KernelEntry kernel_table(int tc, int bn, int ak, int bk) {
#define SHG_ENTRY(TC, BN, AK, BK) \
    if (tc == TC && bn == BN && ak == AK && bk == BK) return {tile_kernel_ptr<TC, BN, AK, BK>(), tile_smem<TC, BN, AK, BK>()};
#define SHG_ENTRY4(TC, BN) SHG_ENTRY(TC, BN, 0, 0) SHG_ENTRY(TC, BN, 0, 1) SHG_ENTRY(TC, BN, 1, 0) SHG_ENTRY(TC, BN, 1, 1)
    SHG_ENTRY4(kFP16, 64) SHG_ENTRY4(kFP16, 128) SHG_ENTRY4(kFP16, 256)
    SHG_ENTRY4(kTF32, 64) SHG_ENTRY4(kTF32, 128)
#undef SHG_ENTRY4
#undef SHG_ENTRY
    return {nullptr, 0};
}

// TF32, 128 x 256 tiles, B widened to FP32 in the workspace (K-major).
template <int BN, bool AK>
KernelEntry tile_wide_entry() {
    return {reinterpret_cast<void*>(&shgemm_tile_wide_kernel<BN, AK>), TileCfg<kTF32, BN, AK, true, true>::SMEM_BYTES};
}
KernelEntry tile_wide_table(bool ak, int bn) {
    if (bn == 256) return ak ? tile_wide_entry<256, true>() : tile_wide_entry<256, false>();
    return ak ? tile_wide_entry<128, true>() : tile_wide_entry<128, false>();
}

// Tensor-memory operand kernels (binary16 compute, 128 x 256 tiles, B K-major).
template <bool AK, int KC, int SV>
KernelEntry tm_entry() {
    return {reinterpret_cast<void*>(&shgemm_tm_kernel<AK, KC, SV>), TmCfg<AK, KC, SV>::SMEM_BYTES};
}
// kc: k-steps of 64 per FP32 drain (1 or 2); sv: operand ring variant (0 or 1)
// The CTA-pair form (256 x 256 tiles over two SMs).
KernelEntry tm2_kernel_table(bool ak) {
    if (ak) return {reinterpret_cast<void*>(&shgemm_tm2_kernel<true>), Tm2Cfg<true>::SMEM_BYTES};
    return {reinterpret_cast<void*>(&shgemm_tm2_kernel<false>), Tm2Cfg<false>::SMEM_BYTES};
}

// Clusters of 2 of the pair kernel that can be resident at once: a GPC with an odd number of
// free SMs leaves one out, so the persistent grid is sized by the occupancy query, not by SMs / 2
// (a cluster beyond it would start only when another one finished, doubling the tail).
int query_max_pairs(const KernelEntry& e, int num_sms) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * (num_sms / 2));
    cfg.blockDim = dim3(Tm2Cfg<true>::NUM_THREADS);
    cfg.dynamicSmemBytes = e.smem;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, e.fn, &cfg) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return num_sms / 2;
    }
    return std::min(n, num_sms / 2);
}

KernelEntry tm_kernel_table(bool ak, int kc, int sv) {
    if (sv == 1) {
        if (kc == 2) return ak ? tm_entry<true, 2, 1>() : tm_entry<false, 2, 1>();
        return ak ? tm_entry<true, 1, 1>() : tm_entry<false, 1, 1>();
    }
    if (kc == 2) return ak ? tm_entry<true, 2, 0>() : tm_entry<false, 2, 0>();
    return ak ? tm_entry<true, 1, 0>() : tm_entry<false, 1, 0>();
}

template <int TC, int BN, bool AK, bool BW>
KernelEntry grouped_entry() {
    return {reinterpret_cast<void*>(&shgemm_grouped_kernel<TC, BN, AK, true, BW>),
            TileCfg<TC, BN, AK, true, BW>::SMEM_BYTES};
}

// Grouped kernels (B K-major): binary16 compute with tile N up to 256; TF32 up to 128 with
// a binary16 B, up to 256 with a widened (FP32) B.
constexpr int kGroupedMaxBnF16 = 256, kGroupedMaxBnTf32 = 128, kGroupedMaxBnTf32Wide = 256;
KernelEntry grouped_table(int tc, int ak, bool b_wide) {
    if (tc == kFP16) return ak ? grouped_entry<kFP16, kGroupedMaxBnF16, true, false>()
                               : grouped_entry<kFP16, kGroupedMaxBnF16, false, false>();
    if (b_wide) return ak ? grouped_entry<kTF32, kGroupedMaxBnTf32Wide, true, true>()
                          : grouped_entry<kTF32, kGroupedMaxBnTf32Wide, false, true>();
    return ak ? grouped_entry<kTF32, kGroupedMaxBnTf32, true, false>()
              : grouped_entry<kTF32, kGroupedMaxBnTf32, false, false>();
}

// Table layout (device copy and host staging): problems, then units, then the unit count.
constexpr int kGroupedMaxProblems = 8192;
constexpr int kGroupedMaxUnits = 1 << 16;

bool table_alloc(GroupedTable& t, int max_problems) {
    t.max_problems = max_problems;
    t.units_off = sizeof(GroupedProblem) * static_cast<size_t>(max_problems);
    t.count_off = t.units_off + sizeof(int2) * kGroupedMaxUnits;
    t.bytes = t.count_off + 256;
    if (cudaMalloc(&t.dev, t.bytes) != cudaSuccess || cudaMallocHost(&t.host, t.bytes) != cudaSuccess ||
        cudaEventCreateWithFlags(&t.copied, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

void table_free(GroupedTable& t) {
    if (t.copied) {
        cudaEventSynchronize(t.copied);
        cudaEventDestroy(t.copied);
    }
    cudaFree(t.dev);
    cudaFreeHost(t.host);
    t = GroupedTable{};
}

// ------------------------------------------------------------------ small kernels
// C = beta * C (k == 0: the product is empty); beta from device memory when beta_dev is set.
__global__ void scale_c_kernel(float* c, uint64_t ldc, int rows, int cols, float beta, const float* beta_dev) {
    if (beta_dev) beta = *beta_dev;
    const size_t total = static_cast<size_t>(rows) * cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int r = static_cast<int>(idx % rows);
        const int cc = static_cast<int>(idx / rows);
        float* d = c + r + static_cast<size_t>(cc) * ldc;
        *d = (beta == 0.0f) ? 0.0f : __fmul_rn(beta, *d);
    }
}

// Copies a rows x cols column-major block into a buffer with a 16-byte aligned
// leading dimension (the staging path for operands TMA cannot address).
template <typename T>
__global__ void pack_kernel(const T* __restrict__ src, uint64_t ld_src, T* __restrict__ dst, uint64_t ld_dst,
                            int rows, int cols) {
    const size_t total = static_cast<size_t>(rows) * cols;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t r = idx % rows, c = idx / rows;
        dst[r + c * ld_dst] = src[r + c * ld_src];
    }
}

// Widens a k x n binary16 K-contiguous operand (leading dimension ldb) to FP32 with
// leading dimension ld_dst (the B operand of the TF32 kernels that load it unconverted).
__global__ void widen_b_kernel(const __half* __restrict__ src, uint64_t ldb, float* __restrict__ dst,
                               uint64_t ld_dst, int k, int n) {
    const size_t total = static_cast<size_t>(k) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t r = idx % k, c = idx / k;
        dst[r + c * ld_dst] = __half2float(src[r + c * ldb]);
    }
}

// Widens a k x n binary16 K-contiguous operand to FP32 laid out as k-blocks of 32:
// dst[(kb * n + col) * 32 + j] = src[col * ldb + 32 kb + j], zero where 32 kb + j >= k. One
// 32-deep TF32 step of a 256-column tile is then one contiguous 32 KB run (FP32 columns 4 MB
// apart would put each of the tile's columns on a page of its own, as with block_b_kernel).
__global__ void widen_b_blocked_kernel(const __half* __restrict__ src, uint64_t ldb, float* __restrict__ dst, int k,
                                       int n, int kblocks) {
    const size_t total = static_cast<size_t>(n) * kblocks * 32;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int j = static_cast<int>(idx & 31);
        const size_t rest = idx >> 5;
        const int col = static_cast<int>(rest % n);
        const size_t kb = rest / n;
        const size_t r = kb * 32 + j;
        dst[idx] = r < static_cast<size_t>(k) ? __half2float(src[static_cast<size_t>(col) * ldb + r]) : 0.0f;
    }
}

// Re-lays a k x n binary16 K-contiguous operand (leading dimension ldb, 16-byte aligned
// columns) out as k-blocks: dst[(kb * n + col) * 64 + j] = src[col * ldb + 64 kb + j], zero
// where 64 kb + j >= k. One 64-deep step of a 256-column tile is then one contiguous 32 KB
// run instead of 256 rows a leading dimension apart. A thread moves 16 bytes; a warp reads
// 512 contiguous bytes of one column.
__global__ void block_b_kernel(const __half* __restrict__ src, uint64_t ldb, __half* __restrict__ dst, int k, int n,
                               int kblocks) {
    const size_t total = static_cast<size_t>(n) * kblocks * 8;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int c8 = static_cast<int>(idx & 7);
        const size_t rest = idx >> 3;
        const int kb = static_cast<int>(rest % kblocks);
        const int col = static_cast<int>(rest / kblocks);
        const size_t k0 = static_cast<size_t>(kb) * 64 + c8 * 8;
        const __half* s = src + static_cast<size_t>(col) * ldb + k0;
        uint4 v;
        if (k0 + 8 <= static_cast<size_t>(k)) {
            v = *reinterpret_cast<const uint4*>(s);
        } else {
            __half t[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) t[j] = (k0 + j < static_cast<size_t>(k)) ? s[j] : __float2half(0.0f);
            v = *reinterpret_cast<const uint4*>(t);
        }
        *reinterpret_cast<uint4*>(dst + (static_cast<size_t>(kb) * n + col) * 64 + c8 * 8) = v;
    }
}

// Deterministic split-K reduction: slices summed in fixed order 0..S-1, then the
// same alpha/beta epilogue as the tile kernel (C is not read when beta == 0).
__global__ void splitk_reduce_kernel(const float* __restrict__ ws, int slices, int m, int n, float* c,
                                     uint64_t ldc, int op_c, float alpha, float beta, const float* alpha_dev,
                                     const float* beta_dev) {
    if (alpha_dev) alpha = *alpha_dev;
    if (beta_dev) beta = *beta_dev;
    const size_t mn = static_cast<size_t>(m) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < mn;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        size_t row, col;
        if (op_c == kOpN) {
            row = idx % m;
            col = idx / m;
        } else {  // walk C's memory order so stores stay coalesced
            col = idx % n;
            row = idx / n;
        }
        const size_t w = row + col * m;
        float s = ws[w];
        for (int sl = 1; sl < slices; ++sl) s = __fadd_rn(s, ws[w + static_cast<size_t>(sl) * mn]);
        float* d = (op_c == kOpN) ? c + row + col * ldc : c + col + row * ldc;
        *d = (beta == 0.0f) ? __fmul_rn(s, alpha) : __fmaf_rn(s, alpha, __fmul_rn(beta, *d));
    }
}

// Sketch operand generator. GAUSSIAN: entries 2i and 2i + 1 of column c of a k x cols
// column-major Omega are z cos(2 pi u2) and z sin(2 pi u2), z = sqrt(-2 ln u1), u1 and u2 the
// top and middle 24 bits of the counter hash of (seed, c k + 2i) -- splitmix64's finaliser
// (mix64) -- one hash, one logarithm and one sincos per pair; scaled and rounded to binary16.
// RADEMACHER: the top bit of the hash of (seed, c k + r) as the sign of entry r. The block-sign
// stream (SHGEMM_OMEGA_RADEMACHER_BLOCKS) hashes (seed, c * ceil(k / 64) + r / 64) once per 64
// entries of a column and takes bit block_sign_bit(r mod 64): the stream the grouped kernel
// generates as it goes (rademacher_block_bits, gen_b_rows).
__device__ __forceinline__ void omega_store(void* dst, uint64_t i, float v, int fp32) {
    const __half hv = __float2half_rn(v);
    if (fp32)
        static_cast<float*>(dst)[i] = __half2float(hv);
    else
        static_cast<__half*>(dst)[i] = hv;
}

// Thread t of nt writes its share of one Omega.
__device__ __forceinline__ void omega_fill(const shgemm_b200_omega_job& j, int fp32, uint64_t t, uint64_t nt) {
    const uint64_t k = j.k, cols = j.cols, ld = j.ld;
    const float scale = j.scale;
    if (j.dist == SHGEMM_OMEGA_GAUSSIAN) {
        const uint64_t kp = (k + 1) / 2, total = kp * cols;
        for (uint64_t idx = t; idx < total; idx += nt) {
            const uint64_t c = idx / kp, r = 2 * (idx - c * kp);
            const uint64_t x = mix64(j.seed * 0x9E3779B97F4A7C15ull + c * k + r + 1);
            const float u1 = static_cast<float>((x >> 40) + 1) * 0x1p-24f;  // (0, 1]
            const float u2 = static_cast<float>((x >> 16) & 0xFFFFFFull) * 0x1p-24f;
            const float z = scale * sqrtf(-2.0f * logf(u1));
            float sn, cs;
            sincospif(2.0f * u2, &sn, &cs);
            omega_store(j.dst, r + c * ld, z * cs, fp32);
            if (r + 1 < k) omega_store(j.dst, r + 1 + c * ld, z * sn, fp32);
        }
        return;
    }
    const uint64_t total = k * cols, kblocks = (k + 63) / 64;
    for (uint64_t idx = t; idx < total; idx += nt) {
        const uint64_t c = idx / k, r = idx - c * k;
        bool neg;
        if (j.dist == SHGEMM_OMEGA_RADEMACHER_BLOCKS)
            neg = (rademacher_block_bits(j.seed, c * kblocks + r / 64) >> block_sign_bit(static_cast<int>(r % 64))) & 1;
        else
            neg = mix64(j.seed * 0x9E3779B97F4A7C15ull + idx + 1) >> 63;
        omega_store(j.dst, r + c * ld, neg ? -scale : scale, fp32);
    }
}

constexpr int kOmegaJobsPerLaunch = 64;
struct OmegaBatch {
    shgemm_b200_omega_job job[kOmegaJobsPerLaunch];
    int fp32;
};

// blockIdx.y = job; the x blocks of a job share its entries.
__global__ void omega_kernel(const __grid_constant__ OmegaBatch b) {
    omega_fill(b.job[blockIdx.y], b.fp32, blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x,
               static_cast<uint64_t>(gridDim.x) * blockDim.x);
}

__global__ void selftest_wait_kernel(int* error_flag, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        ptx::mbar_init(&bar, 1);
        abort_flag = 0;
        ptx::fence_mbarrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // Nothing ever arrives on `bar`: the bounded wait must give up.
        if (!ptx::mbar_wait(&bar, 0, &abort_flag, limit_ns)) atomicCAS(error_flag, 0, kErrMmaTimeout);
    }
    __syncthreads();
}

// ------------------------------------------------------------------ FP64 evaluation
template <typename T>
__device__ __forceinline__ double to_d(T v);
template <>
__device__ __forceinline__ double to_d<float>(float v) { return static_cast<double>(v); }
template <>
__device__ __forceinline__ double to_d<__half>(__half v) { return static_cast<double>(__half2float(v)); }

// 64x64 output tile per 256-thread block, 4x4 doubles per thread.
template <typename TA, typename TB>
__global__ void __launch_bounds__(256) eval_dgemm_kernel(int op_a, int op_b, int m, int n, int k, const TA* a,
                                                         uint64_t lda, const TB* b, uint64_t ldb, double* c) {
    __shared__ double As[16][64 + 1];
    __shared__ double Bs[16][64 + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.x * 64, n0 = blockIdx.y * 64;
    double acc[4][4] = {};
    for (int k0 = 0; k0 < k; k0 += 16) {
        for (int i = threadIdx.x; i < 16 * 64; i += 256) {
            const int kk = i / 64, r = i % 64;
            const int gi = m0 + r, gk = k0 + kk;
            double va = 0.0;
            if (gi < m && gk < k) va = to_d(op_a == kOpN ? a[gi + gk * lda] : a[gk + gi * lda]);
            As[kk][r] = va;
            const int gj = n0 + r;
            double vb = 0.0;
            if (gj < n && gk < k) vb = to_d(op_b == kOpN ? b[gk + gj * ldb] : b[gj + gk * ldb]);
            Bs[kk][r] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            double ar[4], br[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) ar[i] = As[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) br[j] = Bs[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(ar[i], br[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gi = m0 + tx + 16 * i, gj = n0 + ty + 16 * j;
            if (gi < m && gj < n) c[gi + static_cast<size_t>(gj) * m] = acc[i][j];
        }
}

__global__ void eval_error_kernel(size_t m, size_t n, const float* c, uint64_t ldc, int op_c, const double* c64,
                                  double alpha, double beta, const float* c0, double* partial) {
    double s_diff = 0.0, s_ref = 0.0, s_max = 0.0, s_mismatch = 0.0;
    const size_t total = m * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t i = idx % m, j = idx / m;
        const size_t ci = (op_c == kOpN) ? i + j * ldc : j + i * ldc;
        double ref = alpha * c64[idx];
        if (beta != 0.0) ref += beta * static_cast<double>(c0[ci]);
        const double v = static_cast<double>(c[ci]);
        const bool fv = isfinite(v), fr = isfinite(ref);
        if (fv && fr) {
            const double d = v - ref;
            s_diff += d * d;
            s_ref += ref * ref;
            if (ref != 0.0) s_max = fmax(s_max, fabs(d) / fabs(ref));
        } else if (fv != fr) {
            s_mismatch += 1.0;
        }
    }
    __shared__ double red[4][256];
    red[0][threadIdx.x] = s_diff;
    red[1][threadIdx.x] = s_ref;
    red[2][threadIdx.x] = s_max;
    red[3][threadIdx.x] = s_mismatch;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] = fmax(red[2][threadIdx.x], red[2][threadIdx.x + s]);
            red[3][threadIdx.x] += red[3][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int q = 0; q < 4; ++q) partial[blockIdx.x * 4 + q] = red[q][0];
    }
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int launch_status() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SHGEMM_STATUS_OK : SHGEMM_STATUS_LAUNCH_FAILED;
}

struct Plan {
    int level;  // 0: the smaller tile N, 1: the larger one
    int bn;
    int tiles_m, tiles_n;
    int total_steps;
    int slices;
    int steps_per_slice;
    int kc;  // tensor-memory kernel: k-steps of 64 per FP32 drain (0: the handle's SHGEMM_CFG_K_CHUNK)
    int sv;  // tensor-memory kernel: operand ring variant (-1: the handle's SHGEMM_CFG_TM_STAGES)
    int pair;  // tensor-memory kernel in CTA pairs: 1 yes, 0 no (-1: the handle's SHGEMM_CFG_PAIR_TILES)
};

double wave_efficiency(long long units, int sms) {
    const long long waves = (units + sms - 1) / sms;
    return static_cast<double>(units) / static_cast<double>(waves * sms);
}

// Tile N per level: binary16 compute {128, 256}, TF32 {64, 128}; n <= 64 always
// takes N = 64, which wastes no MMA columns.
int level_bn(int tc, int level) { return tc == kFP16 ? (level ? 256 : 128) : (level ? 128 : 64); }

// Tiling and split-K plan. `split_k`: 0 automatic, 1 never, s > 1 forced. Split-K
// partials need slices * m * n floats of scratch, bounded by `ws_bytes`.
// Shape bucket of the autotuner: compute type, operand layouts and floor(log2) of m, n, k.
int ilog2(size_t x) {
    int r = 0;
    while (x > 1) {
        x >>= 1;
        ++r;
    }
    return r;
}
uint64_t tune_key(int tc, int op_a, int op_b, size_t m, size_t n, size_t k) {
    return (static_cast<uint64_t>(tc) << 27) | (static_cast<uint64_t>(op_a) << 26) |
           (static_cast<uint64_t>(op_b) << 25) | (static_cast<uint64_t>(ilog2(m)) << 16) |
           (static_cast<uint64_t>(ilog2(n)) << 8) | static_cast<uint64_t>(ilog2(k));
}
// Grouped launches: the tile N of the problems in one n bucket, floor(log2 n).
constexpr uint64_t kTuneGrouped = uint64_t(1) << 30;
uint64_t tune_key_grouped(int tc, int op_a, int b_fp32, int log2n) {
    return kTuneGrouped | (static_cast<uint64_t>(tc) << 27) | (static_cast<uint64_t>(op_a) << 26) |
           (static_cast<uint64_t>(b_fp32) << 25) | (static_cast<uint64_t>(log2n) << 8);
}

// A tuned configuration applied to a shape: the tile N and the slice count it names,
// the slices capped by what the workspace holds and by the k-steps there are.
Plan plan_from_tuned(const shgemm_b200_tuned_config& t, size_t m, size_t n, size_t k, int tc, size_t ws_bytes) {
    Plan p{};
    const int bk = (tc == kFP16) ? 64 : 32;
    p.total_steps = static_cast<int>((k + bk - 1) / bk);
    p.tiles_m = static_cast<int>((m + 127) / 128);
    p.bn = t.tile_n;
    p.level = p.bn == level_bn(tc, 1) ? 1 : 0;
    p.tiles_n = static_cast<int>((n + p.bn - 1) / p.bn);
    const size_t per_slice = m * n * sizeof(float);
    const int fit = per_slice ? static_cast<int>(std::min<size_t>(ws_bytes / per_slice, 1024)) : 0;
    int slices = std::max(1, t.slices);
    if (slices > 1 && fit < 2) slices = 1;
    slices = std::min({slices, std::max(fit, 1), p.total_steps});
    p.steps_per_slice = (p.total_steps + slices - 1) / slices;
    p.slices = (p.total_steps + p.steps_per_slice - 1) / p.steps_per_slice;
    p.kc = t.k_chunk == 128 ? 2 : 0;  // a 64-k entry leaves the handle's SHGEMM_CFG_K_CHUNK in force
    p.sv = t.stages == 1 ? 1 : 0;
    p.pair = t.cta_group == 2 ? 1 : (t.cta_group == 1 ? 0 : -1);
    return p;
}

Plan make_plan_for(int num_sms, int fixed_level, long long split_k, size_t m, size_t n, size_t k, int tc,
                   size_t ws_bytes, int force_bn = 0) {
    Plan p{};
    p.sv = -1;
    p.pair = -1;
    const int bk = (tc == kFP16) ? 64 : 32;
    p.total_steps = static_cast<int>((k + bk - 1) / bk);
    p.tiles_m = static_cast<int>((m + 127) / 128);
    const size_t per_slice = m * n * sizeof(float);
    const int fit = per_slice ? static_cast<int>(std::min<size_t>(ws_bytes / per_slice, 1024)) : 0;
    const bool can_split = split_k != 1 && fit >= 2 && k >= 4096;
    // Level choice mirrors the reference (src/shgemm.cu:643-656): the large tile when it
    // fills the machine (or when split-K will), else the small one; a fixed level overrides.
    const int small = level_bn(tc, 0), big = level_bn(tc, 1);
    const long long tiles_big = static_cast<long long>(p.tiles_m) * ((n + big - 1) / big);
    int level = 0;
    if (n > static_cast<size_t>(small) && (tiles_big >= num_sms || can_split)) level = 1;
    if (fixed_level == SHGEMM_LEVEL_P0 || fixed_level == SHGEMM_LEVEL_P1) level = fixed_level;
    p.level = level;
    p.bn = level_bn(tc, level);
    if (n <= 64 && fixed_level == SHGEMM_LEVEL_AUTO) p.bn = 64;
    if (force_bn) {  // a kernel with one tile shape (the widened-B TF32 kernel)
        p.level = 1;
        p.bn = force_bn;
    }
    p.tiles_n = static_cast<int>((n + p.bn - 1) / p.bn);
    const long long tiles = static_cast<long long>(p.tiles_m) * p.tiles_n;
    // Split-K: deterministic slices when the tiles alone leave SMs idle and k is long;
    // the slice count maximises the fraction of busy SMs over the waves.
    int slices = 1;
    if (split_k > 1) {
        slices = static_cast<int>(std::min<long long>(split_k, fit >= 2 ? fit : 1));
    } else if (can_split && tiles < num_sms) {
        double best = wave_efficiency(tiles, num_sms);
        for (int s = 2; s <= std::min(fit, 64); ++s) {
            if (p.total_steps / s < 8) break;
            const double e = wave_efficiency(tiles * s, num_sms);
            if (e > best + 0.02) {
                best = e;
                slices = s;
            }
        }
    }
    slices = std::max(1, std::min(slices, p.total_steps));
    p.steps_per_slice = (p.total_steps + slices - 1) / slices;
    p.slices = (p.total_steps + p.steps_per_slice - 1) / p.steps_per_slice;
    return p;
}

// The plan of a call: the autotuner's entry for the shape's bucket when there is one
// (and neither a fixed level nor a forced split overrides it), else the heuristic.
Plan make_plan(shgemm_b200_handle* h, int op_a, int op_b, size_t m, size_t n, size_t k, int tc, size_t ws_bytes,
               int* group_m) {
    *group_m = static_cast<int>(h->group_m);
    if (h->autotune_mode != 0 && h->fixed_level == SHGEMM_LEVEL_AUTO && h->split_k == 0) {
        std::lock_guard<std::mutex> lk(h->tune_mu);
        auto it = h->tuned.find(tune_key(tc, op_a, op_b, m, n, k));
        if (it != h->tuned.end()) {
            *group_m = it->second.group_m;
            return plan_from_tuned(it->second, m, n, k, tc, ws_bytes);
        }
    }
    return make_plan_for(h->num_sms, h->fixed_level, h->split_k, m, n, k, tc, ws_bytes);
}

}  // namespace

extern "C" {

const char* shgemm_b200_status_string(int s) {
    switch (s) {
        case SHGEMM_STATUS_OK: return "SHGEMM_STATUS_OK";
        case SHGEMM_STATUS_INVALID_VALUE: return "SHGEMM_STATUS_INVALID_VALUE";
        case SHGEMM_STATUS_NOT_SUPPORTED: return "SHGEMM_STATUS_NOT_SUPPORTED";
        case SHGEMM_STATUS_ALLOC_FAILED: return "SHGEMM_STATUS_ALLOC_FAILED";
        case SHGEMM_STATUS_LAUNCH_FAILED: return "SHGEMM_STATUS_LAUNCH_FAILED";
        case SHGEMM_STATUS_TIMEOUT: return "SHGEMM_STATUS_TIMEOUT";
        case SHGEMM_STATUS_CUDA_ERROR: return "SHGEMM_STATUS_CUDA_ERROR";
        case SHGEMM_STATUS_SCRATCH_TOO_SMALL: return "SHGEMM_STATUS_SCRATCH_TOO_SMALL";
        default: return "SHGEMM_STATUS_UNKNOWN";
    }
}

int shgemm_b200_create(shgemm_b200_handle_t* out, int device) {
    if (!out) return SHGEMM_STATUS_INVALID_VALUE;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return SHGEMM_STATUS_INVALID_VALUE;
    }
    DeviceGuard g(device);
    int major = 0, minor = 0, sms = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (major != 10 || minor != 0) return SHGEMM_STATUS_NOT_SUPPORTED;  // sm_100a code only
    if (!encode_fn()) return SHGEMM_STATUS_NOT_SUPPORTED;
    auto* h = new shgemm_b200_handle();
    h->device = device;
    h->num_sms = sms;
    const char* dbg = std::getenv("MTK_SHGEMM_DEBUG");  // same switch as src/shgemm.cu:407-410
    if (dbg && dbg[0] == '1') h->debug_mode = 1;
    const char* lvl = std::getenv("MTK_SHGEMM_KERNEL_LEVEL");  // src/shgemm.cu:411-414
    if (lvl && (lvl[0] == '0' || lvl[0] == '1') && lvl[1] == '\0') h->fixed_level = lvl[0] - '0';
    if (cudaMalloc(&h->error_word, sizeof(int)) != cudaSuccess) {
        delete h;
        return SHGEMM_STATUS_ALLOC_FAILED;
    }
    cudaMemset(h->error_word, 0, sizeof(int));
    // Default split-K workspace: 64 MiB (room for e.g. 16 slices of a 1024 x 1024 C).
    h->workspace_bytes = size_t(64) << 20;
    if (cudaMalloc(&h->workspace, h->workspace_bytes) != cudaSuccess) {
        cudaFree(h->error_word);
        delete h;
        return SHGEMM_STATUS_ALLOC_FAILED;
    }
    for (int tc = 0; tc < 2; ++tc)
        for (int bn : {64, 128, 256})
            for (int ak = 0; ak < 2; ++ak)
                for (int bk = 0; bk < 2; ++bk) {
                    KernelEntry e = kernel_table(tc, bn, ak, bk);
                    if (!e.fn) continue;
                    if (cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem) !=
                        cudaSuccess) {
                        cudaGetLastError();
                        cudaFree(h->workspace);
                        cudaFree(h->error_word);
                        delete h;
                        return SHGEMM_STATUS_NOT_SUPPORTED;
                    }
                }
    for (int ak = 0; ak < 2; ++ak)
        for (int kc = 1; kc <= 2; ++kc)
            for (int sv = 0; sv < 2; ++sv) {
                KernelEntry e = tm_kernel_table(ak != 0, kc, sv);
                cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem);
            }
    for (int ak = 0; ak < 2; ++ak) {
        KernelEntry e = tm2_kernel_table(ak != 0);
        cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem);
        for (int bn : {128, 256}) {
            e = tile_wide_table(ak != 0, bn);
            cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem);
        }
    }
    h->max_pairs = query_max_pairs(tm2_kernel_table(true), sms);
    for (int tc = 0; tc < 2; ++tc)
        for (int ak = 0; ak < 2; ++ak)
            for (int bw = 0; bw < 2; ++bw) {
                KernelEntry e = grouped_table(tc, ak, bw != 0);
                cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem);
            }
    if (cudaGetLastError() != cudaSuccess || !table_alloc(h->grouped, kGroupedMaxProblems) ||
        !table_alloc(h->single, 1)) {
        cudaGetLastError();
        table_free(h->grouped);
        table_free(h->single);
        cudaFree(h->workspace);
        cudaFree(h->error_word);
        delete h;
        return SHGEMM_STATUS_ALLOC_FAILED;
    }
    *out = h;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_destroy(shgemm_b200_handle_t h) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    DeviceGuard g(h->device);
    shgemm_b200_release_host_staging(h);
    for (cudaEvent_t& e : h->host_ev)
        if (e) cudaEventDestroy(e);
    if (h->host_in) cudaStreamDestroy(h->host_in);
    if (h->host_out) cudaStreamDestroy(h->host_out);
    table_free(h->grouped);
    table_free(h->single);
    cudaFree(h->workspace);
    cudaFree(h->error_word);
    delete h;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_set_stream(shgemm_b200_handle_t h, void* s) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    h->stream = static_cast<cudaStream_t>(s);
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_set_kernel_level(shgemm_b200_handle_t h, int level) {
    if (!h || level < SHGEMM_LEVEL_AUTO || level > SHGEMM_LEVEL_P1) return SHGEMM_STATUS_INVALID_VALUE;
    h->fixed_level = level;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_set_debug_mode(shgemm_b200_handle_t h, unsigned on) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    h->debug_mode = on;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_set_config(shgemm_b200_handle_t h, int key, long long v) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    switch (key) {
        case SHGEMM_CFG_SPLIT_K:
            if (v < 0 || v > 1024) return SHGEMM_STATUS_INVALID_VALUE;
            h->split_k = v;
            return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_WAIT_LIMIT_MS:
            if (v < 1 || v > 600000) return SHGEMM_STATUS_INVALID_VALUE;
            h->wait_limit_ms = v;
            return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_GROUP_M:
            if (v < 1 || v > 1024) return SHGEMM_STATUS_INVALID_VALUE;
            h->group_m = v;
            return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_GROUPED_B_FP32:
            if (v != 0 && v != 1) return SHGEMM_STATUS_INVALID_VALUE;
            h->grouped_b_fp32 = static_cast<int>(v);
            return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_AUTOTUNE:
            if (v < 0 || v > 2) return SHGEMM_STATUS_INVALID_VALUE;
            h->autotune_mode = static_cast<int>(v);
            return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_TILE_KERNEL:
            if (v < 0 || v > 1) return SHGEMM_STATUS_INVALID_VALUE;
            h->tile_kernel = static_cast<int>(v);
            return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_K_CHUNK:
            if (v != 64 && v != 128) return SHGEMM_STATUS_INVALID_VALUE;
            h->k_chunk = static_cast<int>(v);
            return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_HOST_BLOCK_COLS:
            if (v < 0 || v >= (1ll << 31)) return SHGEMM_STATUS_INVALID_VALUE;
            h->host_block_cols = v;
            return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_TM_STAGES:
            if (v != 0 && v != 1) return SHGEMM_STATUS_INVALID_VALUE;
            h->tm_stages = static_cast<int>(v);
            return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_PAIR_TILES:
            if (v != 0 && v != 1) return SHGEMM_STATUS_INVALID_VALUE;
            h->pair_tiles = static_cast<int>(v);
            return SHGEMM_STATUS_OK;
        default:
            return SHGEMM_STATUS_INVALID_VALUE;
    }
}

int shgemm_b200_get_config(shgemm_b200_handle_t h, int key, long long* v) {
    if (!h || !v) return SHGEMM_STATUS_INVALID_VALUE;
    switch (key) {
        case SHGEMM_CFG_SPLIT_K: *v = h->split_k; return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_WAIT_LIMIT_MS: *v = h->wait_limit_ms; return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_GROUP_M: *v = h->group_m; return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_GROUPED_B_FP32: *v = h->grouped_b_fp32; return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_AUTOTUNE: *v = h->autotune_mode; return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_TILE_KERNEL: *v = h->tile_kernel; return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_K_CHUNK: *v = h->k_chunk; return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_HOST_BLOCK_COLS: *v = h->host_block_cols; return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_TM_STAGES: *v = h->tm_stages; return SHGEMM_STATUS_OK;
        case SHGEMM_CFG_PAIR_TILES: *v = h->pair_tiles; return SHGEMM_STATUS_OK;
        default: return SHGEMM_STATUS_INVALID_VALUE;
    }
}

int shgemm_b200_set_workspace_size(shgemm_b200_handle_t h, size_t bytes) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    DeviceGuard g(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return SHGEMM_STATUS_CUDA_ERROR;
    float* w = nullptr;
    if (bytes > 0 && cudaMalloc(&w, bytes) != cudaSuccess) {
        cudaGetLastError();
        return SHGEMM_STATUS_ALLOC_FAILED;
    }
    cudaFree(h->workspace);
    h->workspace = w;
    h->workspace_bytes = bytes;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_plan_preview(int num_sms, size_t m, size_t n, size_t k, int compute_type, size_t workspace_bytes,
                             int* level, int* tile_n, int* slices) {
    if (num_sms < 1 || (compute_type != SHGEMM_TC_FP16 && compute_type != SHGEMM_TC_TF32) || !level || !tile_n ||
        !slices || m == 0 || n == 0 || k == 0)
        return SHGEMM_STATUS_INVALID_VALUE;
    const Plan p = make_plan_for(num_sms, SHGEMM_LEVEL_AUTO, 0, m, n, k,
                                 compute_type == SHGEMM_TC_TF32 ? kTF32 : kFP16, workspace_bytes);
    *level = p.level;
    *tile_n = p.bn;
    *slices = p.slices;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_get_workspace(shgemm_b200_handle_t h, void** ptr, size_t* bytes) {
    if (!h || !ptr || !bytes) return SHGEMM_STATUS_INVALID_VALUE;
    *ptr = h->workspace;
    *bytes = h->workspace_bytes;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_check_error(shgemm_b200_handle_t h, int* device_code) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    DeviceGuard g(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return SHGEMM_STATUS_CUDA_ERROR;
    int code = 0;
    if (cudaMemcpy(&code, h->error_word, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SHGEMM_STATUS_CUDA_ERROR;
    if (code) cudaMemset(h->error_word, 0, sizeof(int));
    if (device_code) *device_code = code;
    return code ? SHGEMM_STATUS_TIMEOUT : SHGEMM_STATUS_OK;
}

int shgemm_b200_get_launch_count(shgemm_b200_handle_t h, long long* count) {
    if (!h || !count) return SHGEMM_STATUS_INVALID_VALUE;
    *count = h->launches.load();
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_generate_omega_batch(void* cuda_stream, const struct shgemm_b200_omega_job* jobs, int count,
                                     int fp32) {
    if (count < 0 || (count > 0 && !jobs) || (fp32 != 0 && fp32 != 1)) return SHGEMM_STATUS_INVALID_VALUE;
    for (int i = 0; i < count; ++i) {
        const shgemm_b200_omega_job& j = jobs[i];
        if ((j.dist != SHGEMM_OMEGA_GAUSSIAN && j.dist != SHGEMM_OMEGA_RADEMACHER &&
             j.dist != SHGEMM_OMEGA_RADEMACHER_BLOCKS) ||
            j.ld < j.k || (j.k > 0 && j.cols > 0 && !j.dst))
            return SHGEMM_STATUS_INVALID_VALUE;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (int first = 0; first < count; first += kOmegaJobsPerLaunch) {
        OmegaBatch b;
        std::memset(&b, 0, sizeof(b));
        b.fp32 = fp32;
        int n = 0;
        uint64_t most = 0, all = 0;
        for (int i = first; i < count && i < first + kOmegaJobsPerLaunch; ++i) {
            if (jobs[i].k == 0 || jobs[i].cols == 0) continue;
            b.job[n++] = jobs[i];
            const uint64_t items = jobs[i].dist == SHGEMM_OMEGA_GAUSSIAN ? (jobs[i].k + 1) / 2 * jobs[i].cols
                                                                         : static_cast<uint64_t>(jobs[i].k) * jobs[i].cols;
            most = std::max(most, items);
            all += items;
        }
        if (n == 0) continue;
        // blocks per job: the largest job's items, with the whole launch near 8 blocks per SM
        const uint64_t cap = std::max<uint64_t>(1, (static_cast<uint64_t>(sms) * 8 * most + all - 1) / all);
        const unsigned bx = static_cast<unsigned>(std::min<uint64_t>((most + 255) / 256, cap));
        omega_kernel<<<dim3(bx, n), 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(b);
        if (cudaGetLastError() != cudaSuccess) return SHGEMM_STATUS_LAUNCH_FAILED;
    }
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_generate_omega(void* cuda_stream, void* dst, size_t ld, size_t k, size_t cols, int dist,
                               unsigned long long seed, float scale, int fp32) {
    const shgemm_b200_omega_job j{dst, ld, k, cols, seed, scale, dist};
    return shgemm_b200_generate_omega_batch(cuda_stream, &j, 1, fp32);
}

int shgemm_b200_selftest_wait_timeout(shgemm_b200_handle_t h, unsigned limit_us, int* observed) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    DeviceGuard g(h->device);
    selftest_wait_kernel<<<1, 32, 0, h->stream>>>(h->error_word, static_cast<uint64_t>(limit_us) * 1000ull);
    h->launches++;
    if (launch_status() != SHGEMM_STATUS_OK) return SHGEMM_STATUS_LAUNCH_FAILED;
    int code = 0;
    const int st = shgemm_b200_check_error(h, &code);
    if (observed) *observed = code;
    return st;
}

}  // extern "C"

// Device-resident scalars for one call: each pointer, when set, replaces alpha or beta.
struct DevScalars {
    const float* alpha = nullptr;
    const float* beta = nullptr;
};

static int run_tiled(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                     const float* a, size_t lda, const void* b, size_t ldb, float beta, float* c, size_t ldc, int tc,
                     int op_c, int* level_out, float* splitk_ws, size_t splitk_bytes,
                     const shgemm_b200_tuned_config* force = nullptr, DevScalars dev = DevScalars{}) {
    int group_m = 8;
    const bool a_kmajor = (op_a == kOpT);
    const bool b_kmajor = (op_b == kOpN);
    const int bk = (tc == kFP16) ? 64 : 32;
    auto plan_with = [&](size_t ws_bytes) {
        return force ? plan_from_tuned(*force, m, n, k, tc, ws_bytes)
                     : make_plan(h, op_a, op_b, m, n, k, tc, ws_bytes, &group_m);
    };
    // A binary16 K-major operand whose columns lie >= 1 MiB apart puts each of a tile's 256
    // columns on a page of its own: every 64-deep step then needs 256 address translations
    // on top of the FP32 tile's, more than an SM's translation caches keep while streaming
    // (the loads run at about half speed). When the workspace has room, such a B is re-laid
    // out once per call as contiguous k-blocks (block_b_kernel) ahead of the split-K partials.
    const size_t kblocks = (k + 63) / 64;
    const size_t bblk_bytes = (kblocks * n * 128 + 255) / 256 * 256;
    bool block_b = tc == kFP16 && b_kmajor && h->tile_kernel == 0 && ldb * 2 >= kBlockBMinPitchBytes &&
                   splitk_bytes >= bblk_bytes && kblocks < (1u << 31);
    Plan pl{};
    if (block_b) {
        pl = plan_with(splitk_bytes - bblk_bytes);
        if (pl.bn != 256) block_b = false;
    }
    // TF32 compute with a K-major binary16 B and n > 64: when the workspace also holds B widened
    // to FP32 (ahead of the split-K partials), B is widened once per call and a 128 x 256 (or,
    // for n <= 128, 128 x 128) kernel loads it as the TF32 tile layout itself (the kernel that
    // widens B tile by tile in its split warps runs at about a third of the rate). Split-K as
    // usual.
    const int wide_bn = n > 128 ? 256 : 128;
    const size_t wkb = (k + 31) / 32;  // k-blocks of the widened B
    const size_t wide_bytes = (wkb * 32 * n * sizeof(float) + 255) / 256 * 256;
    bool wide_b = tc == kTF32 && b_kmajor && !force && h->tile_kernel == 0 &&
                        h->fixed_level == SHGEMM_LEVEL_AUTO && n > 64 && splitk_bytes >= wide_bytes &&
                        k <= static_cast<size_t>(INT32_MAX) && wkb * n < (size_t(1) << 31);
    if (wide_b) {
        // taken when it keeps enough SMs busy: the widened-B kernel does a unit's work ~3x as fast,
        // but the widened B leaves less room for split-K partials
        const Plan pw = make_plan_for(h->num_sms, h->fixed_level, h->split_k, m, n, k, tc, splitk_bytes - wide_bytes,
                                      wide_bn);
        int gm_n = 8;
        const Plan pn = make_plan(h, op_a, op_b, m, n, k, tc, splitk_bytes, &gm_n);
        auto busy = [&](const Plan& q) {
            const long long units = static_cast<long long>(q.tiles_m) * q.tiles_n * q.slices;
            return units >= h->num_sms ? wave_efficiency(units, h->num_sms)
                                       : static_cast<double>(units) / h->num_sms;
        };
        wide_b = 2.0 * busy(pw) >= busy(pn);
        if (wide_b) {
            group_m = static_cast<int>(h->group_m);
            pl = pw;
        } else {
            group_m = gm_n;
            pl = pn;
        }
    } else if (!block_b) {
        pl = plan_with(splitk_bytes);
    }
    if (force) group_m = force->group_m;
    float* part_ws = block_b ? splitk_ws + bblk_bytes / sizeof(float)
                             : wide_b ? splitk_ws + wide_bytes / sizeof(float) : splitk_ws;
    __half* b_blk = reinterpret_cast<__half*>(splitk_ws);
    float* b_wide = splitk_ws;
    // binary16 compute with 128 x 256 tiles and a K-major B: the tensor-memory operand kernel,
    // in CTA pairs (256 x 256 tiles, SHGEMM_CFG_PAIR_TILES) when B is not re-laid out and the
    // drain chunk and ring are the defaults
    const bool use_tm = tc == kFP16 && pl.bn == 256 && b_kmajor && h->tile_kernel == 0;
    const int kc = pl.kc ? pl.kc : h->k_chunk / 64;
    const int sv = pl.sv >= 0 ? pl.sv : h->tm_stages;
    const int pair = pl.pair >= 0 ? pl.pair : h->pair_tiles;
    const bool use_tm2 = use_tm && pair == 1 && !block_b && kc == 1 && sv == 0 && h->num_sms >= 2;

    TileGemmParams P;
    std::memset(&P, 0, sizeof(P));
    bool ok;
    // FP32 operand: K-major tiles are [128 rows][32 floats] with a 128-byte swizzle;
    // M-major tiles are [bk][box floats] unswizzled (one 128-wide box for the
    // tensor-memory kernel, a_mmajor_box(tc) wide boxes for the others).
    // The tensor-memory kernel loads a K-major tile as one 3-D box of whole 256-byte row
    // segments when k allows it (it streams at ~6.1 TB/s against ~4.4 TB/s for two
    // 128-byte-wide boxes over rows a full leading dimension apart).
    if (a_kmajor && use_tm && !use_tm2 && k % 32 == 0 && make_tmap_a_paired(&P.tmap_a, a, k, m, lda * 4)) {
        ok = true;
        P.a_rows_paired = 1;
    } else if (a_kmajor)
        ok = make_tmap(&P.tmap_a, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a, k, m, lda * 4, 32, 128,
                       CU_TENSOR_MAP_SWIZZLE_128B);
    else
        ok = make_tmap(&P.tmap_a, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a, m, k, lda * 4,
                       use_tm ? 128 : a_mmajor_box(tc, wide_b), bk, CU_TENSOR_MAP_SWIZZLE_NONE);
    if (!ok) return SHGEMM_STATUS_NOT_SUPPORTED;
    if (wide_b) {  // k-blocks {32 k, n columns, kblocks}: a [bn n][32 k] box is the TF32 tile layout
        ok = make_tmap_3d(&P.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, b_wide, 32, n, wkb, 128, n * 128, 32, wide_bn,
                          1, CU_TENSOR_MAP_SWIZZLE_128B);
    } else if (tc == kFP16) {
        if (block_b)  // k-blocks {64 k, n columns, kblocks}: one 64 x 256 tile step is 32 KB contiguous
            ok = make_tmap_3d(&P.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, b_blk, 64, n, kblocks, 128, n * 128, 64,
                              pl.bn, 1, CU_TENSOR_MAP_SWIZZLE_128B);
        else if (b_kmajor)  // CTA pairs: each CTA loads 64 of every 128 columns
            ok = make_tmap(&P.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, b, k, n, ldb * 2, 64, use_tm2 ? 64 : pl.bn,
                           CU_TENSOR_MAP_SWIZZLE_128B);
        else
            ok = make_tmap(&P.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, b, n, k, ldb * 2, 64, 64,
                           CU_TENSOR_MAP_SWIZZLE_128B);
    } else {
        if (b_kmajor)
            ok = make_tmap(&P.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, b, k, n, ldb * 2, 32, pl.bn,
                           CU_TENSOR_MAP_SWIZZLE_64B);
        else
            ok = make_tmap(&P.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, b, n, k, ldb * 2, pl.bn, 32,
                           CU_TENSOR_MAP_SWIZZLE_NONE);
    }
    if (!ok) return SHGEMM_STATUS_NOT_SUPPORTED;

    P.c = c;
    P.ldc = ldc;
    P.workspace = part_ws;
    P.error_flag = h->error_word;
    P.wait_limit_ns = static_cast<uint64_t>(h->wait_limit_ms) * 1000000ull;
    P.m = static_cast<int>(m);
    P.n = static_cast<int>(n);
    P.k = static_cast<int>(k);
    P.op_c = op_c;
    P.alpha = alpha;
    P.beta = beta;
    P.alpha_dev = dev.alpha;
    P.beta_dev = dev.beta;
    P.tiles_m = pl.tiles_m;
    P.tiles_n = pl.tiles_n;
    P.num_slices = pl.slices;
    P.steps_per_slice = pl.steps_per_slice;
    P.num_units = pl.tiles_m * pl.tiles_n * pl.slices;
    P.group_m = group_m;
    P.a_read_once = use_tm && !use_tm2 && pl.tiles_n == 1;
    P.b_blocked = (block_b || wide_b) ? 1 : 0;
    if (use_tm2) {  // pair tiles of 256 rows
        P.tiles_m = static_cast<int>((m + 255) / 256);
        P.num_units = P.tiles_m * pl.tiles_n * pl.slices;
    }

    const KernelEntry e = use_tm2 ? tm2_kernel_table(a_kmajor)
                          : use_tm ? tm_kernel_table(a_kmajor, kc, sv)
                          : wide_b ? tile_wide_table(a_kmajor, wide_bn)
                                   : kernel_table(tc, pl.bn, a_kmajor, b_kmajor);
    const int threads = use_tm ? TmCfg<true, 1, 0>::NUM_THREADS : 512;
    if (!e.fn) return SHGEMM_STATUS_NOT_SUPPORTED;
    // pairs: whole clusters of 2, one pair per two SMs
    const int grid = use_tm2 ? 2 * std::min(P.num_units, std::min(h->max_pairs, h->num_sms / 2))
                             : std::min(P.num_units, h->num_sms);
    if (h->debug_mode) {
        std::printf("[shape=(%zu,%zu,%zu),op_a=%s,op_b=%s,compute_type=%s] kernel_level = %d, tile = 128x%d, "
                    "k_slices = %d, chunk_k = %d, grid = %d%s\n",
                    m, n, k, op_a == kOpN ? "N" : "T", op_b == kOpN ? "N" : "T", tc == kTF32 ? "TF32" : "FP16",
                    pl.level, pl.bn, pl.slices, use_tm ? 64 * kc : bk, grid,
                    use_tm2 ? ", operands in TMEM, CTA pairs" : use_tm ? ", operands in TMEM"
                                                              : wide_b ? ", B widened to FP32" : "");
    }
    if (wide_b) {
        const size_t total = wkb * 32 * n;
        const int blocks = static_cast<int>(std::min<size_t>((total + 255) / 256, size_t(h->num_sms) * 16));
        widen_b_blocked_kernel<<<blocks, 256, 0, h->stream>>>(static_cast<const __half*>(b), ldb, b_wide,
                                                              static_cast<int>(k), static_cast<int>(n),
                                                              static_cast<int>(wkb));
        h->launches++;
        if (launch_status() != SHGEMM_STATUS_OK) return SHGEMM_STATUS_LAUNCH_FAILED;
    }
    if (block_b) {
        const size_t total = kblocks * n * 8;
        const int blocks = static_cast<int>(std::min<size_t>((total + 255) / 256, size_t(h->num_sms) * 16));
        block_b_kernel<<<blocks, 256, 0, h->stream>>>(static_cast<const __half*>(b), ldb, b_blk, static_cast<int>(k),
                                                      static_cast<int>(n), static_cast<int>(kblocks));
        h->launches++;
        if (launch_status() != SHGEMM_STATUS_OK) return SHGEMM_STATUS_LAUNCH_FAILED;
    }
    void* args[] = {&P};
    cudaError_t err = cudaLaunchKernel(e.fn, dim3(grid), dim3(threads), args, e.smem, h->stream);
    h->launches++;
    if (err != cudaSuccess) {
        cudaGetLastError();
        return SHGEMM_STATUS_LAUNCH_FAILED;
    }
    if (pl.slices > 1) {
        const size_t mn = m * n;
        const int blocks = static_cast<int>(std::min<size_t>((mn + 255) / 256, size_t(h->num_sms) * 8));
        splitk_reduce_kernel<<<blocks, 256, 0, h->stream>>>(part_ws, pl.slices, P.m, P.n, c, ldc, op_c, alpha, beta,
                                                            dev.alpha, dev.beta);
        h->launches++;
        if (launch_status() != SHGEMM_STATUS_OK) return SHGEMM_STATUS_LAUNCH_FAILED;
    }
    if (level_out) *level_out = (pl.slices > 1) ? SHGEMM_LEVEL_P0 : pl.level;
    return SHGEMM_STATUS_OK;
}

static size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

template <typename T>
static void launch_pack(shgemm_b200_handle_t h, const T* src, size_t ld_src, T* dst, size_t ld_dst, size_t rows,
                        size_t cols) {
    const size_t total = rows * cols;
    const int blocks = static_cast<int>(std::min<size_t>((total + 255) / 256, size_t(h->num_sms) * 16));
    pack_kernel<T><<<blocks, 256, 0, h->stream>>>(src, ld_src, dst, ld_dst, static_cast<int>(rows),
                                                  static_cast<int>(cols));
    h->launches++;
}

// TF32 compute with a K-contiguous binary16 B: widen B once into the handle's workspace
// and run the 128 x 256 TF32 kernel that loads FP32 B unconverted (the grouped kernel on
// a one-problem table). Taken only for eager calls (not while capturing: a captured
// grouped launch replays whatever table the handle stages later), when the workspace
// holds the widened B, and when 128 x 256 tiles fill the GPU (no split-K wanted);
// otherwise SHGEMM_STATUS_NOT_SUPPORTED and the caller uses the tile kernel.
// Stages a batch into table `t` and enqueues its copy and one grouped launch (defined with
// the grouped entry points below).
static int grouped_run(shgemm_b200_handle_t h, GroupedTable& t, bool b_wide, int op_a, int op_b, int tc, int op_c,
                       const shgemm_b200_problem* probs, int count, DevScalars dev = DevScalars{});

static int tf32_widened_b(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                          const float* a, size_t lda, const void* b, size_t ldb, float beta, float* c, size_t ldc,
                          int op_c, int* level_out, DevScalars dev) {
    if (op_b != kOpN || !h->single.dev || h->tile_kernel != 0 || h->fixed_level != SHGEMM_LEVEL_AUTO ||
        h->split_k > 1)
        return SHGEMM_STATUS_NOT_SUPPORTED;
    const size_t ldw = (k + 3) / 4 * 4;
    if (ldw * n * sizeof(float) > h->workspace_bytes) return SHGEMM_STATUS_NOT_SUPPORTED;
    const long long tiles = static_cast<long long>((m + 127) / 128) * static_cast<long long>((n + 255) / 256);
    if (tiles < h->num_sms || tiles > kGroupedMaxUnits) return SHGEMM_STATUS_NOT_SUPPORTED;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return SHGEMM_STATUS_NOT_SUPPORTED;
    }
    const size_t total = k * n;
    const int blocks = static_cast<int>(std::min<size_t>((total + 255) / 256, size_t(h->num_sms) * 16));
    widen_b_kernel<<<blocks, 256, 0, h->stream>>>(static_cast<const __half*>(b), ldb, h->workspace, ldw,
                                                  static_cast<int>(k), static_cast<int>(n));
    h->launches++;
    if (launch_status() != SHGEMM_STATUS_OK) return SHGEMM_STATUS_LAUNCH_FAILED;
    shgemm_b200_problem q{};
    q.m = m;
    q.n = n;
    q.k = k;
    q.a = a;
    q.lda = lda;
    q.b = h->workspace;
    q.ldb = ldw;
    q.c = c;
    q.ldc = ldc;
    q.alpha = alpha;
    q.beta = beta;
    // the handle's own one-problem table: the caller's grouped staging, which a captured
    // graph may replay, is left untouched
    const int st = grouped_run(h, h->single, true, op_a, kOpN, kTF32, op_c, &q, 1, dev);
    if (st == SHGEMM_STATUS_OK && level_out) *level_out = SHGEMM_LEVEL_P1;
    return st;
}

// The dispatch behind shgemm_b200_shgemm (host scalars: alpha, beta) and
// shgemm_b200_shgemm_device_scalars (dev.alpha / dev.beta device addresses, read by the kernels).
static int shgemm_impl(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                       const float* a, size_t lda, const void* b, size_t ldb, float beta, float* c, size_t ldc,
                       int tc, int op_c, int* level_out, DevScalars dev) {
    if ((op_a != kOpN && op_a != kOpT) || (op_b != kOpN && op_b != kOpT) || (op_c != kOpN && op_c != kOpT) ||
        (tc != kFP16 && tc != kTF32))
        return SHGEMM_STATUS_INVALID_VALUE;
    if (m == 0 || n == 0) {
        if (level_out) *level_out = SHGEMM_LEVEL_P0;
        return SHGEMM_STATUS_OK;
    }
    const size_t a_rows = (op_a == kOpN) ? m : k;
    const size_t b_rows = (op_b == kOpN) ? k : n;
    const size_t c_rows = (op_c == kOpN) ? m : n;
    if (!c || ldc < c_rows) return SHGEMM_STATUS_INVALID_VALUE;
    if (k > 0 && (!a || !b || lda < std::max<size_t>(1, a_rows) || ldb < std::max<size_t>(1, b_rows)))
        return SHGEMM_STATUS_INVALID_VALUE;
    if (m >= (1u << 31) || n >= (1u << 31) || k >= (1u << 31)) return SHGEMM_STATUS_NOT_SUPPORTED;
    DeviceGuard g(h->device);

    if (k == 0) {  // empty product: C = beta * C
        const size_t rows = c_rows, cols = (op_c == kOpN) ? n : m;
        const int blocks = static_cast<int>(std::min<size_t>((rows * cols + 255) / 256, 4096));
        scale_c_kernel<<<blocks, 256, 0, h->stream>>>(c, ldc, static_cast<int>(rows), static_cast<int>(cols), beta,
                                                      dev.beta);
        h->launches++;
        if (level_out) *level_out = SHGEMM_LEVEL_P0;
        return launch_status();
    }
    // TMA addresses 16-byte aligned bases with 16-byte aligned leading dimensions.
    const bool pack_a = (reinterpret_cast<uintptr_t>(a) & 15) || (lda * 4) % 16;
    const bool pack_b = (reinterpret_cast<uintptr_t>(b) & 15) || (ldb * 2) % 16;
    if (!pack_a && !pack_b) {
        if (tc == kTF32) {
            const int st =
                tf32_widened_b(h, op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, op_c, level_out, dev);
            if (st != SHGEMM_STATUS_NOT_SUPPORTED) return st;
        }
        // SHGEMM_CFG_AUTOTUNE = 2: an untuned bucket is tuned on this call's operands first
        // (C is overwritten by the candidates, harmless when beta == 0 and C is laid out op_n).
        if (h->autotune_mode == 2 && beta == 0.0f && !dev.beta && op_c == kOpN &&
            h->fixed_level == SHGEMM_LEVEL_AUTO && h->split_k == 0) {
            bool have;
            {
                std::lock_guard<std::mutex> lk(h->tune_mu);
                have = h->tuned.count(tune_key(tc, op_a, op_b, m, n, k)) != 0;
            }
            cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
            if (!have && cudaStreamIsCapturing(h->stream, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone) {
                const int st = shgemm_b200_autotune(h, op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc, tc, nullptr);
                if (st != SHGEMM_STATUS_OK) return st;
            }
            cudaGetLastError();
        }
        return run_tiled(h, op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, tc, op_c, level_out,
                         h->workspace, h->workspace_bytes, nullptr, dev);
    }

    // Staging path: copy the unaligned operand(s) slab by slab (k-slabs of a multiple
    // of 64) into the handle's workspace with aligned leading dimensions, then run the
    // tile kernel per slab, accumulating into C (beta for the first slab, 1 after).
    auto a_bytes = [&](size_t kb) { return pack_a ? (op_a == kOpN ? round_up(m, 4) * kb : round_up(kb, 4) * m) * 4 : 0; };
    auto b_bytes = [&](size_t kb) { return pack_b ? (op_b == kOpN ? round_up(kb, 8) * n : round_up(n, 8) * kb) * 2 : 0; };
    size_t kb = k;
    while (round_up(a_bytes(kb), 256) + round_up(b_bytes(kb), 256) > h->workspace_bytes) {
        if (kb <= 64) return SHGEMM_STATUS_NOT_SUPPORTED;  // even one 64-deep slab does not fit
        kb = std::max<size_t>(64, round_up(kb / 2, 64));
    }
    float* a_st = h->workspace;
    __half* b_st = reinterpret_cast<__half*>(reinterpret_cast<char*>(h->workspace) + round_up(a_bytes(kb), 256));
    int level = SHGEMM_LEVEL_P0;
    for (size_t k0 = 0; k0 < k; k0 += kb) {
        const size_t kk = std::min(kb, k - k0);
        const float* as;
        size_t lda_s;
        if (pack_a) {
            if (op_a == kOpN) {
                lda_s = round_up(m, 4);
                launch_pack<float>(h, a + k0 * lda, lda, a_st, lda_s, m, kk);
            } else {
                lda_s = round_up(kk, 4);
                launch_pack<float>(h, a + k0, lda, a_st, lda_s, kk, m);
            }
            as = a_st;
        } else {
            as = (op_a == kOpN) ? a + k0 * lda : a + k0;
            lda_s = lda;
        }
        const __half* bh = static_cast<const __half*>(b);
        const __half* bs;
        size_t ldb_s;
        if (pack_b) {
            if (op_b == kOpN) {
                ldb_s = round_up(kk, 8);
                launch_pack<__half>(h, bh + k0, ldb, b_st, ldb_s, kk, n);
            } else {
                ldb_s = round_up(n, 8);
                launch_pack<__half>(h, bh + k0 * ldb, ldb, b_st, ldb_s, n, kk);
            }
            bs = b_st;
        } else {
            bs = (op_b == kOpN) ? bh + k0 : bh + k0 * ldb;
            ldb_s = ldb;
        }
        if (launch_status() != SHGEMM_STATUS_OK) return SHGEMM_STATUS_LAUNCH_FAILED;
        DevScalars ds = dev;
        if (k0 > 0) ds.beta = nullptr;  // later slabs accumulate: beta = 1
        const int st = run_tiled(h, op_a, op_b, m, n, kk, alpha, as, lda_s, bs, ldb_s, k0 == 0 ? beta : 1.0f, c,
                                 ldc, tc, op_c, &level, nullptr, 0, nullptr, ds);
        if (st != SHGEMM_STATUS_OK) return st;
    }
    if (level_out) *level_out = level;
    return SHGEMM_STATUS_OK;
}

extern "C" {

int shgemm_b200_shgemm(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k,
                       const float* alpha_ptr, const float* a, size_t lda, const void* b, size_t ldb,
                       const float* beta_ptr, float* c, size_t ldc, int tc, int op_c, int* level_out) {
    if (!h || !alpha_ptr || !beta_ptr) return SHGEMM_STATUS_INVALID_VALUE;
    return shgemm_impl(h, op_a, op_b, m, n, k, *alpha_ptr, a, lda, b, ldb, *beta_ptr, c, ldc, tc, op_c, level_out,
                       DevScalars{});
}

int shgemm_b200_shgemm_device_scalars(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                      const float* alpha_dev, const float* a, size_t lda, const void* b, size_t ldb,
                                      const float* beta_dev, float* c, size_t ldc, int tc, int op_c,
                                      int* level_out) {
    if (!h || !alpha_dev || !beta_dev) return SHGEMM_STATUS_INVALID_VALUE;
    if ((reinterpret_cast<uintptr_t>(alpha_dev) & 3) || (reinterpret_cast<uintptr_t>(beta_dev) & 3))
        return SHGEMM_STATUS_INVALID_VALUE;
    DevScalars dev;
    dev.alpha = alpha_dev;
    dev.beta = beta_dev;
    // alpha = 1, beta = 1 stand in on the host: the kernels read the device values, and with
    // beta != 0 on the host side nothing assumes that C may be left unread
    return shgemm_impl(h, op_a, op_b, m, n, k, 1.0f, a, lda, b, ldb, 1.0f, c, ldc, tc, op_c, level_out, dev);
}

int shgemm_b200_hsgemm_device_scalars(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                      const float* alpha_dev, const void* a, size_t lda, const float* b, size_t ldb,
                                      const float* beta_dev, float* c, size_t ldc, int tc, int op_c,
                                      int* level_out) {
    // the transposition identity of shgemm_b200_hsgemm (include/shgemm/shgemm.hpp:142-156)
    auto inv = [](int op) { return op == kOpN ? kOpT : kOpN; };
    if ((op_a != kOpN && op_a != kOpT) || (op_b != kOpN && op_b != kOpT) || (op_c != kOpN && op_c != kOpT))
        return SHGEMM_STATUS_INVALID_VALUE;
    return shgemm_b200_shgemm_device_scalars(h, inv(op_b), inv(op_a), n, m, k, alpha_dev, b, ldb, a, lda, beta_dev,
                                             c, ldc, tc, inv(op_c), level_out);
}

// ---------------------------------------------------------------- autotuner
static bool tile_n_valid(int tc, int bn) { return bn == 64 || bn == 128 || (bn == 256 && tc == kFP16); }

// Median device time of `reps` runs of one configuration (after one untimed run).
static int time_config(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k, const float* a,
                       size_t lda, const void* b, size_t ldb, float* c, size_t ldc, int tc,
                       const shgemm_b200_tuned_config& cfg, int reps, float* us) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        if (e0) cudaEventDestroy(e0);
        return SHGEMM_STATUS_CUDA_ERROR;
    }
    int lvl = 0, st = SHGEMM_STATUS_OK;
    std::vector<float> t;
    for (int r = -1; r < reps && st == SHGEMM_STATUS_OK; ++r) {
        cudaEventRecord(e0, h->stream);
        st = run_tiled(h, op_a, op_b, m, n, k, 1.0f, a, lda, b, ldb, 0.0f, c, ldc, tc, kOpN, &lvl, h->workspace,
                       h->workspace_bytes, &cfg);
        cudaEventRecord(e1, h->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = SHGEMM_STATUS_CUDA_ERROR;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r >= 0) t.push_back(ms * 1000.0f);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != SHGEMM_STATUS_OK) {
        cudaGetLastError();
        return st;
    }
    int code = 0;
    if (shgemm_b200_check_error(h, &code) != SHGEMM_STATUS_OK) return SHGEMM_STATUS_TIMEOUT;
    std::sort(t.begin(), t.end());
    *us = t[t.size() / 2];
    return SHGEMM_STATUS_OK;
}

// The k-chunk accuracy gate samples up to two blocks of C: the top-left and the bottom-right
// 128 x 128 (one block when they coincide).
static int sampled_blocks(size_t m, size_t n, size_t* r0, size_t* c0, size_t* bm, size_t* bn) {
    *bm = std::min<size_t>(m, 128);
    *bn = std::min<size_t>(n, 128);
    r0[0] = 0;
    c0[0] = 0;
    r0[1] = m - *bm;
    c0[1] = n - *bn;
    return (r0[1] == 0 && c0[1] == 0) ? 1 : 2;
}

// Relative Frobenius error against FP64 (ref64, one buffer per block) of the op_n result C
// over the sampled blocks; SHGEMM_STATUS_INVALID_VALUE when C and FP64 disagree on finiteness.
static int block_error(shgemm_b200_handle_t h, size_t m, size_t n, const float* c, size_t ldc, double* const* ref64,
                       double* err) {
    size_t r0[2], c0[2], bm, bn;
    const int nb = sampled_blocks(m, n, r0, c0, &bm, &bn);
    double d2 = 0, r2 = 0;
    for (int i = 0; i < nb; ++i) {
        double out[4];
        const int st = shgemm_b200_eval_error(h, bm, bn, c + r0[i] + c0[i] * ldc, ldc, kOpN, ref64[i], 1.0, 0.0,
                                              nullptr, out);
        if (st != SHGEMM_STATUS_OK) return st;
        if (out[3] != 0) return SHGEMM_STATUS_INVALID_VALUE;
        d2 += out[0] * out[0];
        r2 += out[1] * out[1];
    }
    *err = r2 > 0 ? std::sqrt(d2 / r2) : std::sqrt(d2);
    return SHGEMM_STATUS_OK;
}

// The accuracy gate of the 128-k chunk: its sampled error against FP64 at most 1.25x the
// 64-k chunk's (plus an FP32-ulp floor). The FP64 blocks come from the library's evaluation
// kernels on the same operands.
static int k_chunk_gate(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k, const float* a,
                        size_t lda, const void* b, size_t ldb, float* c, size_t ldc, int tc,
                        shgemm_b200_tuned_config cfg64, shgemm_b200_tuned_config cfg128, bool* pass,
                        double* e64_out, double* e128_out) {
    *pass = false;
    size_t r0[2], c0[2], bm, bn;
    const int nb = sampled_blocks(m, n, r0, c0, &bm, &bn);
    double* ref[2] = {nullptr, nullptr};
    int st = SHGEMM_STATUS_OK;
    for (int i = 0; i < nb && st == SHGEMM_STATUS_OK; ++i) {
        if (cudaMalloc(&ref[i], bm * bn * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            st = SHGEMM_STATUS_ALLOC_FAILED;
            break;
        }
        const float* ab = op_a == kOpN ? a + r0[i] : a + r0[i] * lda;
        const __half* bh = static_cast<const __half*>(b);
        const __half* bb = op_b == kOpN ? bh + c0[i] * ldb : bh + c0[i];
        st = shgemm_b200_eval_dgemm(h, op_a, op_b, bm, bn, k, ab, lda, bb, ldb, ref[i]);
    }
    double e[2] = {0, 0};
    for (int j = 0; j < 2 && st == SHGEMM_STATUS_OK; ++j) {
        int lvl = 0;
        st = run_tiled(h, op_a, op_b, m, n, k, 1.0f, a, lda, b, ldb, 0.0f, c, ldc, tc, kOpN, &lvl, h->workspace,
                       h->workspace_bytes, j == 0 ? &cfg64 : &cfg128);
        if (st == SHGEMM_STATUS_OK && cudaStreamSynchronize(h->stream) != cudaSuccess) st = SHGEMM_STATUS_CUDA_ERROR;
        if (st == SHGEMM_STATUS_OK) {
            int code = 0;
            if (shgemm_b200_check_error(h, &code) != SHGEMM_STATUS_OK) st = SHGEMM_STATUS_TIMEOUT;
        }
        if (st == SHGEMM_STATUS_OK) {
            const int be = block_error(h, m, n, c, ldc, ref, &e[j]);
            if (be == SHGEMM_STATUS_INVALID_VALUE)
                e[j] = 1e300;  // a finite/non-finite disagreement: the candidate fails
            else
                st = be;
        }
    }
    for (double* r : ref) cudaFree(r);
    if (st != SHGEMM_STATUS_OK) {
        cudaGetLastError();
        return st;
    }
    *e64_out = e[0];
    *e128_out = e[1];
    *pass = e[1] <= 1.25 * e[0] + 4.0 * 5.9604644775390625e-8;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_autotune(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k, const float* a,
                         size_t lda, const void* b, size_t ldb, float* c, size_t ldc, int tc,
                         shgemm_b200_tuned_config* best_out) {
    if (!h || !c || m == 0 || n == 0 || k == 0 || !a || !b) return SHGEMM_STATUS_INVALID_VALUE;
    if ((op_a != kOpN && op_a != kOpT) || (op_b != kOpN && op_b != kOpT) || (tc != kFP16 && tc != kTF32))
        return SHGEMM_STATUS_INVALID_VALUE;
    if (ldc < m || lda < (op_a == kOpN ? m : k) || ldb < (op_b == kOpN ? k : n)) return SHGEMM_STATUS_INVALID_VALUE;
    if ((reinterpret_cast<uintptr_t>(a) & 15) || (lda * 4) % 16 || (reinterpret_cast<uintptr_t>(b) & 15) ||
        (ldb * 2) % 16 || m >= (1u << 31) || n >= (1u << 31) || k >= (1u << 31))
        return SHGEMM_STATUS_NOT_SUPPORTED;
    DeviceGuard g(h->device);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return SHGEMM_STATUS_NOT_SUPPORTED;
    }
    const int bk = tc == kFP16 ? 64 : 32;
    const int steps = static_cast<int>((k + bk - 1) / bk);
    const size_t per_slice = m * n * sizeof(float);
    const int fit = static_cast<int>(std::min<size_t>(h->workspace_bytes / per_slice, 1024));
    const int tile_ns[] = {64, 128, 256};
    const int slice_set[] = {1, 2, 3, 4, 6, 8, 12, 16};
    auto cfg_of = [](int bn, int sl, int gm, int sv, int kchunk, int cg = 1) {
        shgemm_b200_tuned_config c{};
        c.tile_n = bn;
        c.slices = sl;
        c.group_m = gm;
        c.stages = sv;
        c.k_chunk = kchunk;
        c.cta_group = cg;
        return c;
    };
    auto same = [](const shgemm_b200_tuned_config& x, const shgemm_b200_tuned_config& y) {
        return x.tile_n == y.tile_n && x.slices == y.slices && x.group_m == y.group_m && x.stages == y.stages &&
               x.k_chunk == y.k_chunk && x.cta_group == y.cta_group;
    };
    // one timed run of the heuristic plan sizes the repetitions
    shgemm_b200_tuned_config best{};
    {
        const Plan hp = make_plan_for(h->num_sms, SHGEMM_LEVEL_AUTO, 0, m, n, k, tc, h->workspace_bytes);
        best = cfg_of(hp.bn, hp.slices, static_cast<int>(h->group_m), h->tm_stages, 64, h->pair_tiles ? 2 : 1);
        const int st = time_config(h, op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc, tc, best, 1, &best.time_us);
        if (st != SHGEMM_STATUS_OK) return st;
    }
    const int reps = best.time_us > 50000.0f ? 1 : 3;
    auto consider = [&](shgemm_b200_tuned_config cand) -> int {
        if (same(cand, best) && best.time_us < 3.0e38f) return SHGEMM_STATUS_OK;
        const int st = time_config(h, op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc, tc, cand, reps, &cand.time_us);
        if (st != SHGEMM_STATUS_OK) return st;
        if (cand.time_us < best.time_us) best = cand;
        return SHGEMM_STATUS_OK;
    };
    {
        // re-time the heuristic plan with the same repetitions as the candidates
        shgemm_b200_tuned_config heur = best;
        best.time_us = 3.4e38f;
        const int st = consider(heur);
        if (st != SHGEMM_STATUS_OK) return st;
    }
    for (int bn : tile_ns) {
        if (!tile_n_valid(tc, bn)) continue;
        const long long tiles = static_cast<long long>((m + 127) / 128) * static_cast<long long>((n + bn - 1) / bn);
        for (int sl : slice_set) {
            if (sl > 1 && (sl > fit || steps / sl < 4 || tiles >= 2LL * h->num_sms)) continue;
            const int st = consider(cfg_of(bn, sl, static_cast<int>(h->group_m), best.stages, 64));
            if (st != SHGEMM_STATUS_OK) return st;
        }
    }
    for (int gm : {2, 4, 8, 16, 32}) {
        const int st = consider(cfg_of(best.tile_n, best.slices, gm, best.stages, 64));
        if (st != SHGEMM_STATUS_OK) return st;
    }
    // The 128 x 256 binary16 tiles of the tensor-memory kernel: its operand ring, then the
    // 128-k drain chunk, which is kept only if it is faster and passes the accuracy gate.
    const bool tm = tc == kFP16 && best.tile_n == 256 && op_b == kOpN && h->tile_kernel == 0;
    double gate_e64 = -1, gate_e128 = -1;
    int gate = -1;  // -1 not run, 0 failed, 1 passed
    if (tm) {
        int st = consider(cfg_of(best.tile_n, best.slices, best.group_m, 1 - best.stages, 64));
        if (st != SHGEMM_STATUS_OK) return st;
        // CTA pairs (256 x 256 tiles over two SMs): the default ring and drain chunk only
        st = consider(cfg_of(best.tile_n, best.slices, best.group_m, 0, 64, 2));
        if (st != SHGEMM_STATUS_OK) return st;
        shgemm_b200_tuned_config c128 = cfg_of(best.tile_n, best.slices, best.group_m, best.stages, 128);
        if (best.cta_group != 2)
            st = time_config(h, op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc, tc, c128, reps, &c128.time_us);
        if (st != SHGEMM_STATUS_OK) return st;
        if (best.cta_group != 2 && c128.time_us < best.time_us) {
            bool pass = false;
            st = k_chunk_gate(h, op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc, tc, best, c128, &pass, &gate_e64,
                              &gate_e128);
            if (st != SHGEMM_STATUS_OK) return st;
            gate = pass ? 1 : 0;
            if (pass) best = c128;
        }
    }
    {
        std::lock_guard<std::mutex> lk(h->tune_mu);
        h->tuned[tune_key(tc, op_a, op_b, m, n, k)] = best;
    }
    if (h->debug_mode) {
        std::printf("[autotune] (%zu,%zu,%zu) %s: tile = 128x%d, k_slices = %d, group_m = %d, stages = %d, "
                    "k_chunk = %d, cta_group = %d, %.1f us\n",
                    m, n, k, tc == kTF32 ? "TF32" : "FP16", best.tile_n, best.slices, best.group_m, best.stages,
                    best.k_chunk, best.cta_group, best.time_us);
        if (gate >= 0)
            std::printf("[autotune] k_chunk 128 accuracy gate %s: sampled error %.3e vs %.3e at 64\n",
                        gate ? "passed" : "failed", gate_e128, gate_e64);
    }
    if (best_out) *best_out = best;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_autotune_lookup(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k, int tc,
                                shgemm_b200_tuned_config* cfg) {
    if (!h || !cfg || m == 0 || n == 0 || k == 0) return SHGEMM_STATUS_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(h->tune_mu);
    auto it = h->tuned.find(tune_key(tc, op_a, op_b, m, n, k));
    if (it == h->tuned.end()) return SHGEMM_STATUS_INVALID_VALUE;
    *cfg = it->second;
    return SHGEMM_STATUS_OK;
}

// Text format, one entry per line:
//   kind tc op_a op_b log2m log2n log2k tile_n slices group_m stages k_chunk cta_group time_us
// kind 0: a plain shape bucket; kind 1: a grouped n bucket (op_b holds the B format, 1 =
// FP32; log2m and log2k are 0). Lines of the earlier 10-field form (no kind, stages and
// k_chunk) load as plain entries with the default ring and a 64-k chunk.
int shgemm_b200_autotune_save(shgemm_b200_handle_t h, const char* path) {
    if (!h || !path) return SHGEMM_STATUS_INVALID_VALUE;
    FILE* f = std::fopen(path, "w");
    if (!f) return SHGEMM_STATUS_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(h->tune_mu);
    std::fprintf(f, "# shgemm_b200 autotune v2: kind tc op_a op_b log2m log2n log2k tile_n slices group_m stages "
                    "k_chunk cta_group time_us\n");
    for (const auto& kv : h->tuned) {
        const uint64_t key = kv.first;
        const shgemm_b200_tuned_config& t = kv.second;
        std::fprintf(f, "%d %d %d %d %d %d %d %d %d %d %d %d %d %.3f\n", (key & kTuneGrouped) ? 1 : 0,
                     static_cast<int>((key >> 27) & 1), static_cast<int>((key >> 26) & 1),
                     static_cast<int>((key >> 25) & 1), static_cast<int>((key >> 16) & 0xFF),
                     static_cast<int>((key >> 8) & 0xFF), static_cast<int>(key & 0xFF), t.tile_n, t.slices, t.group_m,
                     t.stages, t.k_chunk, t.cta_group, t.time_us);
    }
    const bool ok = std::fclose(f) == 0;
    return ok ? SHGEMM_STATUS_OK : SHGEMM_STATUS_INVALID_VALUE;
}

int shgemm_b200_autotune_load(shgemm_b200_handle_t h, const char* path) {
    if (!h || !path) return SHGEMM_STATUS_INVALID_VALUE;
    FILE* f = std::fopen(path, "r");
    if (!f) return SHGEMM_STATUS_INVALID_VALUE;
    char line[256];
    int status = SHGEMM_STATUS_OK;
    std::map<uint64_t, shgemm_b200_tuned_config> add;
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        int kind = 0, tc, oa, ob, lm, ln, lk, bn, sl, gm, sv = 0, kch = 64, cg = 1;
        float us;
        const int got = std::sscanf(line, "%d %d %d %d %d %d %d %d %d %d %d %d %d %f", &kind, &tc, &oa, &ob, &lm, &ln,
                                    &lk, &bn, &sl, &gm, &sv, &kch, &cg, &us);
        if (got != 14) {  // the earlier form: tc op_a op_b log2m log2n log2k tile_n slices group_m time_us
            kind = 0;
            sv = 0;
            kch = 64;
            cg = 1;
            if (std::sscanf(line, "%d %d %d %d %d %d %d %d %d %f", &tc, &oa, &ob, &lm, &ln, &lk, &bn, &sl, &gm, &us) !=
                10) {
                status = SHGEMM_STATUS_INVALID_VALUE;
                break;
            }
        }
        const bool bad_common = (kind != 0 && kind != 1) || (tc != kFP16 && tc != kTF32) || (oa != 0 && oa != 1) ||
                                (ob != 0 && ob != 1) || lm < 0 || lm > 40 || ln < 0 || ln > 40 || lk < 0 || lk > 40;
        const bool bad_plain = kind == 0 && (!tile_n_valid(tc, bn) || sl < 1 || sl > 1024 || gm < 1 || gm > 1024 ||
                                             (sv != 0 && sv != 1) || (kch != 64 && kch != 128) || (cg != 1 && cg != 2));
        const bool bad_grouped = kind == 1 && !(bn == 32 || bn == 64 || bn == 128 || bn == 256);
        if (bad_common || bad_plain || bad_grouped) {
            status = SHGEMM_STATUS_INVALID_VALUE;
            break;
        }
        shgemm_b200_tuned_config t{};
        t.tile_n = bn;
        t.slices = kind ? 1 : sl;
        t.group_m = kind ? 1 : gm;
        t.time_us = us;
        t.stages = kind ? 0 : sv;
        t.k_chunk = kind ? 64 : kch;
        t.cta_group = kind ? 1 : cg;
        uint64_t key;
        if (kind == 1) {
            key = tune_key_grouped(tc, oa, ob, ln);
        } else {
            key = (static_cast<uint64_t>(tc) << 27) | (static_cast<uint64_t>(oa) << 26) |
                  (static_cast<uint64_t>(ob) << 25) | (static_cast<uint64_t>(lm) << 16) |
                  (static_cast<uint64_t>(ln) << 8) | static_cast<uint64_t>(lk);
        }
        add[key] = t;
    }
    std::fclose(f);
    if (status != SHGEMM_STATUS_OK) return status;
    std::lock_guard<std::mutex> lk(h->tune_mu);
    for (const auto& kv : add) h->tuned[kv.first] = kv.second;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_autotune_clear(shgemm_b200_handle_t h) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(h->tune_mu);
    h->tuned.clear();
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_hsgemm(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k,
                       const float* alpha, const void* a, size_t lda, const float* b, size_t ldb, const float* beta,
                       float* c, size_t ldc, int tc, int op_c, int* level_out) {
    // C = A B  <=>  C^T = B^T A^T with the FP32 operand on the left and C written
    // transposed (include/shgemm/shgemm.hpp:142-156).
    auto inv = [](int op) { return op == kOpN ? kOpT : kOpN; };
    if ((op_a != kOpN && op_a != kOpT) || (op_b != kOpN && op_b != kOpT) || (op_c != kOpN && op_c != kOpT))
        return SHGEMM_STATUS_INVALID_VALUE;
    return shgemm_b200_shgemm(h, inv(op_b), inv(op_a), n, m, k, alpha, b, ldb, a, lda, beta, c, ldc, tc, inv(op_c),
                              level_out);
}

int shgemm_b200_release_host_staging(shgemm_b200_handle_t h) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    if (!h->host_stage) return SHGEMM_STATUS_OK;
    DeviceGuard g(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return SHGEMM_STATUS_CUDA_ERROR;
    if (h->host_in) cudaStreamSynchronize(h->host_in);
    if (h->host_out) cudaStreamSynchronize(h->host_out);
    cudaFree(h->host_stage);
    h->host_stage = nullptr;
    h->host_stage_bytes = 0;
    return SHGEMM_STATUS_OK;
}

// Host-buffer SHGEMM. A goes to the device once; C is then produced in column blocks that
// rotate through three staging slots: the copy-in stream brings block j's B columns (and C
// columns when beta != 0) while the handle's stream computes block j - 1 with the device
// entry point and the copy-out stream returns block j - 2, so both copy directions overlap
// the tensor work; the third slot lets block j + 1 go up before block j - 2 has come back
// (with two, the upload stream waited for every download). Events order the three streams;
// the handle's stream waits for the last copy-outs, so synchronising it covers the call.
int shgemm_b200_shgemm_host(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k,
                            const float* alpha_ptr, const float* a, size_t lda, const void* b, size_t ldb,
                            const float* beta_ptr, float* c, size_t ldc, int tc, int op_c, int* level_out) {
    if (!h || !alpha_ptr || !beta_ptr) return SHGEMM_STATUS_INVALID_VALUE;
    if ((op_a != kOpN && op_a != kOpT) || (op_b != kOpN && op_b != kOpT) || (op_c != kOpN && op_c != kOpT) ||
        (tc != kFP16 && tc != kTF32))
        return SHGEMM_STATUS_INVALID_VALUE;
    if (m == 0 || n == 0) {
        if (level_out) *level_out = SHGEMM_LEVEL_P0;
        return SHGEMM_STATUS_OK;
    }
    const size_t a_rows = (op_a == kOpN) ? m : k, a_cols = (op_a == kOpN) ? k : m;
    const size_t b_rows = (op_b == kOpN) ? k : n;
    const size_t c_rows = (op_c == kOpN) ? m : n;
    if (!c || ldc < c_rows) return SHGEMM_STATUS_INVALID_VALUE;
    if (k > 0 && (!a || !b || lda < std::max<size_t>(1, a_rows) || ldb < std::max<size_t>(1, b_rows)))
        return SHGEMM_STATUS_INVALID_VALUE;
    if (m >= (1u << 31) || n >= (1u << 31) || k >= (1u << 31)) return SHGEMM_STATUS_NOT_SUPPORTED;
    const float alpha = *alpha_ptr, beta = *beta_ptr;
    DeviceGuard g(h->device);

    // column blocks: a multiple of the 256-wide tile, about sixteen per call by default (the
    // last block's compute and download are the part no upload hides)
    constexpr int kSlots = 3;
    size_t nb = h->host_block_cols > 0 ? static_cast<size_t>(h->host_block_cols)
                                       : std::max<size_t>(256, round_up((n + 15) / 16, 256));
    nb = std::min(nb, n);
    const size_t nblocks = (n + nb - 1) / nb;
    // device layouts: 16-byte aligned leading dimensions, each region 256-byte aligned
    const size_t lda_d = round_up(std::max<size_t>(a_rows, 1), 4);
    const size_t a_bytes = round_up(lda_d * a_cols * 4, 256);
    const size_t ldb_d = (op_b == kOpN) ? round_up(std::max<size_t>(k, 1), 8) : round_up(nb, 8);
    const size_t b_blk = round_up(((op_b == kOpN) ? ldb_d * nb : ldb_d * k) * 2, 256);
    const size_t ldc_d = (op_c == kOpN) ? round_up(m, 4) : round_up(nb, 4);
    const size_t c_blk = round_up(((op_c == kOpN) ? ldc_d * nb : ldc_d * m) * 4, 256);
    const size_t need = a_bytes + kSlots * (b_blk + c_blk);

    if (!h->host_in) {
        if (cudaStreamCreateWithFlags(&h->host_in, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&h->host_out, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            return SHGEMM_STATUS_CUDA_ERROR;
        }
        for (cudaEvent_t& e : h->host_ev)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                return SHGEMM_STATUS_CUDA_ERROR;
            }
    }
    if (need > h->host_stage_bytes) {  // grow the staging (the one allocation of this entry point)
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(h->stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
            return SHGEMM_STATUS_NOT_SUPPORTED;
        const int st = shgemm_b200_release_host_staging(h);
        if (st != SHGEMM_STATUS_OK) return st;
        if (cudaMalloc(&h->host_stage, need) != cudaSuccess) {
            cudaGetLastError();
            h->host_stage = nullptr;
            return SHGEMM_STATUS_ALLOC_FAILED;
        }
        h->host_stage_bytes = need;
    }
    char* base = static_cast<char*>(h->host_stage);
    float* a_d = reinterpret_cast<float*>(base);
    __half* b_s[kSlots];
    float* c_s[kSlots];
    for (int sl = 0; sl < kSlots; ++sl) {
        b_s[sl] = reinterpret_cast<__half*>(base + a_bytes + sl * b_blk);
        c_s[sl] = reinterpret_cast<float*>(base + a_bytes + kSlots * b_blk + sl * c_blk);
    }
    cudaEvent_t ev_start = h->host_ev[0], *ev_in = h->host_ev + 1, *ev_comp = ev_in + kSlots,
                *ev_out = ev_comp + kSlots;
    const __half* bh = static_cast<const __half*>(b);

    // the copy streams start after everything already queued on the handle's stream
    cudaEventRecord(ev_start, h->stream);
    cudaStreamWaitEvent(h->host_in, ev_start, 0);
    cudaStreamWaitEvent(h->host_out, ev_start, 0);
    if (k > 0)
        cudaMemcpy2DAsync(a_d, lda_d * 4, a, lda * 4, a_rows * 4, a_cols, cudaMemcpyHostToDevice, h->host_in);
    int level = SHGEMM_LEVEL_P0;
    for (size_t j = 0; j < nblocks; ++j) {
        const int slot = static_cast<int>(j % kSlots);
        const size_t c0 = j * nb, nbj = std::min(nb, n - c0);
        if (j >= kSlots) cudaStreamWaitEvent(h->host_in, ev_out[slot], 0);  // the slot's last block is home
        if (k > 0) {
            if (op_b == kOpN)
                cudaMemcpy2DAsync(b_s[slot], ldb_d * 2, bh + c0 * ldb, ldb * 2, k * 2, nbj, cudaMemcpyHostToDevice,
                                  h->host_in);
            else
                cudaMemcpy2DAsync(b_s[slot], ldb_d * 2, bh + c0, ldb * 2, nbj * 2, k, cudaMemcpyHostToDevice,
                                  h->host_in);
        }
        if (beta != 0.0f) {
            if (op_c == kOpN)
                cudaMemcpy2DAsync(c_s[slot], ldc_d * 4, c + c0 * ldc, ldc * 4, m * 4, nbj, cudaMemcpyHostToDevice,
                                  h->host_in);
            else
                cudaMemcpy2DAsync(c_s[slot], ldc_d * 4, c + c0, ldc * 4, nbj * 4, m, cudaMemcpyHostToDevice,
                                  h->host_in);
        }
        cudaEventRecord(ev_in[slot], h->host_in);
        cudaStreamWaitEvent(h->stream, ev_in[slot], 0);
        int lvl = SHGEMM_LEVEL_P0;
        const int st = shgemm_b200_shgemm(h, op_a, op_b, m, nbj, k, &alpha, a_d, lda_d, b_s[slot], ldb_d, &beta,
                                          c_s[slot], ldc_d, tc, op_c, &lvl);
        if (st != SHGEMM_STATUS_OK) {
            // join the copy streams before returning, so that nothing of this call is still
            // reading or writing the staging when the next call on the handle reuses it
            cudaEventRecord(ev_in[slot], h->host_in);
            cudaStreamWaitEvent(h->stream, ev_in[slot], 0);
            for (size_t sl = 0; sl < std::min<size_t>(j, kSlots); ++sl) cudaStreamWaitEvent(h->stream, ev_out[sl], 0);
            return st;
        }
        if (j == 0) level = lvl;
        cudaEventRecord(ev_comp[slot], h->stream);
        cudaStreamWaitEvent(h->host_out, ev_comp[slot], 0);
        if (op_c == kOpN)
            cudaMemcpy2DAsync(c + c0 * ldc, ldc * 4, c_s[slot], ldc_d * 4, m * 4, nbj, cudaMemcpyDeviceToHost,
                              h->host_out);
        else
            cudaMemcpy2DAsync(c + c0, ldc * 4, c_s[slot], ldc_d * 4, nbj * 4, m, cudaMemcpyDeviceToHost, h->host_out);
        cudaEventRecord(ev_out[slot], h->host_out);
    }
    for (size_t sl = 0; sl < std::min<size_t>(nblocks, kSlots); ++sl) cudaStreamWaitEvent(h->stream, ev_out[sl], 0);
    if (cudaGetLastError() != cudaSuccess) return SHGEMM_STATUS_CUDA_ERROR;
    if (level_out) *level_out = level;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_hsgemm_host(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k,
                            const float* alpha, const void* a, size_t lda, const float* b, size_t ldb,
                            const float* beta, float* c, size_t ldc, int tc, int op_c, int* level_out) {
    // the same transposition identity as shgemm_b200_hsgemm, on the host-buffer path
    auto inv = [](int op) { return op == kOpN ? kOpT : kOpN; };
    if ((op_a != kOpN && op_a != kOpT) || (op_b != kOpN && op_b != kOpT) || (op_c != kOpN && op_c != kOpT))
        return SHGEMM_STATUS_INVALID_VALUE;
    return shgemm_b200_shgemm_host(h, inv(op_b), inv(op_a), n, m, k, alpha, b, ldb, a, lda, beta, c, ldc, tc,
                                   inv(op_c), level_out);
}

static int eval_dgemm_impl(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k, const void* a,
                           size_t lda, const void* b, size_t ldb, double* c64, bool a_is_float) {
    if (!h || !a || !b || !c64 || m == 0 || n == 0) return SHGEMM_STATUS_INVALID_VALUE;
    if (m >= (1u << 31) || n >= (1u << 31) || k >= (1u << 31)) return SHGEMM_STATUS_NOT_SUPPORTED;
    DeviceGuard g(h->device);
    const dim3 grid(static_cast<unsigned>((m + 63) / 64), static_cast<unsigned>((n + 63) / 64));
    if (a_is_float)
        eval_dgemm_kernel<float, __half><<<grid, 256, 0, h->stream>>>(
            op_a, op_b, (int)m, (int)n, (int)k, static_cast<const float*>(a), lda, static_cast<const __half*>(b), ldb,
            c64);
    else
        eval_dgemm_kernel<__half, float><<<grid, 256, 0, h->stream>>>(
            op_a, op_b, (int)m, (int)n, (int)k, static_cast<const __half*>(a), lda, static_cast<const float*>(b), ldb,
            c64);
    return launch_status();
}

int shgemm_b200_eval_dgemm(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k, const float* a,
                           size_t lda, const void* b, size_t ldb, double* c64) {
    return eval_dgemm_impl(h, op_a, op_b, m, n, k, a, lda, b, ldb, c64, true);
}

int shgemm_b200_eval_dgemm_hs(shgemm_b200_handle_t h, int op_a, int op_b, size_t m, size_t n, size_t k,
                              const void* a, size_t lda, const float* b, size_t ldb, double* c64) {
    return eval_dgemm_impl(h, op_a, op_b, m, n, k, a, lda, b, ldb, c64, false);
}

int shgemm_b200_eval_error(shgemm_b200_handle_t h, size_t m, size_t n, const float* c, size_t ldc, int op_c,
                           const double* c64, double alpha, double beta, const float* c0, double* out) {
    if (!h || !c || !c64 || !out || (beta != 0.0 && !c0)) return SHGEMM_STATUS_INVALID_VALUE;
    DeviceGuard g(h->device);
    const int blocks = 1024;
    double* partial = nullptr;
    if (cudaMalloc(&partial, sizeof(double) * 4 * blocks) != cudaSuccess) return SHGEMM_STATUS_ALLOC_FAILED;
    eval_error_kernel<<<blocks, 256, 0, h->stream>>>(m, n, c, ldc, op_c, c64, alpha, beta, c0, partial);
    int st = launch_status();
    std::vector<double> hp(4 * blocks);
    if (st == SHGEMM_STATUS_OK) {
        if (cudaMemcpyAsync(hp.data(), partial, sizeof(double) * 4 * blocks, cudaMemcpyDeviceToHost, h->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess)
            st = SHGEMM_STATUS_CUDA_ERROR;
    }
    cudaFree(partial);
    if (st != SHGEMM_STATUS_OK) return st;
    double d = 0, r = 0, mx = 0, mm = 0;
    for (int i = 0; i < blocks; ++i) {
        d += hp[4 * i];
        r += hp[4 * i + 1];
        mx = std::max(mx, hp[4 * i + 2]);
        mm += hp[4 * i + 3];
    }
    out[0] = std::sqrt(d);
    out[1] = std::sqrt(r);
    out[2] = mx;
    out[3] = mm;
    return SHGEMM_STATUS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Grouped launches: many problems, one persistent kernel.
namespace {

int grouped_max_bn(int tc, bool b_wide) {
    return tc == kFP16 ? kGroupedMaxBnF16 : (b_wide ? kGroupedMaxBnTf32Wide : kGroupedMaxBnTf32);
}

// The default rule: the smallest power of two (>= 32) covering n, up to the kernel's tile.
int grouped_tile_n(int tc, bool b_wide, size_t n) {
    const int cap = grouped_max_bn(tc, b_wide);
    int bn = 32;
    while (bn < cap && static_cast<size_t>(bn) < n) bn *= 2;
    return bn;
}

bool grouped_bn_valid(int tc, bool b_wide, int bn) {
    return (bn == 32 || bn == 64 || bn == 128 || bn == 256) && bn <= grouped_max_bn(tc, b_wide);
}

// Tile N per n bucket for one staging call: the autotuner's entries (when the handle uses
// them), else the default rule; looked up once per bucket.
struct GroupedTileChoice {
    int bn_of[64] = {};
    shgemm_b200_handle_t h = nullptr;
    int tc = 0, op_a = 0;
    bool b_wide = false;
    int get(size_t n) {
        const int L = ilog2(n);
        if (L < 0 || L >= 64) return grouped_tile_n(tc, b_wide, n);
        if (!bn_of[L]) {
            int bn = 0;
            if (h->autotune_mode != 0) {
                std::lock_guard<std::mutex> lk(h->tune_mu);
                auto it = h->tuned.find(tune_key_grouped(tc, op_a, b_wide ? 1 : 0, L));
                if (it != h->tuned.end() && grouped_bn_valid(tc, b_wide, it->second.tile_n)) bn = it->second.tile_n;
            }
            bn_of[L] = bn ? bn : -1;
        }
        return bn_of[L] > 0 ? bn_of[L] : grouped_tile_n(tc, b_wide, n);
    }
};

// Writes the problem table and the unit list of a batch into table t's pinned host staging.
int grouped_stage(shgemm_b200_handle_t h, GroupedTable& t, bool b_wide, int op_a, int op_b, int tc, int op_c,
                  const shgemm_b200_problem* probs, int count) {
    if (!h || count < 0 || (count > 0 && !probs)) return SHGEMM_STATUS_INVALID_VALUE;
    if ((op_a != kOpN && op_a != kOpT) || op_b != kOpN || (op_c != kOpN && op_c != kOpT) ||
        (tc != kFP16 && tc != kTF32))
        return op_b == kOpT ? SHGEMM_STATUS_NOT_SUPPORTED : SHGEMM_STATUS_INVALID_VALUE;
    if (count > t.max_problems) return SHGEMM_STATUS_NOT_SUPPORTED;
    // The staging buffer may still be the source of a pending eager copy: wait for it
    // (not while capturing, where host waits are illegal; copies replayed from a
    // captured graph are the caller's to wait for).
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &cap) != cudaSuccess) cap = cudaStreamCaptureStatusNone;
    if (cap == cudaStreamCaptureStatusNone && cudaEventSynchronize(t.copied) != cudaSuccess) {
        cudaGetLastError();
        return SHGEMM_STATUS_CUDA_ERROR;
    }
    auto* host = static_cast<uint8_t*>(t.host);
    auto* gp = reinterpret_cast<GroupedProblem*>(host);
    auto* units = reinterpret_cast<int2*>(host + t.units_off);
    const int bk = tc == kFP16 ? 64 : 32;
    b_wide = b_wide && tc == kTF32;  // B given as FP32 (exact binary16 values)
    const size_t b_elem = b_wide ? 4 : 2;
    GroupedTileChoice tiles;
    tiles.h = h;
    tiles.tc = tc;
    tiles.op_a = op_a;
    tiles.b_wide = b_wide;
    struct Cost {
        long long cost;
        int2 unit;
    };
    std::vector<Cost> list;
    list.reserve(static_cast<size_t>(count) * 4);
    for (int i = 0; i < count; ++i) {
        const shgemm_b200_problem& q = probs[i];
        GroupedProblem& g = gp[i];
        std::memset(&g, 0, sizeof(g));
        if (q.m == 0 || q.n == 0) continue;
        const size_t a_rows = op_a == kOpN ? q.m : q.k, b_rows = q.k, c_rows = op_c == kOpN ? q.m : q.n;
        if (!q.c || q.ldc < c_rows) return SHGEMM_STATUS_INVALID_VALUE;
        if (q.m >= (1u << 31) || q.n >= (1u << 31) || q.k >= (1u << 31) || (q.m + 127) / 128 > 0xFFFF)
            return SHGEMM_STATUS_NOT_SUPPORTED;
        const int bn = tiles.get(q.n);
        const long long tiles_n = static_cast<long long>((q.n + bn - 1) / bn);
        if (tiles_n > 0x7FFF) return SHGEMM_STATUS_NOT_SUPPORTED;
        if (q.b_generated != 0 && q.b_generated != SHGEMM_OMEGA_RADEMACHER_BLOCKS) return SHGEMM_STATUS_INVALID_VALUE;
        const bool gen = q.b_generated != 0;
        if (gen && tc != kFP16) return SHGEMM_STATUS_NOT_SUPPORTED;  // generated B: binary16 compute only
        if (q.k > 0) {
            if (!q.a || (!gen && !q.b) || q.lda < std::max<size_t>(1, a_rows) ||
                (!gen && q.ldb < std::max<size_t>(1, b_rows)))
                return SHGEMM_STATUS_INVALID_VALUE;
            if ((reinterpret_cast<uintptr_t>(q.a) & 15) || (q.lda * 4) % 16 ||
                (!gen && ((reinterpret_cast<uintptr_t>(q.b) & 15) || (q.ldb * b_elem) % 16)))
                return SHGEMM_STATUS_NOT_SUPPORTED;  // grouped launches take TMA-addressable operands only
            bool ok = op_a == kOpT ? make_tmap(&g.tmap_a, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, q.a, q.k, q.m, q.lda * 4, 32,
                                               128, CU_TENSOR_MAP_SWIZZLE_128B)
                                   : make_tmap(&g.tmap_a, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, q.a, q.m, q.k, q.lda * 4,
                                               a_mmajor_box(tc, b_wide), bk, CU_TENSOR_MAP_SWIZZLE_NONE);
            if (gen) {
                g.b_gen = 1;  // the producer writes B's stages itself: no tensor map
                g.gen_seed = q.omega_seed;
            } else if (tc == kFP16)
                ok = ok && make_tmap(&g.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, q.b, q.k, q.n, q.ldb * 2, 64, bn,
                                     CU_TENSOR_MAP_SWIZZLE_128B);
            else if (b_wide)  // [bn][32] FP32 rows of 128 bytes: the TF32 tile layout itself
                ok = ok && make_tmap(&g.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, q.b, q.k, q.n, q.ldb * 4, 32, bn,
                                     CU_TENSOR_MAP_SWIZZLE_128B);
            else
                ok = ok && make_tmap(&g.tmap_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, q.b, q.k, q.n, q.ldb * 2, 32, bn,
                                     CU_TENSOR_MAP_SWIZZLE_64B);
            if (!ok) return SHGEMM_STATUS_NOT_SUPPORTED;
        }
        g.c = q.c;
        g.ldc = q.ldc;
        g.m = static_cast<int>(q.m);
        g.n = static_cast<int>(q.n);
        g.k = static_cast<int>(q.k);
        g.bn = bn;
        g.steps = static_cast<int>((q.k + bk - 1) / bk);
        g.alpha = q.alpha;
        g.beta = q.beta;
        const int tiles_m = static_cast<int>((q.m + 127) / 128);
        for (int tn = 0; tn < tiles_n; ++tn)
            for (int tm = 0; tm < tiles_m; ++tm)
                list.push_back({static_cast<long long>(g.steps + 1) * (1024 + bn), make_int2(i, tm | (tn << 16))});
    }
    if (list.size() > static_cast<size_t>(kGroupedMaxUnits)) return SHGEMM_STATUS_NOT_SUPPORTED;
    // Longest units first: the persistent CTAs claim them in this order as they free up,
    // which balances uneven k (greedy longest-processing-time order). A unit's time is its k-steps times a
    // step's time, which the A tile's stream sets for every tile N (measured per step on
    // single-class batches: 0.93 us at N = 32 and 64, 0.99 at 128, 1.1 at 256), hence
    // 1024 + bn per step.
    std::stable_sort(list.begin(), list.end(), [](const Cost& x, const Cost& y) { return x.cost > y.cost; });
    for (size_t u = 0; u < list.size(); ++u) units[u] = list[u].unit;
    *reinterpret_cast<int*>(host + t.count_off) = static_cast<int>(list.size());
    *reinterpret_cast<int*>(host + t.count_off + sizeof(int)) = 0;  // the launch's unit counter
    t.tc = tc;
    t.b32 = b_wide ? 1 : 0;
    t.op_a = op_a;
    t.op_b = op_b;
    t.op_c = op_c;
    t.units = static_cast<int>(list.size());
    return SHGEMM_STATUS_OK;
}

}  // namespace

static int grouped_run(shgemm_b200_handle_t h, GroupedTable& t, bool b_wide, int op_a, int op_b, int tc, int op_c,
                       const shgemm_b200_problem* probs, int count, DevScalars dev) {
    const int st = grouped_stage(h, t, b_wide, op_a, op_b, tc, op_c, probs, count);
    if (st != SHGEMM_STATUS_OK) return st;
    // problems, units, count and a zeroed unit counter in two copies from the pinned staging
    // (the tables are fixed-offset so a captured graph replays with whatever the staging holds,
    // and each replay starts its counter from zero)
    if (cudaMemcpyAsync(t.dev, t.host, sizeof(GroupedProblem) * static_cast<size_t>(count), cudaMemcpyHostToDevice,
                        h->stream) != cudaSuccess ||
        cudaMemcpyAsync(static_cast<uint8_t*>(t.dev) + t.units_off, static_cast<uint8_t*>(t.host) + t.units_off,
                        t.count_off + 2 * sizeof(int) - t.units_off, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        return SHGEMM_STATUS_CUDA_ERROR;
    t.copied_count = count;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(h->stream, &cap);
    if (cap == cudaStreamCaptureStatusNone) cudaEventRecord(t.copied, h->stream);
    GroupedParams P;
    std::memset(&P, 0, sizeof(P));
    P.problems = static_cast<const GroupedProblem*>(t.dev);
    P.units = reinterpret_cast<const int2*>(static_cast<uint8_t*>(t.dev) + t.units_off);
    P.num_units = reinterpret_cast<const int*>(static_cast<uint8_t*>(t.dev) + t.count_off);
    P.next_unit = reinterpret_cast<int*>(static_cast<uint8_t*>(t.dev) + t.count_off + sizeof(int));
    P.error_flag = h->error_word;
    P.wait_limit_ns = static_cast<uint64_t>(h->wait_limit_ms) * 1000000ull;
    P.op_c = op_c;
    P.alpha_dev = dev.alpha;
    P.beta_dev = dev.beta;
    const KernelEntry e = grouped_table(tc, op_a == kOpT, t.b32 == 1);
    void* args[] = {&P};
    // One CTA per SM whatever the batch: a captured launch stays valid for other batches.
    const cudaError_t err = cudaLaunchKernel(e.fn, dim3(h->num_sms), dim3(512), args, e.smem, h->stream);
    h->launches++;
    if (err != cudaSuccess) {
        cudaGetLastError();
        return SHGEMM_STATUS_LAUNCH_FAILED;
    }
    if (h->debug_mode)
        std::printf("[grouped] problems = %d, units = %d, compute_type = %s\n", count, t.units,
                    tc == kTF32 ? "TF32" : "FP16");
    return SHGEMM_STATUS_OK;
}

extern "C" {

int shgemm_b200_grouped_update(shgemm_b200_handle_t h, int op_a, int op_b, int compute_type, int op_c,
                               const shgemm_b200_problem* problems, int count) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    DeviceGuard g(h->device);
    GroupedTable& t = h->grouped;
    const int prev_tc = t.tc, prev_a = t.op_a, prev_c = t.op_c, prev_b = t.b32;
    const int st = grouped_stage(h, t, h->grouped_b_fp32 != 0, op_a, op_b, compute_type, op_c, problems, count);
    if (st != SHGEMM_STATUS_OK) return st;
    // A captured launch was built for one kernel variant and copies a fixed number of
    // problem slots: the batch must keep the variant and fit those slots.
    if (prev_tc >= 0 && (prev_tc != compute_type || prev_a != op_a || prev_c != op_c || prev_b != t.b32))
        return SHGEMM_STATUS_INVALID_VALUE;
    if (count > t.copied_count) return SHGEMM_STATUS_INVALID_VALUE;
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_shgemm_grouped(shgemm_b200_handle_t h, int op_a, int op_b, int compute_type, int op_c,
                               const shgemm_b200_problem* problems, int count) {
    if (!h) return SHGEMM_STATUS_INVALID_VALUE;
    DeviceGuard g(h->device);
    return grouped_run(h, h->grouped, h->grouped_b_fp32 != 0, op_a, op_b, compute_type, op_c, problems, count);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuning of grouped launches: tile N per n bucket.
extern "C" {

int shgemm_b200_autotune_grouped(shgemm_b200_handle_t h, int op_a, int op_b, int tc, int op_c,
                                 const shgemm_b200_problem* probs, int count, int* tuned_out) {
    if (tuned_out) *tuned_out = 0;
    if (!h || count < 1 || !probs) return SHGEMM_STATUS_INVALID_VALUE;
    DeviceGuard g(h->device);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return SHGEMM_STATUS_NOT_SUPPORTED;
    }
    const bool b_wide = tc == kTF32 && h->grouped_b_fp32 != 0;
    const int cap_bn = grouped_max_bn(tc, b_wide);
    std::vector<int> buckets;
    for (int i = 0; i < count; ++i)
        if (probs[i].m > 0 && probs[i].n > 0) buckets.push_back(ilog2(probs[i].n));
    std::sort(buckets.begin(), buckets.end());
    buckets.erase(std::unique(buckets.begin(), buckets.end()), buckets.end());
    if (buckets.empty()) return SHGEMM_STATUS_OK;

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        if (e0) cudaEventDestroy(e0);
        return SHGEMM_STATUS_CUDA_ERROR;
    }
    // the batch's median time with the current table (one untimed launch first)
    auto time_batch = [&](float* us) -> int {
        std::vector<float> t;
        for (int r = -1; r < 3; ++r) {
            cudaEventRecord(e0, h->stream);
            const int st = grouped_run(h, h->grouped, b_wide, op_a, op_b, tc, op_c, probs, count);
            cudaEventRecord(e1, h->stream);
            if (st != SHGEMM_STATUS_OK) return st;
            if (cudaEventSynchronize(e1) != cudaSuccess) return SHGEMM_STATUS_CUDA_ERROR;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (r >= 0) t.push_back(ms * 1000.0f);
        }
        int code = 0;
        if (shgemm_b200_check_error(h, &code) != SHGEMM_STATUS_OK) return SHGEMM_STATUS_TIMEOUT;
        std::sort(t.begin(), t.end());
        *us = t[t.size() / 2];
        return SHGEMM_STATUS_OK;
    };
    auto set_entry = [&](int L, int bn, float us) {
        std::lock_guard<std::mutex> lk(h->tune_mu);
        shgemm_b200_tuned_config c{};
        c.tile_n = bn;
        c.slices = 1;
        c.group_m = 1;
        c.time_us = us;
        c.k_chunk = 64;
        c.cta_group = 1;
        h->tuned[tune_key_grouped(tc, op_a, b_wide ? 1 : 0, L)] = c;
    };
    const int saved_mode = h->autotune_mode;
    if (h->autotune_mode == 0) h->autotune_mode = 1;  // the timing runs must see the trial entries
    // start from the current choice of every bucket (an entry, or the default rule)
    std::vector<int> choice(buckets.size());
    for (size_t b = 0; b < buckets.size(); ++b) {
        const int L = buckets[b];
        int bn = 0;
        {
            std::lock_guard<std::mutex> lk(h->tune_mu);
            auto it = h->tuned.find(tune_key_grouped(tc, op_a, b_wide ? 1 : 0, L));
            if (it != h->tuned.end() && grouped_bn_valid(tc, b_wide, it->second.tile_n)) bn = it->second.tile_n;
        }
        choice[b] = bn ? bn : grouped_tile_n(tc, b_wide, size_t(1) << L);
        set_entry(L, choice[b], 0.0f);
    }
    float best_us = 0;
    int st = time_batch(&best_us);
    for (size_t b = 0; b < buckets.size() && st == SHGEMM_STATUS_OK; ++b) {
        const int L = buckets[b];
        for (int bn = 32; bn <= cap_bn && st == SHGEMM_STATUS_OK; bn *= 2) {
            if (bn == choice[b]) continue;
            set_entry(L, bn, 0.0f);
            float us = 0;
            st = time_batch(&us);
            if (st == SHGEMM_STATUS_OK && us < best_us) {
                best_us = us;
                choice[b] = bn;
            }
        }
        set_entry(L, choice[b], best_us);
    }
    h->autotune_mode = saved_mode;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != SHGEMM_STATUS_OK) {
        cudaGetLastError();
        return st;
    }
    if (h->debug_mode) {
        for (size_t b = 0; b < buckets.size(); ++b)
            std::printf("[autotune grouped] %s n in [%zu, %zu): tile N = %d\n", tc == kTF32 ? "TF32" : "FP16",
                        size_t(1) << buckets[b], size_t(2) << buckets[b], choice[b]);
        std::printf("[autotune grouped] batch of %d problems: %.1f us\n", count, best_us);
    }
    if (tuned_out) *tuned_out = static_cast<int>(buckets.size());
    return SHGEMM_STATUS_OK;
}

int shgemm_b200_autotune_grouped_lookup(shgemm_b200_handle_t h, int op_a, int tc, int b_fp32, size_t n, int* tile_n) {
    if (!h || !tile_n || n == 0) return SHGEMM_STATUS_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(h->tune_mu);
    auto it = h->tuned.find(tune_key_grouped(tc, op_a, b_fp32 ? 1 : 0, ilog2(n)));
    if (it == h->tuned.end()) return SHGEMM_STATUS_INVALID_VALUE;
    *tile_n = it->second.tile_n;
    return SHGEMM_STATUS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free split-K entry point.
//
// For callers that cannot call cudaMalloc (for example code running inside an
// allocator callback, a custom memory manager that forbids other allocations, or
// a process whose device memory is fully reserved up front). It runs the same
// tile kernel and split-K reduction as shgemm_b200_shgemm, but keeps the split-K
// partials and the error word in file-scope device arrays instead of a handle's
// workspace, so it needs no handle and allocates nothing.
//
// The scratch array below is part of the library image: every GPU that loads
// the library holds it (16 MiB) until the process exits.
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchBytes / sizeof(float)];
static __device__ __align__(256) int g_noalloc_error;

struct NoAllocDevice {
    bool ready = false;
    int num_sms = 0;
    int fixed_level = SHGEMM_LEVEL_AUTO;  // MTK_SHGEMM_KERNEL_LEVEL, as shgemm_b200_create reads it
    unsigned debug_mode = 0;              // MTK_SHGEMM_DEBUG
    float* scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int* error_word = nullptr; // device address of g_noalloc_error on this device
};
constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mutex;

// One-time set-up on the current device: resolve the device addresses of the
// file-scope arrays (their names are host-side stand-ins in host code) and raise
// the dynamic shared memory limit of every tile kernel. Allocates nothing.
int noalloc_setup(int dev, NoAllocDevice*& out) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) return SHGEMM_STATUS_NOT_SUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        int major = 0, minor = 0, sms = 0;
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (major != 10 || minor != 0 || !encode_fn()) return SHGEMM_STATUS_NOT_SUPPORTED;
        void* sp = nullptr;
        void* ep = nullptr;
        if (cudaGetSymbolAddress(&sp, g_noalloc_scratch) != cudaSuccess ||
            cudaGetSymbolAddress(&ep, g_noalloc_error) != cudaSuccess) {
            cudaGetLastError();
            return SHGEMM_STATUS_CUDA_ERROR;
        }
        for (int tc = 0; tc < 2; ++tc)
            for (int bn : {64, 128, 256})
                for (int ak = 0; ak < 2; ++ak)
                    for (int bk = 0; bk < 2; ++bk) {
                        KernelEntry e = kernel_table(tc, bn, ak, bk);
                        if (!e.fn) continue;
                        if (cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem) !=
                            cudaSuccess) {
                            cudaGetLastError();
                            return SHGEMM_STATUS_NOT_SUPPORTED;
                        }
                    }
        for (int ak = 0; ak < 2; ++ak)
            for (int kc = 1; kc <= 2; ++kc)
                for (int sv = 0; sv < 2; ++sv) {
                    KernelEntry e = tm_kernel_table(ak != 0, kc, sv);
                    if (cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem) !=
                        cudaSuccess) {
                        cudaGetLastError();
                        return SHGEMM_STATUS_NOT_SUPPORTED;
                    }
                }
        for (int ak = 0; ak < 2; ++ak) {
            for (KernelEntry e : {tm2_kernel_table(ak != 0), tile_wide_table(ak != 0, 128), tile_wide_table(ak != 0, 256)}) {
                if (cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem) != cudaSuccess) {
                    cudaGetLastError();
                    return SHGEMM_STATUS_NOT_SUPPORTED;
                }
            }
        }
        d.num_sms = sms;
        const char* dbg = std::getenv("MTK_SHGEMM_DEBUG");
        d.debug_mode = (dbg && dbg[0] == '1') ? 1u : 0u;
        const char* lvl = std::getenv("MTK_SHGEMM_KERNEL_LEVEL");
        if (lvl && (lvl[0] == '0' || lvl[0] == '1') && lvl[1] == '\0') d.fixed_level = lvl[0] - '0';
        d.scratch = static_cast<float*>(sp);
        d.error_word = static_cast<int*>(ep);
        d.ready = true;
    }
    out = &d;
    return SHGEMM_STATUS_OK;
}
}  // namespace

extern "C" {

size_t shgemm_b200_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

int shgemm_b200_shgemm_noalloc(void* cuda_stream, int op_a, int op_b, size_t m, size_t n, size_t k,
                               const float* alpha, const float* a, size_t lda, const void* b, size_t ldb,
                               const float* beta, float* c, size_t ldc, int compute_type, int op_c, int* level_out) {
    if (!alpha || !beta) return SHGEMM_STATUS_INVALID_VALUE;
    // The split-K partials need at least two slices of m x n floats in the scratch.
    if (m * n > kNoAllocScratchBytes / sizeof(float) / 2) return SHGEMM_STATUS_SCRATCH_TOO_SMALL;
    if (k > 0 && ((reinterpret_cast<uintptr_t>(a) & 15) || (reinterpret_cast<uintptr_t>(b) & 15) || (lda * 4) % 16 ||
                  (ldb * 2) % 16))
        return SHGEMM_STATUS_NOT_SUPPORTED;  // the staging path would need more scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SHGEMM_STATUS_CUDA_ERROR;
    NoAllocDevice* d = nullptr;
    const int st = noalloc_setup(dev, d);
    if (st != SHGEMM_STATUS_OK) return st;
    // A stack-resident handle: the existing dispatch path, pointed at the static arrays.
    shgemm_b200_handle h;
    h.device = dev;
    h.num_sms = d->num_sms;
    h.stream = static_cast<cudaStream_t>(cuda_stream);
    h.workspace = d->scratch;
    h.workspace_bytes = kNoAllocScratchBytes;
    h.error_word = d->error_word;
    h.fixed_level = d->fixed_level;
    h.debug_mode = d->debug_mode;
    // The error word is sticky: a timeout stays recorded until shgemm_b200_noalloc_check_error
    // reads and clears it, so a later call cannot hide an earlier one's failure.
    return shgemm_b200_shgemm(&h, op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, compute_type, op_c,
                              level_out);
}

int shgemm_b200_noalloc_check_error(void* cuda_stream, int* device_code) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SHGEMM_STATUS_CUDA_ERROR;
    NoAllocDevice* d = nullptr;
    const int st = noalloc_setup(dev, d);
    if (st != SHGEMM_STATUS_OK) return st;
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(cuda_stream)) != cudaSuccess) return SHGEMM_STATUS_CUDA_ERROR;
    int code = 0;
    if (cudaMemcpy(&code, d->error_word, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SHGEMM_STATUS_CUDA_ERROR;
    if (code && cudaMemset(d->error_word, 0, sizeof(int)) != cudaSuccess) return SHGEMM_STATUS_CUDA_ERROR;
    if (device_code) *device_code = code;
    return code ? SHGEMM_STATUS_TIMEOUT : SHGEMM_STATUS_OK;
}

}  // extern "C"
