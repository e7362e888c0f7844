// Persistent, warp-specialised SHGEMM tile kernel for sm_100a.
//
// C = alpha * op(A) * op(B) + beta * C, A FP32, B binary16, column-major.
// The error-corrected method of the reference (src/wmmae_shgemm.hpp:11-125):
// the FP32 operand is split on the fly into hi = T(a) and lo = T(2^11 (a - hi))
// with T = binary16 or TF32; hi*B and lo*B are issued as two tcgen05 MMAs into
// separate TMEM accumulators. The hi accumulator is restarted every k-chunk and
// drained into registers, where chunks are summed with round-to-nearest FP32
// adds (the reference adds every k-fragment's hi product the same way, which
// avoids the tensor core's truncating accumulation); lo accumulates over the
// whole k range and is folded in once at the end as hi + lo * 2^-11
// (tcec store_matrix_sync, call site src/shgemm.cu:87-99). The epilogue applies
// alpha/beta like src/dmem_accessor.hpp:187-356 (C is not read when beta == 0)
// or, for split-K, writes the slice's partial to a workspace that a separate
// kernel reduces in fixed slice order.
//
// Warp roles (448 threads, one CTA per SM):
//   warp 0      TMA producer: raw FP32 A tile + binary16 B tile per k-step
//   warp 1      TMEM allocator + single-thread UMMA issuer
//   warps 2-5   split warpgroup: thread t owns tile row t; writes hi/lo (and,
//               for TF32, the widened B) as 128B-swizzled K-major UMMA tiles
//   warps 6-13  epilogue: TMEM lane quadrant (warp % 4) x column half
// Pipelines: load ring (TMA -> split/MMA), split ring (split -> MMA), two hi
// TMEM buffers (MMA <-> epilogue ping-pong per k-chunk), two lo TMEM buffers
// (alternating per tile). Every wait is bounded; on timeout the kernel records
// an error code, drains its own in-flight copies and MMAs, frees TMEM and exits.
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
    int tiles_m, tiles_n;
    int num_slices;       // split-K slices (1: the epilogue writes C)
    int steps_per_slice;  // k-steps per slice
    int num_units;        // tiles_m * tiles_n * num_slices
    int group_m;          // rasterisation group along m
    int chunk_steps;      // k-steps per hi-accumulator drain
};

template <int TC, int BN_, bool A_KMAJOR, bool B_KMAJOR>
struct TileCfg {
    static constexpr int BM = 128;
    static constexpr int BN = BN_;
    static constexpr bool kTf32 = (TC == kTF32);
    static constexpr int BK = kTf32 ? 32 : 64;  // one 128-byte swizzle row of the compute type
    static constexpr int UMMA_K = kTf32 ? 8 : 16;
    static constexpr int KSUB = BK / UMMA_K;  // MMAs per operand pair per k-step
    static constexpr int A_RAW = BM * BK * 4;
    static constexpr int B_RAW = BN * BK * 2;
    static constexpr int LOAD_STAGE = A_RAW + B_RAW;
    static constexpr int HI_BYTES = BM * 128;  // BM rows of 128 bytes (both modes)
    static constexpr int BT_BYTES = kTf32 ? BN * 128 : 0;
    static constexpr int SPLIT_STAGE = 2 * HI_BYTES + BT_BYTES;
    static constexpr int SPLIT_STAGES = 2;
    static constexpr int SMEM_BUDGET = 220 * 1024;
    static constexpr int LS_FIT = (SMEM_BUDGET - SPLIT_STAGES * SPLIT_STAGE) / LOAD_STAGE;
    static constexpr int LOAD_STAGES = LS_FIT > 6 ? 6 : LS_FIT;
    static_assert(LOAD_STAGES >= 2, "shared memory budget");
    static constexpr int NUM_THREADS = 448;
    static constexpr int TMEM_COLS = 512;
    static constexpr int HALF_N = BN / 2;  // columns per epilogue warp
    static constexpr int BAR_BYTES = 1024;
    static constexpr int SMEM_BYTES =
        LOAD_STAGES * LOAD_STAGE + SPLIT_STAGES * SPLIT_STAGE + BAR_BYTES + 1024 /*alignment slack*/;
    static_assert(BN == 64 || BN == 128, "tile N");
    static_assert(LOAD_STAGE % 1024 == 0 && SPLIT_STAGE % 1024 == 0, "1024B-aligned stages");
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

template <int TC, int BN, bool A_KMAJOR, bool B_KMAJOR>
__global__ void __launch_bounds__(448, 1) shgemm_tile_kernel(const __grid_constant__ TileGemmParams p) {
    using Cfg = TileCfg<TC, BN, A_KMAJOR, B_KMAJOR>;
    constexpr int LS = Cfg::LOAD_STAGES;
    constexpr int SS = Cfg::SPLIT_STAGES;
    constexpr bool kTf32 = Cfg::kTf32;

    extern __shared__ uint8_t smem_raw[];
    // 1024-byte alignment of the tile region (128B-swizzle atoms repeat every 1024 bytes).
    const uint32_t raw_s = ptx::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
    uint8_t* load_base = smem;
    uint8_t* split_base = load_base + LS * Cfg::LOAD_STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(split_base + SS * Cfg::SPLIT_STAGE);
    uint64_t* load_full = bars;
    uint64_t* load_empty = load_full + LS;
    uint64_t* split_full = load_empty + LS;
    uint64_t* split_empty = split_full + SS;
    uint64_t* hi_full = split_empty + SS;
    uint64_t* hi_empty = hi_full + 2;
    uint64_t* lo_full = hi_empty + 2;
    uint64_t* lo_empty = lo_full + 2;
    uint64_t* drain_bar = lo_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < LS; ++s) {
            ptx::mbar_init(&load_full[s], 1);
            ptx::mbar_init(&load_empty[s], kTf32 ? 4 : 1);
        }
        for (int s = 0; s < SS; ++s) {
            ptx::mbar_init(&split_full[s], 4);
            ptx::mbar_init(&split_empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            ptx::mbar_init(&hi_full[b], 1);
            ptx::mbar_init(&hi_empty[b], 8);
            ptx::mbar_init(&lo_full[b], 1);
            ptx::mbar_init(&lo_empty[b], 8);
        }
        ptx::mbar_init(drain_bar, 1);
        *abort_flag = 0;
        ptx::fence_mbarrier_init();
    }
    if (warp == 0 && lane == 0) {
        ptx::tma_prefetch_desc(&p.tmap_a);
        ptx::tma_prefetch_desc(&p.tmap_b);
    }
    if (warp == 1) {
        ptx::tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const int total_steps = (p.k + Cfg::BK - 1) / Cfg::BK;
    const uint64_t limit = p.wait_limit_ns;

    auto fail = [&](int code) {
        *abort_flag = 1;
        atomicCAS(p.error_flag, 0, code);
    };

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            int ls = 0;
            uint32_t lph = 0;
            uint32_t issued_mask = 0, issued_par = 0;  // per stage: a load is in flight / its phase parity
            for (int u = blockIdx.x; u < p.num_units; u += gridDim.x) {
                int tm, tn, slice, s0, s1;
                decode_unit(p, u, tm, tn, slice);
                step_range(p, slice, total_steps, s0, s1);
                for (int st = s0; st < s1; ++st) {
                    if (!ptx::mbar_wait(&load_empty[ls], lph ^ 1u, abort_flag, limit)) {
                        fail(kErrProducerTimeout);
                        goto producer_done;
                    }
                    uint8_t* a_dst = load_base + ls * Cfg::LOAD_STAGE;
                    uint8_t* b_dst = a_dst + Cfg::A_RAW;
                    ptx::mbar_arrive_expect_tx(&load_full[ls], Cfg::LOAD_STAGE);
                    const int kc = st * Cfg::BK;
                    if constexpr (A_KMAJOR) {
#pragma unroll
                        for (int sub = 0; sub < Cfg::BK / 32; ++sub)
                            ptx::tma_load_2d(a_dst + sub * (Cfg::BM * 128), &p.tmap_a, &load_full[ls], kc + 32 * sub,
                                             tm * Cfg::BM);
                    } else {
                        ptx::tma_load_2d(a_dst, &p.tmap_a, &load_full[ls], tm * Cfg::BM, kc);
                    }
                    if constexpr (B_KMAJOR) {
                        ptx::tma_load_2d(b_dst, &p.tmap_b, &load_full[ls], kc, tn * BN);
                    } else if constexpr (!kTf32) {
#pragma unroll
                        for (int sub = 0; sub < BN / 64; ++sub)
                            ptx::tma_load_2d(b_dst + sub * (Cfg::BK * 128), &p.tmap_b, &load_full[ls],
                                             tn * BN + 64 * sub, kc);
                    } else {
                        ptx::tma_load_2d(b_dst, &p.tmap_b, &load_full[ls], tn * BN, kc);
                    }
                    issued_mask |= 1u << ls;
                    issued_par = (issued_par & ~(1u << ls)) | (lph << ls);
                    if (++ls == LS) {
                        ls = 0;
                        lph ^= 1u;
                    }
                }
            }
        producer_done:
            // Never leave with bulk copies in flight into this CTA's shared memory.
            for (int s = 0; s < LS; ++s) {
                if (issued_mask & (1u << s)) {
                    const uint64_t t0 = ptx::globaltimer_ns();
                    while (!ptx::mbar_try_wait(&load_full[s], (issued_par >> s) & 1u)) {
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
            constexpr uint32_t idesc = ptx::make_idesc(kTf32, !kTf32 && !B_KMAJOR, Cfg::BM, BN);
            int ls = 0, ss = 0;
            uint32_t lph = 0, sph = 0, gc = 0, t_iter = 0;
            bool issued_any = false;
            for (int u = blockIdx.x; u < p.num_units; u += gridDim.x) {
                int tm, tn, slice, s0, s1;
                decode_unit(p, u, tm, tn, slice);
                step_range(p, slice, total_steps, s0, s1);
                const int nsteps = s1 - s0;
                const uint32_t lb = t_iter & 1u;
                if (!ptx::mbar_wait(&lo_empty[lb], ((t_iter >> 1) & 1u) ^ 1u, abort_flag, limit)) {
                    fail(kErrMmaTimeout);
                    goto mma_done;
                }
                ptx::tc_fence_after();
                {
                    const uint32_t d_lo = tmem_base + 256u + lb * 128u;
                    for (int i = 0; i < nsteps; ++i) {
                        const bool chunk_start = (i % p.chunk_steps) == 0;
                        const uint32_t hb = gc & 1u;
                        if (chunk_start) {
                            if (!ptx::mbar_wait(&hi_empty[hb], ((gc >> 1) & 1u) ^ 1u, abort_flag, limit)) {
                                fail(kErrMmaTimeout);
                                goto mma_done;
                            }
                        }
                        if constexpr (!kTf32) {
                            if (!ptx::mbar_wait(&load_full[ls], lph, abort_flag, limit)) {
                                fail(kErrMmaTimeout);
                                goto mma_done;
                            }
                        }
                        if (!ptx::mbar_wait(&split_full[ss], sph, abort_flag, limit)) {
                            fail(kErrMmaTimeout);
                            goto mma_done;
                        }
                        ptx::tc_fence_after();
                        const uint32_t d_hi = tmem_base + hb * 128u;
                        const uint32_t hi_s = ptx::smem_u32(split_base + ss * Cfg::SPLIT_STAGE);
                        const uint32_t lo_s = hi_s + Cfg::HI_BYTES;
                        uint32_t b_s;
                        if constexpr (kTf32) {
                            b_s = lo_s + Cfg::HI_BYTES;
                        } else {
                            b_s = ptx::smem_u32(load_base + ls * Cfg::LOAD_STAGE + Cfg::A_RAW);
                        }
#pragma unroll
                        for (int kk = 0; kk < Cfg::KSUB; ++kk) {
                            const uint64_t a_hi = ptx::make_smem_desc(hi_s + kk * 32, 16, 1024, ptx::kLayoutSW128);
                            const uint64_t a_lo = ptx::make_smem_desc(lo_s + kk * 32, 16, 1024, ptx::kLayoutSW128);
                            uint64_t bd;
                            if constexpr (kTf32 || B_KMAJOR) {
                                bd = ptx::make_smem_desc(b_s + kk * 32, 16, 1024, ptx::kLayoutSW128);
                            } else {
                                // MN-major binary16 B: 64-wide MN atoms Cfg::BK*128 bytes apart, 8-row
                                // k groups 1024 bytes apart; one UMMA_K=16 step = 16 rows of 128 bytes.
                                bd = ptx::make_smem_desc(b_s + kk * 2048, Cfg::BK * 128, 1024, ptx::kLayoutSW128);
                            }
                            const uint32_t acc_hi = (!chunk_start || kk > 0) ? 1u : 0u;
                            const uint32_t acc_lo = (i > 0 || kk > 0) ? 1u : 0u;
                            if constexpr (kTf32) {
                                ptx::umma_tf32_ss(d_hi, a_hi, bd, idesc, acc_hi);
                                ptx::umma_tf32_ss(d_lo, a_lo, bd, idesc, acc_lo);
                            } else {
                                ptx::umma_f16_ss(d_hi, a_hi, bd, idesc, acc_hi);
                                ptx::umma_f16_ss(d_lo, a_lo, bd, idesc, acc_lo);
                            }
                        }
                        issued_any = true;
                        ptx::umma_commit(&split_empty[ss]);
                        if constexpr (!kTf32) {
                            ptx::umma_commit(&load_empty[ls]);
                            if (++ls == LS) {
                                ls = 0;
                                lph ^= 1u;
                            }
                        }
                        if (++ss == SS) {
                            ss = 0;
                            sph ^= 1u;
                        }
                        const bool chunk_end = ((i + 1) % p.chunk_steps) == 0 || (i + 1) == nsteps;
                        if (chunk_end) {
                            ptx::umma_commit(&hi_full[hb]);
                            ++gc;
                        }
                    }
                }
                ptx::umma_commit(&lo_full[lb]);
                ++t_iter;
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
    } else if (warp < 6) {
        // ------------------------------------------------------------ split warpgroup
        const int t = (warp - 2) * 32 + lane;  // tile row (and B row in TF32 mode)
        int ls = 0, ss = 0;
        uint32_t lph = 0, sph = 0;
        for (int u = blockIdx.x; u < p.num_units; u += gridDim.x) {
            int tm, tn, slice, s0, s1;
            decode_unit(p, u, tm, tn, slice);
            step_range(p, slice, total_steps, s0, s1);
            for (int st = s0; st < s1; ++st) {
                if (!ptx::mbar_wait(&load_full[ls], lph, abort_flag, limit) ||
                    !ptx::mbar_wait(&split_empty[ss], sph ^ 1u, abort_flag, limit)) {
                    fail(kErrSplitTimeout);
                    goto split_done;
                }
                {
                    const uint8_t* a_raw = load_base + ls * Cfg::LOAD_STAGE;
                    uint8_t* hi_t = split_base + ss * Cfg::SPLIT_STAGE;
                    uint8_t* lo_t = hi_t + Cfg::HI_BYTES;
                    const int sw = t & 7;
                    if constexpr (!kTf32) {
#pragma unroll
                        for (int c = 0; c < 8; ++c) {  // 16-byte output chunk = 8 k values
                            float v[8];
                            if constexpr (A_KMAJOR) {
                                const uint8_t* row = a_raw + (c >> 2) * (Cfg::BM * 128) + t * 128;
                                const int j0 = (c & 3) * 2;
                                const float4 x0 = *reinterpret_cast<const float4*>(row + ((j0 ^ sw) << 4));
                                const float4 x1 = *reinterpret_cast<const float4*>(row + (((j0 + 1) ^ sw) << 4));
                                v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w;
                                v[4] = x1.x; v[5] = x1.y; v[6] = x1.z; v[7] = x1.w;
                            } else {
                                const float* af = reinterpret_cast<const float*>(a_raw);
#pragma unroll
                                for (int e = 0; e < 8; ++e) v[e] = af[(c * 8 + e) * Cfg::BM + t];
                            }
                            uint32_t h[4], l[4];
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                const __half2 hh = __floats2half2_rn(v[2 * e], v[2 * e + 1]);
                                const float2 hf = __half22float2(hh);
                                const __half2 ll =
                                    __floats2half2_rn(__fmul_rn(__fsub_rn(v[2 * e], hf.x), 2048.0f),
                                                      __fmul_rn(__fsub_rn(v[2 * e + 1], hf.y), 2048.0f));
                                h[e] = *reinterpret_cast<const uint32_t*>(&hh);
                                l[e] = *reinterpret_cast<const uint32_t*>(&ll);
                            }
                            const int off = t * 128 + ((c ^ sw) << 4);
                            *reinterpret_cast<uint4*>(hi_t + off) = make_uint4(h[0], h[1], h[2], h[3]);
                            *reinterpret_cast<uint4*>(lo_t + off) = make_uint4(l[0], l[1], l[2], l[3]);
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < 8; ++c) {  // 16-byte output chunk = 4 k values
                            float v[4];
                            if constexpr (A_KMAJOR) {
                                const float4 x = *reinterpret_cast<const float4*>(a_raw + t * 128 + ((c ^ sw) << 4));
                                v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
                            } else {
                                const float* af = reinterpret_cast<const float*>(a_raw);
#pragma unroll
                                for (int e = 0; e < 4; ++e) v[e] = af[(c * 4 + e) * Cfg::BM + t];
                            }
                            float hv[4], lv[4];
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                hv[e] = ptx::to_tf32_rna(v[e]);
                                lv[e] = ptx::to_tf32_rna(__fmul_rn(__fsub_rn(v[e], hv[e]), 2048.0f));
                            }
                            const int off = t * 128 + ((c ^ sw) << 4);
                            *reinterpret_cast<float4*>(hi_t + off) = make_float4(hv[0], hv[1], hv[2], hv[3]);
                            *reinterpret_cast<float4*>(lo_t + off) = make_float4(lv[0], lv[1], lv[2], lv[3]);
                        }
                        // Widen B (binary16 is exact in TF32): thread t writes K-major row n = t.
                        if (t < BN) {
                            const uint8_t* b_raw = a_raw + Cfg::A_RAW;
                            uint8_t* bt = lo_t + Cfg::HI_BYTES;
                            if constexpr (B_KMAJOR) {
                                // raw tile [BN][32] binary16, 64-byte rows, 64B swizzle
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    const uint4 hx = *reinterpret_cast<const uint4*>(
                                        b_raw + t * 64 + ((q ^ ((t >> 1) & 3)) << 4));
                                    const __half2* hp = reinterpret_cast<const __half2*>(&hx);
                                    const float2 f0 = __half22float2(hp[0]);
                                    const float2 f1 = __half22float2(hp[1]);
                                    const float2 f2 = __half22float2(hp[2]);
                                    const float2 f3 = __half22float2(hp[3]);
                                    *reinterpret_cast<float4*>(bt + t * 128 + (((2 * q) ^ sw) << 4)) =
                                        make_float4(f0.x, f0.y, f1.x, f1.y);
                                    *reinterpret_cast<float4*>(bt + t * 128 + (((2 * q + 1) ^ sw) << 4)) =
                                        make_float4(f2.x, f2.y, f3.x, f3.y);
                                }
                            } else {
                                // raw tile [32 k][BN] binary16, no swizzle
                                const __half* bh = reinterpret_cast<const __half*>(b_raw);
#pragma unroll
                                for (int c = 0; c < 8; ++c) {
                                    float4 f;
                                    f.x = __half2float(bh[(c * 4 + 0) * BN + t]);
                                    f.y = __half2float(bh[(c * 4 + 1) * BN + t]);
                                    f.z = __half2float(bh[(c * 4 + 2) * BN + t]);
                                    f.w = __half2float(bh[(c * 4 + 3) * BN + t]);
                                    *reinterpret_cast<float4*>(bt + t * 128 + ((c ^ sw) << 4)) = f;
                                }
                            }
                        }
                    }
                }
                // Make the generic-proxy stores visible to the tensor core (async proxy).
                ptx::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    ptx::mbar_arrive(&split_full[ss]);
                    if constexpr (kTf32) ptx::mbar_arrive(&load_empty[ls]);
                }
                if (++ls == LS) {
                    ls = 0;
                    lph ^= 1u;
                }
                if (++ss == SS) {
                    ss = 0;
                    sph ^= 1u;
                }
            }
        }
    split_done:;
    } else {
        // ------------------------------------------------------------ epilogue
        constexpr int HN = Cfg::HALF_N;
        const int q = warp & 3;             // TMEM lane quadrant this warp may access
        const int half = (warp - 6) >> 2;   // column half of the tile
        const int row_in_tile = q * 32 + lane;
        const uint32_t lane_addr = static_cast<uint32_t>(q * 32) << 16;
        uint32_t gc = 0, t_iter = 0;
        for (int u = blockIdx.x; u < p.num_units; u += gridDim.x) {
            int tm, tn, slice, s0, s1;
            decode_unit(p, u, tm, tn, slice);
            step_range(p, slice, total_steps, s0, s1);
            const int nsteps = s1 - s0;
            const int nchunks = (nsteps + p.chunk_steps - 1) / p.chunk_steps;
            float acc[HN];
#pragma unroll
            for (int j = 0; j < HN; ++j) acc[j] = 0.0f;
            for (int c = 0; c < nchunks; ++c) {
                const uint32_t hb = gc & 1u;
                if (!ptx::mbar_wait(&hi_full[hb], (gc >> 1) & 1u, abort_flag, limit)) {
                    fail(kErrEpilogueTimeout);
                    goto epi_done;
                }
                ptx::tc_fence_after();
#pragma unroll
                for (int j0 = 0; j0 < HN; j0 += 32) {
                    uint32_t r[32];
                    ptx::tmem_ld_32x32b_x32(tmem_base + lane_addr + hb * 128u + half * HN + j0, r);
                    ptx::tmem_ld_wait();
#pragma unroll
                    for (int e = 0; e < 32; ++e) acc[j0 + e] = __fadd_rn(acc[j0 + e], __uint_as_float(r[e]));
                }
                ptx::tc_fence_before();
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&hi_empty[hb]);
                ++gc;
            }
            {
                const uint32_t lb = t_iter & 1u;
                if (!ptx::mbar_wait(&lo_full[lb], (t_iter >> 1) & 1u, abort_flag, limit)) {
                    fail(kErrEpilogueTimeout);
                    goto epi_done;
                }
                ptx::tc_fence_after();
#pragma unroll
                for (int j0 = 0; j0 < HN; j0 += 32) {
                    uint32_t r[32];
                    ptx::tmem_ld_32x32b_x32(tmem_base + lane_addr + 256u + lb * 128u + half * HN + j0, r);
                    ptx::tmem_ld_wait();
#pragma unroll
                    for (int e = 0; e < 32; ++e)
                        acc[j0 + e] = __fadd_rn(acc[j0 + e], __fmul_rn(__uint_as_float(r[e]), 0x1p-11f));
                }
                ptx::tc_fence_before();
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&lo_empty[lb]);
            }
            {
                const int row = tm * Cfg::BM + row_in_tile;
                const int col0 = tn * BN + half * HN;
                if (row < p.m) {
                    if (p.num_slices > 1) {
                        float* w = p.workspace + static_cast<size_t>(slice) * p.n * p.m + row;
#pragma unroll
                        for (int j = 0; j < HN; ++j) {
                            const int col = col0 + j;
                            if (col < p.n) w[static_cast<size_t>(col) * p.m] = acc[j];
                        }
                    } else if (p.op_c == kOpN) {
                        float* cp = p.c + row;
#pragma unroll
                        for (int j = 0; j < HN; ++j) {
                            const int col = col0 + j;
                            if (col < p.n) {
                                float* dst = cp + static_cast<size_t>(col) * p.ldc;
                                *dst = (p.beta == 0.0f) ? __fmul_rn(acc[j], p.alpha)
                                                        : __fmaf_rn(acc[j], p.alpha, __fmul_rn(p.beta, *dst));
                            }
                        }
                    } else {
                        float* cp = p.c + static_cast<size_t>(row) * p.ldc;
#pragma unroll
                        for (int j = 0; j < HN; ++j) {
                            const int col = col0 + j;
                            if (col < p.n) {
                                float* dst = cp + col;
                                *dst = (p.beta == 0.0f) ? __fmul_rn(acc[j], p.alpha)
                                                        : __fmaf_rn(acc[j], p.alpha, __fmul_rn(p.beta, *dst));
                            }
                        }
                    }
                }
            }
            ++t_iter;
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

}  // namespace shgemm_b200
