// CTA-pair form of the tensor-memory operand kernel (binary16 compute, B K-major): a pair of
// CTAs on two SMs (a cluster of 2) computes a 256 x 256 tile with tcgen05.mma.cta_group::2.
// Same products in the same order as shgemm_tm_kernel -- per k-step of 64, lo products into
// a fresh accumulator, folded with scale 2^-11 under the first hi product, then the other hi
// products, drained and added in round-to-nearest FP32 every k-step -- so C is bit-identical.
//
// What the pair changes: each CTA splits and keeps in its tensor memory only its own 128 rows
// of A, as before, but holds only half of the tile's B columns: every N-half of 128 columns is
// 64 columns in each CTA's shared memory, and a pair MMA (M = 256) reads both halves. Each SM
// therefore loads 16 KB of B per k-step instead of 32 KB, for the same MMA work.
//
// Roles in each CTA (640 threads): 8 split warps and 8 epilogue warps as in shgemm_tm_kernel,
// warp 16 the TMA producer (and tensor-memory allocator), warps 17-19 the three MMA issuers of
// the even CTA (idle in the odd one), one per accumulator buffer: half-step g (N-half g mod 2
// of k-step g / 2) goes to issuer g mod 3 and buffer g mod 3, so an issuer has three
// half-steps of tensor work (~1500 cycles) to do its barrier waits and commits in while the
// other two keep the tensor pipe fed. Barriers the even CTA's issuers wait on -- operand
// stages written (t_full), B stages landed (b_full), accumulator buffers drained (d_empty) --
// live in the even CTA and count both CTAs' arrivals; the odd CTA's split and epilogue warps
// arrive there through the cluster window (relaxed arrivals: they publish completed
// tensor-memory accesses only), and both CTAs' B loads complete on the even CTA's b_full.
// The issuers' commits arrive on the barriers of both CTAs (one commit per barrier, by address).
// Every wait is bounded, as in the other kernels.
#pragma once

#include "shgemm_kernel_tm.cuh"

namespace shgemm_b200 {

template <bool A_KMAJOR>
struct Tm2Cfg {
    static constexpr int BM = 128;       // rows per CTA
    static constexpr int PAIR_M = 256;   // rows per pair tile
    static constexpr int BN = 256;
    static constexpr int HALF_N = 128;
    static constexpr int B_COLS = 64;    // B columns per CTA per N-half
    static constexpr int BK = 64;
    static constexpr int A_STAGE = BM * BK * 4;          // raw FP32 tile (32 KB)
    static constexpr int B_STAGE = 2 * B_COLS * BK * 2;  // two N-halves x 64 columns x 64 k (16 KB)
    static constexpr int SA = 4, SB = 6, ST = 2, ND = 3;
    static constexpr int NUM_THREADS = 640;
    static constexpr int SPLIT_WARPS = 8, EPI_WARP0 = 8, CTRL_WARP0 = 16;
    static constexpr int LAUNCH_REGS = 96;
    static constexpr int SPLIT_REGS = 64, EPI_REGS = 152, CTRL_REGS = 48;
    static_assert(256 * SPLIT_REGS + 256 * EPI_REGS + 128 * CTRL_REGS <= NUM_THREADS * LAUNCH_REGS,
                  "register split exceeds the launch allocation");
    static constexpr int TMEM_COLS = 512;
    static constexpr int TMEM_OPERAND0 = ND * HALF_N;  // 384
    static_assert(TMEM_OPERAND0 + ST * 64 <= TMEM_COLS, "tensor memory budget");
    static constexpr int BAR_BYTES = 1024;
    static constexpr int SMEM_BYTES = SA * A_STAGE + SB * B_STAGE + BAR_BYTES + 1024;
    static_assert(SMEM_BYTES <= 232448, "dynamic shared memory limit");
};

template <bool A_KMAJOR>
__device__ __forceinline__ void tm2_kernel_body(const TileGemmParams& p) {
    using Cfg = Tm2Cfg<A_KMAJOR>;
    constexpr int SA = Cfg::SA, SB = Cfg::SB, ST = Cfg::ST;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_s = ptx::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
    uint8_t* a_base = smem;
    uint8_t* b_base = a_base + SA * Cfg::A_STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(b_base + SB * Cfg::B_STAGE);
    uint64_t* a_full = bars;              // TMA landed the raw A tile (this CTA)
    uint64_t* a_free = a_full + SA;       // every split warp of this CTA has read it
    uint64_t* b_full = a_free + SA;       // even CTA: both CTAs' B halves landed
    uint64_t* b_empty = b_full + SB;      // pair MMAs reading the stage completed
    uint64_t* t_full = b_empty + SB;      // even CTA: both CTAs' hi/lo operand stages written
    uint64_t* t_empty = t_full + ST;      // pair MMAs reading the operand stage completed
    uint64_t* d_full = t_empty + ST;      // accumulator buffer ready to drain
    uint64_t* d_empty = d_full + Cfg::ND; // even CTA: both CTAs drained the buffer
    uint64_t* drain_bar = d_empty + Cfg::ND;  // per issuer: its last MMAs completed
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + Cfg::ND);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t rank = ptx::cluster_ctarank();
    const bool leader = rank == 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < SA; ++s) {
            ptx::mbar_init(&a_full[s], 1);
            ptx::mbar_init(&a_free[s], Cfg::SPLIT_WARPS);
        }
        for (int s = 0; s < SB; ++s) {
            ptx::mbar_init(&b_full[s], 1);   // the even CTA's producer (expect_tx of both halves)
            ptx::mbar_init(&b_empty[s], 2);  // both issuers' commits
        }
        for (int t = 0; t < ST; ++t) {
            ptx::mbar_init(&t_full[t], 2 * Cfg::SPLIT_WARPS);  // split warps of both CTAs
            ptx::mbar_init(&t_empty[t], 2);
        }
        for (int b = 0; b < Cfg::ND; ++b) {
            ptx::mbar_init(&d_full[b], 1);
            ptx::mbar_init(&d_empty[b], 16);  // epilogue warps of both CTAs
        }
        for (int b = 0; b < Cfg::ND; ++b) ptx::mbar_init(&drain_bar[b], 1);
        *abort_flag = 0;
        ptx::fence_mbarrier_init();
    }
    if (warp == Cfg::CTRL_WARP0) {
        if (lane == 0) prefetch_params_maps(p);
        __syncwarp();
        ptx::tmem_alloc_pair(tmem_slot, Cfg::TMEM_COLS);
    }
    ptx::tc_fence_before();
    ptx::cluster_sync();  // both CTAs' barriers initialised and tensor memory allocated
    ptx::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const int num_units = unit_count(p);
    const int pair = blockIdx.x >> 1, num_pairs = gridDim.x >> 1;
    const uint64_t limit = p.wait_limit_ns;
    auto fail = [&](int code) {
        *abort_flag = 1;
        atomicCAS(p.error_flag, 0, code);
    };
    // the even CTA's copies of the pair barriers, in the cluster window
    auto lead = [&](const uint64_t* bar) { return ptx::mapa_shared(bar, 0); };
    auto peer = [&](const uint64_t* bar) { return ptx::mapa_shared(bar, rank ^ 1u); };
    auto self = [&](const uint64_t* bar) { return ptx::mapa_shared(bar, rank); };

    if (warp < Cfg::EPI_WARP0) {
        // ---------------------------------------------------------------- split warps
        ptx::setmaxnreg_dec<Cfg::SPLIT_REGS>();
        const int q = warp & 3;
        const int kh = warp >> 2;
        const int row = q * 32 + lane;
        const uint32_t lane_addr = static_cast<uint32_t>(q * 32) << 16;
        const int seg = kh * Cfg::BM + row;  // K-major raw tile: two 2-D boxes, one per k-half
        const int sw = seg & 7;
        const int fl = (lane >> 2) & 1;
        int as = 0, ts = 0;
        uint32_t aph = 0, tph = 0;
        for (int u = pair; u < num_units; u += num_pairs) {
            UnitDesc ud;
            get_unit<Cfg>(p, u, ud);
            for (int st = ud.s0; st < ud.s1; ++st) {
                if (!ptx::mbar_wait(&a_full[as], aph, abort_flag, limit) ||
                    !ptx::mbar_wait_cluster(&t_empty[ts], tph ^ 1u, abort_flag, limit)) {
                    fail(kErrSplitTimeout);
                    goto split_done;
                }
                ptx::tc_fence_after();
                {
                    const uint8_t* ast = a_base + as * Cfg::A_STAGE;
                    const uint32_t tcol = tmem_base + lane_addr + Cfg::TMEM_OPERAND0 + ts * 64;
                    uint32_t hw[16], lw[16];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        float v[16];
                        if constexpr (A_KMAJOR) {
                            const uint8_t* rp = ast + seg * 128;
                            float4 x[4];
#pragma unroll
                            for (int j = 0; j < 4; ++j)
                                x[j] = *reinterpret_cast<const float4*>(rp + ((((4 * c + j) ^ fl) ^ sw) << 4));
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const float4 y = fl ? x[j ^ 1] : x[j];
                                v[4 * j] = y.x;
                                v[4 * j + 1] = y.y;
                                v[4 * j + 2] = y.z;
                                v[4 * j + 3] = y.w;
                            }
                        } else {
                            const uint8_t* cp = ast + (32 * kh + 16 * c) * 512 + row * 4;
#pragma unroll
                            for (int j = 0; j < 16; ++j) v[j] = *reinterpret_cast<const float*>(cp + j * 512);
                        }
                        uint32_t h8[8], l8[8];
                        split16_f16(v, h8, l8);
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            hw[8 * c + e] = h8[e];
                            lw[8 * c + e] = l8[e];
                        }
                    }
                    ptx::tmem_st_32x32b_x16(tcol + 16 * kh, hw);
                    ptx::tmem_st_32x32b_x16(tcol + 32 + 16 * kh, lw);
                }
                ptx::tmem_st_wait();
                ptx::tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    ptx::mbar_arrive_cluster_relaxed(lead(&t_full[ts]));
                    ptx::mbar_arrive(&a_free[as]);
                }
                if (++as == SA) {
                    as = 0;
                    aph ^= 1u;
                }
                if (++ts == ST) {
                    ts = 0;
                    tph ^= 1u;
                }
            }
        }
    split_done:;
    } else if (warp < Cfg::CTRL_WARP0) {
        // ---------------------------------------------------------------- epilogue
        ptx::setmaxnreg_inc<Cfg::EPI_REGS>();
        const DevScalarValues dsc = load_dev_scalars(p);
        const int q = warp & 3;
        const int cq = (warp - Cfg::EPI_WARP0) >> 2;
        const int row_in_tile = static_cast<int>(rank) * Cfg::BM + q * 32 + lane;
        const uint32_t lane_addr = static_cast<uint32_t>(q * 32) << 16;
        uint32_t gc = 0;
        for (int u = pair; u < num_units; u += num_pairs) {
            int nsteps;
            {
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                nsteps = ud.s1 - ud.s0;
                const int row = ud.tm * Cfg::PAIR_M + row_in_tile;
                if ((dsc.on ? dsc.beta : ud.beta) != 0.0f && !ud.partial && row < ud.m) {
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        prefetch_row<64>(ud.c, ud.ldc, output_op(p), row, ud.tn * Cfg::BN + h * Cfg::HALF_N + cq * 64,
                                         ud.n);
                }
            }
            uint64_t acc2[64];
#pragma unroll
            for (int j = 0; j < 64; ++j) acc2[j] = 0ull;
            for (int i = 0; i < nsteps; ++i) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t g = 2 * gc + h, buf = g % Cfg::ND;
                    if (!ptx::mbar_wait_cluster(&d_full[buf], (g / Cfg::ND) & 1u, abort_flag, limit)) {
                        fail(kErrEpilogueTimeout);
                        goto epi_done;
                    }
                    ptx::tc_fence_after();
#pragma unroll
                    for (int j0 = 0; j0 < 64; j0 += 32) {
                        uint32_t r0[16], r1[16];
                        const uint32_t ta = tmem_base + lane_addr + buf * Cfg::HALF_N + cq * 64 + j0;
                        ptx::tmem_ld_32x32b_x16(ta, r0);
                        ptx::tmem_ld_32x32b_x16(ta + 16, r1);
                        ptx::tmem_ld_wait();
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            uint64_t& a0 = acc2[h * 32 + j0 / 2 + e];
                            uint64_t& a1 = acc2[h * 32 + j0 / 2 + 8 + e];
                            a0 = ptx::f2_add(a0, (static_cast<uint64_t>(r0[2 * e + 1]) << 32) | r0[2 * e]);
                            a1 = ptx::f2_add(a1, (static_cast<uint64_t>(r1[2 * e + 1]) << 32) | r1[2 * e]);
                        }
                    }
                    ptx::tc_fence_before();
                    __syncwarp();
                    if (lane == 0) ptx::mbar_arrive_cluster_relaxed(lead(&d_empty[buf]));
                }
                ++gc;
            }
            {
                auto acc = [&](int j) -> float { return (j & 1) ? ptx::f2_hi(acc2[j >> 1]) : ptx::f2_lo(acc2[j >> 1]); };
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                const int row = ud.tm * Cfg::PAIR_M + row_in_tile;
                if (row < ud.m) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int col0 = ud.tn * Cfg::BN + h * Cfg::HALF_N + cq * 64;
                        if (ud.partial) {
                            float* w = ud.partial + row;
#pragma unroll
                            for (int j = 0; j < 64; ++j) {
                                const int col = col0 + j;
                                if (col < ud.n) w[static_cast<size_t>(col) * ud.m] = acc(h * 64 + j);
                            }
                        } else {
                            store_row<64>(ud.c, ud.ldc, output_op(p), row, col0, ud.n, dsc.on ? dsc.alpha : ud.alpha,
                                          dsc.on ? dsc.beta : ud.beta, [&](int j) { return acc(h * 64 + j); });
                        }
                    }
                }
            }
        }
    epi_done:;
    } else {
        ptx::setmaxnreg_dec<Cfg::CTRL_REGS>();
        if (warp == Cfg::CTRL_WARP0 && lane == 0) {
            // ------------------------------------------------------------ TMA producer
            int as = 0, bs = 0;
            uint32_t aph = 0, bph = 0;
            uint32_t a_issued = 0, a_par = 0;
            uint32_t b_armed = 0, b_par = 0;  // even CTA: B phases armed with expect_tx, their parity
            const uint32_t b_full_lead0 = lead(&b_full[0]);
            for (int u = pair; u < num_units; u += num_pairs) {
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                const int row0 = ud.tm * Cfg::PAIR_M + static_cast<int>(rank) * Cfg::BM;
                for (int st = ud.s0; st < ud.s1; ++st) {
                    const int kc = st * Cfg::BK;
                    if (!ptx::mbar_wait(&a_free[as], aph ^ 1u, abort_flag, limit)) {
                        fail(kErrProducerTimeout);
                        goto producer_done;
                    }
                    {
                        uint8_t* a_dst = a_base + as * Cfg::A_STAGE;
                        ptx::mbar_arrive_expect_tx(&a_full[as], Cfg::A_STAGE);
                        if constexpr (A_KMAJOR) {
#pragma unroll
                            for (int sub = 0; sub < 2; ++sub)
                                ptx::tma_load_2d(a_dst + sub * (Cfg::BM * 128), ud.tmap_a, &a_full[as], kc + 32 * sub,
                                                 row0);
                        } else {
                            ptx::tma_load_2d(a_dst, ud.tmap_a, &a_full[as], row0, kc);
                        }
                        a_issued |= 1u << as;
                        a_par = (a_par & ~(1u << as)) | (aph << as);
                    }
                    if (++as == SA) {
                        as = 0;
                        aph ^= 1u;
                    }
                    if (!ptx::mbar_wait_cluster(&b_empty[bs], bph ^ 1u, abort_flag, limit)) {
                        fail(kErrProducerTimeout);
                        goto producer_done;
                    }
                    {
                        // this CTA's 64 columns of each N-half; both CTAs' loads complete on the
                        // even CTA's b_full, which expects the bytes of all four boxes
                        if (leader) {
                            ptx::mbar_arrive_expect_tx(&b_full[bs], 2 * Cfg::B_STAGE);
                            b_armed |= 1u << bs;
                            b_par = (b_par & ~(1u << bs)) | (bph << bs);
                        }
                        uint8_t* b_dst = b_base + bs * Cfg::B_STAGE;
                        const uint32_t bar = b_full_lead0 + bs * 8;
#pragma unroll
                        for (int h = 0; h < 2; ++h)
                            ptx::tma_load_2d_pair(b_dst + h * (Cfg::B_COLS * 128), ud.tmap_b, bar, kc,
                                                  ud.tn * Cfg::BN + h * Cfg::HALF_N + static_cast<int>(rank) * Cfg::B_COLS);
                    }
                    if (++bs == SB) {
                        bs = 0;
                        bph ^= 1u;
                    }
                }
            }
        producer_done:
            // Never leave with copies in flight: this CTA's A copies complete on its own
            // barriers; both CTAs' B copies complete on the even CTA's, so the even CTA's
            // producer waits for every B phase it armed, and the pair's final cluster barrier
            // keeps the odd CTA resident until then.
            if (leader) {
                for (int s = 0; s < SB; ++s) {
                    if (!(b_armed & (1u << s))) continue;
                    const uint32_t par = (b_par >> s) & 1u;
                    const uint64_t t0 = ptx::globaltimer_ns();
                    while (!ptx::mbar_try_wait_cluster(&b_full[s], par, 20000u)) {
                        if (ptx::globaltimer_ns() - t0 > limit) {
                            fail(kErrDrainTimeout);
                            break;
                        }
                    }
                }
            }
            for (int s = 0; s < SA; ++s) {
                if (!(a_issued & (1u << s))) continue;
                const uint32_t par = (a_par >> s) & 1u;
                const uint64_t t0 = ptx::globaltimer_ns();
                while (!ptx::mbar_try_wait(&a_full[s], par)) {
                    if (ptx::globaltimer_ns() - t0 > limit) {
                        fail(kErrDrainTimeout);
                        break;
                    }
                }
            }
        } else if (warp > Cfg::CTRL_WARP0 && lane == 0) {
            const int j = warp - (Cfg::CTRL_WARP0 + 1);  // issuer j: half-steps g = j mod 3, buffer j
            if (leader) {
                // -------------------------------------------------------- MMA issuers (even CTA)
                constexpr uint32_t idesc = ptx::make_idesc(false, false, false, Cfg::PAIR_M, Cfg::HALF_N);
                int ts = 0, bs = 0;
                uint32_t tph = 0, bph = 0, gc = 0;
                const uint32_t d = tmem_base + j * Cfg::HALF_N;
                for (int u = pair; u < num_units; u += num_pairs) {
                    UnitDesc ud;
                    get_unit<Cfg>(p, u, ud);
                    const int nsteps = ud.s1 - ud.s0;
                    for (int i = 0; i < nsteps; ++i) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const uint32_t g = 2 * gc + h;
                            if (g % Cfg::ND != static_cast<uint32_t>(j)) continue;
                            const bool ok = ptx::mbar_wait_cluster(&t_full[ts], tph, abort_flag, limit) &&
                                            ptx::mbar_wait_cluster(&b_full[bs], bph, abort_flag, limit) &&
                                            ptx::mbar_wait_cluster(&d_empty[j], ((g / Cfg::ND) & 1u) ^ 1u, abort_flag,
                                                                   limit);
                            if (!ok) {
                                fail(kErrMmaTimeout);
                                goto mma_done;
                            }
                            ptx::tc_fence_after();
                            {
                                const uint32_t a_hi = tmem_base + Cfg::TMEM_OPERAND0 + ts * 64;
                                // this CTA's 64 rows of N-half h in the stage; the peer's at the same offset
                                auto bd = [&](int kk) -> uint64_t {
                                    return ptx::make_smem_desc(ptx::smem_u32(b_base + bs * Cfg::B_STAGE) +
                                                                   h * (Cfg::B_COLS * 128) + kk * 32,
                                                               16, 1024, ptx::kLayoutSW128);
                                };
#pragma unroll
                                for (int kk = 0; kk < 4; ++kk)
                                    ptx::umma_f16_ts_pair(d, a_hi + 32 + kk * 8, bd(kk), idesc, kk > 0);
                                ptx::umma_f16_ts_scale11_pair(d, a_hi, bd(0), idesc);
#pragma unroll
                                for (int kk = 1; kk < 4; ++kk) ptx::umma_f16_ts_pair(d, a_hi + kk * 8, bd(kk), idesc, 1u);
                            }
                            ptx::umma_commit_pair(self(&d_full[j]));
                            ptx::umma_commit_pair(peer(&d_full[j]));
                            ptx::umma_commit_pair(self(&t_empty[ts]));
                            ptx::umma_commit_pair(peer(&t_empty[ts]));
                            ptx::umma_commit_pair(self(&b_empty[bs]));
                            ptx::umma_commit_pair(peer(&b_empty[bs]));
                        }
                        if (++ts == ST) {
                            ts = 0;
                            tph ^= 1u;
                        }
                        if (++bs == SB) {
                            bs = 0;
                            bph ^= 1u;
                        }
                        ++gc;
                    }
                }
            mma_done:
                // the pair's tensor memory is released only after every MMA of this issuer completed
                ptx::umma_commit_pair(self(&drain_bar[j]));
                ptx::umma_commit_pair(peer(&drain_bar[j]));
            }
            // both CTAs: wait for the even CTA's issuers' final commits before the release
            const uint64_t t0 = ptx::globaltimer_ns();
            while (!ptx::mbar_try_wait_cluster(&drain_bar[j], 0, 20000u)) {
                if (ptx::globaltimer_ns() - t0 > limit) {
                    fail(kErrDrainTimeout);
                    break;
                }
            }
        }
    }

    __syncwarp();
    ptx::tc_fence_before();
    ptx::cluster_sync();
    ptx::tc_fence_after();
    if (warp == Cfg::CTRL_WARP0) ptx::tmem_dealloc_pair(tmem_base, Cfg::TMEM_COLS);
}

// Launched in clusters of 2 (blocks 2i and 2i + 1 are pair i); the grid is a multiple of 2.
template <bool A_KMAJOR>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(640, 1)
    shgemm_tm2_kernel(const __grid_constant__ TileGemmParams p) {
    tm2_kernel_body<A_KMAJOR>(p);
}

}  // namespace shgemm_b200
