// SHGEMM tile kernel with the split operand in tensor memory (binary16 compute,
// 128 x 256 tiles, B K-major). Same arithmetic as the shared-memory kernel in
// shgemm_kernel.cuh -- per k-step of 64: lo products into a fresh accumulator, folded
// with scale 2^-11 under the first hi product, then the other hi products; drained and
// added in round-to-nearest FP32 every k-step (the reference's per-fragment hi/lo
// accumulation, src/wmmae_shgemm.hpp:73-125, with one drain per 64 k) -- with a
// different data path:
//
//  * the split warps read the raw FP32 tile from shared memory and write hi and lo
//    straight into tensor memory (tcgen05.st); the MMAs take A from tensor memory, so
//    shared memory carries only the TMA writes and the B operand reads;
//  * each k-step runs as two N-halves of 128 columns; the halves go round three
//    128-column accumulator buffers, so a buffer's drain overlaps the next two halves'
//    MMAs (about 1024 cycles) instead of one;
//  * 20 warps: 8 split warps (two per TMEM lane quadrant, one per 32-k half of the
//    step), 8 epilogue warps (two per quadrant, one per 64-column quarter of each
//    half), a TMA producer warp and three MMA warps (one per accumulator buffer).
//
// Tensor memory (512 columns): accumulator buffer b at columns [128 b, 128 b + 128), b < 3,
// used by half h of k-step s when (2 s + h) % 3 == b; operand stage t at
// [384 + 64 t, 384 + 64 t + 64): hi in the first 32 columns, lo in the next 32 (row i in
// lane i, k-block kk of 16 in columns 8 kk .. 8 kk + 7).
#pragma once

#include "shgemm_kernel.cuh"

namespace shgemm_b200 {

// KC: k-steps of 64 per FP32 drain (1: every 64 k; 2: every 128 k).
// SV: operand ring variant (0: 4 raw FP32 A stages and 3 binary16 B stages; 1: 3 and 4).
template <bool A_KMAJOR, int KC = 1, int SV = 0>
struct TmCfg {
    static constexpr int BM = 128;
    static constexpr int BN = 256;
    static constexpr int HALF_N = 128;
    static constexpr int BK = 64;
    static constexpr int A_STAGE = BM * BK * 4;  // raw FP32 tile
    static constexpr int B_STAGE = BN * BK * 2;  // [256 n][64 k] binary16, 128-byte swizzle
    // raw A, B and tensor-memory operand stages; 128-column accumulator buffers: a chunk of
    // 2 k-steps holds 2 operand stages while its MMAs run, so it takes 4 stages and 2 buffers
    static constexpr int SA = SV == 0 ? 4 : 3, SB = SV == 0 ? 3 : 4, ST = KC == 1 ? 2 : 4;
    static_assert(SV == 0 || SV == 1, "stage variant");
    static constexpr int ND = KC == 1 ? 3 : 2;
    static_assert(KC == 1 || KC == 2, "k-chunk");
    static constexpr int NUM_THREADS = 640;
    static constexpr int SPLIT_WARPS = 8, EPI_WARP0 = 8, CTRL_WARP0 = 16;
    // setmaxnreg shares: 2 split + 2 epilogue + 1 control warpgroup, out of the
    // 640 x 96 registers the block is launched with.
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

// Splits 16 FP32 values into 8 words of binary16 hi pairs and 8 of lo pairs
// (value 2e in the low half of word e).
__device__ __forceinline__ void split16_f16(const float (&v)[16], uint32_t (&hw)[8], uint32_t (&lw)[8]) {
#pragma unroll
    for (int g = 0; g < 2; ++g) {
        const float w[8] = {v[8 * g], v[8 * g + 1], v[8 * g + 2], v[8 * g + 3],
                            v[8 * g + 4], v[8 * g + 5], v[8 * g + 6], v[8 * g + 7]};
        uint4 h, l;
        split8_f16(w, h, l);
        hw[4 * g] = h.x;
        hw[4 * g + 1] = h.y;
        hw[4 * g + 2] = h.z;
        hw[4 * g + 3] = h.w;
        lw[4 * g] = l.x;
        lw[4 * g + 1] = l.y;
        lw[4 * g + 2] = l.z;
        lw[4 * g + 3] = l.w;
    }
}

template <bool A_KMAJOR, int KC, int SV, class Params>
__device__ __forceinline__ void tm_kernel_body(const Params& p) {
    using Cfg = TmCfg<A_KMAJOR, KC, SV>;
    constexpr int SA = Cfg::SA, SB = Cfg::SB, ST = Cfg::ST;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_s = ptx::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (raw_s & 1023u)) & 1023u);
    uint8_t* a_base = smem;
    uint8_t* b_base = a_base + SA * Cfg::A_STAGE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(b_base + SB * Cfg::B_STAGE);
    uint64_t* a_full = bars;           // TMA landed the raw A tile
    uint64_t* a_free = a_full + SA;    // every split warp has read its share of it
    uint64_t* b_full = a_free + SA;
    uint64_t* b_empty = b_full + SB;   // MMAs reading the B stage completed
    uint64_t* t_full = b_empty + SB;   // hi/lo operand stage written to tensor memory
    uint64_t* t_empty = t_full + ST;   // MMAs reading the operand stage completed
    uint64_t* d_full = t_empty + ST;   // accumulator buffer ready to drain
    uint64_t* d_empty = d_full + Cfg::ND;  // accumulator buffer drained
    uint64_t* drain_bar = d_empty + Cfg::ND;  // one per MMA issuer
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + Cfg::ND);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < SA; ++s) {
            ptx::mbar_init(&a_full[s], 1);
            ptx::mbar_init(&a_free[s], Cfg::SPLIT_WARPS);
        }
        for (int s = 0; s < SB; ++s) {
            ptx::mbar_init(&b_full[s], 1);
            ptx::mbar_init(&b_empty[s], 2);  // the commits of both N-halves' MMAs
        }
        for (int t = 0; t < ST; ++t) {
            ptx::mbar_init(&t_full[t], Cfg::SPLIT_WARPS);
            ptx::mbar_init(&t_empty[t], 2);  // the commits of both N-halves' MMAs
        }
        for (int b = 0; b < Cfg::ND; ++b) {
            ptx::mbar_init(&d_full[b], 1);
            ptx::mbar_init(&d_empty[b], 8);
        }
        for (int b = 0; b < Cfg::ND; ++b) ptx::mbar_init(&drain_bar[b], 1);
        *abort_flag = 0;
        ptx::fence_mbarrier_init();
    }
    if (warp == Cfg::CTRL_WARP0) {
        if (lane == 0) prefetch_params_maps(p);
        __syncwarp();
        ptx::tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const int num_units = unit_count(p);
    const uint64_t limit = p.wait_limit_ns;
    auto fail = [&](int code) {
        *abort_flag = 1;
        atomicCAS(p.error_flag, 0, code);
    };

    if (warp < Cfg::EPI_WARP0) {
        // ---------------------------------------------------------------- split warps
        ptx::setmaxnreg_dec<Cfg::SPLIT_REGS>();
        const int q = warp & 3;    // TMEM lane quadrant: rows 32 q .. 32 q + 31
        const int kh = warp >> 2;  // k 32 kh .. 32 kh + 31 of each step
        const int row = q * 32 + lane;
        const uint32_t lane_addr = static_cast<uint32_t>(q * 32) << 16;
        // K-major raw tile: the 128-byte segment holding this row's k-half kh and its swizzle
        // phase. Lanes 4-7 of every 8 read the two chunks of each pair in swapped order: in the
        // paired layout rows r and r + 4 share a phase, and the swap keeps their loads on
        // different banks (in the per-half layout it only permutes already distinct chunks).
        const int seg = p.a_rows_paired ? 2 * row + kh : kh * Cfg::BM + row;
        const int sw = seg & 7;
        const int fl = (lane >> 2) & 1;
        int as = 0, ts = 0;
        uint32_t aph = 0, tph = 0;
        for (int u = blockIdx.x; u < num_units; u += gridDim.x) {
            UnitDesc ud;
            get_unit<Cfg>(p, u, ud);
            for (int st = ud.s0; st < ud.s1; ++st) {
                if (!ptx::mbar_wait(&a_full[as], aph, abort_flag, limit) ||
                    !ptx::mbar_wait(&t_empty[ts], tph ^ 1u, abort_flag, limit)) {
                    fail(kErrSplitTimeout);
                    goto split_done;
                }
                ptx::tc_fence_after();
                {
                    const uint8_t* ast = a_base + as * Cfg::A_STAGE;
                    const uint32_t tcol = tmem_base + lane_addr + Cfg::TMEM_OPERAND0 + ts * 64;
                    uint32_t hw[16], lw[16];  // both k-blocks of this warp: columns 16 kh .. 16 kh + 15
#pragma unroll
                    for (int c = 0; c < 2; ++c) {  // k-block kk = 2 kh + c of 16 k
                        float v[16];
                        if constexpr (A_KMAJOR) {
                            // 32 floats of the segment, 128-byte swizzle; chunks 4c .. 4c+3
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
                            // raw [64 k][128 m] floats, 512-byte rows: a warp reads 128 contiguous bytes per k
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
                    ptx::mbar_arrive(&t_full[ts]);
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
        const int cq = (warp - Cfg::EPI_WARP0) >> 2;  // 64-column quarter within each half
        const int row_in_tile = q * 32 + lane;
        const uint32_t lane_addr = static_cast<uint32_t>(q * 32) << 16;
        uint32_t gc = 0;
        for (int u = blockIdx.x; u < num_units; u += gridDim.x) {
            int nsteps;
            {
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                nsteps = ud.s1 - ud.s0;
                // beta != 0: C of this thread's row into L2 (kept there) while the tile's k-steps run
                const int row = ud.tm * Cfg::BM + row_in_tile;
                if ((dsc.on ? dsc.beta : ud.beta) != 0.0f && !ud.partial && row < ud.m) {
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        prefetch_row<64>(ud.c, ud.ldc, output_op(p), row, ud.tn * Cfg::BN + h * Cfg::HALF_N + cq * 64,
                                         ud.n);
                }
            }
            uint64_t acc2[64];  // [half][32 column pairs]
#pragma unroll
            for (int j = 0; j < 64; ++j) acc2[j] = 0ull;
            for (int i = 0; i < nsteps; i += KC) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    // half h of k-chunk gc is use (2 gc + h) / ND of buffer (2 gc + h) % ND
                    const uint32_t g = 2 * gc + h, buf = g % Cfg::ND;
                    if (!ptx::mbar_wait(&d_full[buf], (g / Cfg::ND) & 1u, abort_flag, limit)) {
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
                    if (lane == 0) ptx::mbar_arrive(&d_empty[buf]);
                }
                ++gc;
            }
            {
                auto acc = [&](int j) -> float { return (j & 1) ? ptx::f2_hi(acc2[j >> 1]) : ptx::f2_lo(acc2[j >> 1]); };
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                const int row = ud.tm * Cfg::BM + row_in_tile;
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
                                          dsc.on ? dsc.beta : ud.beta,
                                          [&](int j) { return acc(h * 64 + j); });
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
            const uint64_t pol_a = ptx::l2_policy_evict_first();
            int as = 0, bs = 0;
            uint32_t aph = 0, bph = 0;
            uint32_t a_issued = 0, a_par = 0, b_issued = 0, b_par = 0;  // per stage: load in flight, its parity
            for (int u = blockIdx.x; u < num_units; u += gridDim.x) {
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                if (ud.maps_in_global) {
                    ptx::fence_tensormap_acquire(ud.tmap_a);
                    ptx::fence_tensormap_acquire(ud.tmap_b);
                }
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
                            if (p.a_rows_paired) {
                                // one box of 128 rows x 256 bytes: whole row segments per request
                                if (p.a_read_once)
                                    ptx::tma_load_3d_hint(a_dst, ud.tmap_a, &a_full[as], 0, 2 * st, ud.tm * Cfg::BM,
                                                          pol_a);
                                else
                                    ptx::tma_load_3d(a_dst, ud.tmap_a, &a_full[as], 0, 2 * st, ud.tm * Cfg::BM);
                            } else {
#pragma unroll
                                for (int sub = 0; sub < 2; ++sub) {
                                    if (p.a_read_once)
                                        ptx::tma_load_2d_hint(a_dst + sub * (Cfg::BM * 128), ud.tmap_a, &a_full[as],
                                                              kc + 32 * sub, ud.tm * Cfg::BM, pol_a);
                                    else
                                        ptx::tma_load_2d(a_dst + sub * (Cfg::BM * 128), ud.tmap_a, &a_full[as],
                                                         kc + 32 * sub, ud.tm * Cfg::BM);
                                }
                            }
                        } else {
                            if (p.a_read_once)
                                ptx::tma_load_2d_hint(a_dst, ud.tmap_a, &a_full[as], ud.tm * Cfg::BM, kc, pol_a);
                            else
                                ptx::tma_load_2d(a_dst, ud.tmap_a, &a_full[as], ud.tm * Cfg::BM, kc);
                        }
                        a_issued |= 1u << as;
                        a_par = (a_par & ~(1u << as)) | (aph << as);
                    }
                    if (++as == SA) {
                        as = 0;
                        aph ^= 1u;
                    }
                    if (!ptx::mbar_wait(&b_empty[bs], bph ^ 1u, abort_flag, limit)) {
                        fail(kErrProducerTimeout);
                        goto producer_done;
                    }
                    ptx::mbar_arrive_expect_tx(&b_full[bs], Cfg::B_STAGE);
                    if (p.b_blocked)
                        ptx::tma_load_3d(b_base + bs * Cfg::B_STAGE, ud.tmap_b, &b_full[bs], 0, ud.tn * Cfg::BN, st);
                    else
                        ptx::tma_load_2d(b_base + bs * Cfg::B_STAGE, ud.tmap_b, &b_full[bs], kc, ud.tn * Cfg::BN);
                    b_issued |= 1u << bs;
                    b_par = (b_par & ~(1u << bs)) | (bph << bs);
                    if (++bs == SB) {
                        bs = 0;
                        bph ^= 1u;
                    }
                }
            }
        producer_done:
            // Never leave with bulk copies in flight into this CTA's shared memory.
            for (int s = 0; s < SA + SB; ++s) {
                const bool is_a = s < SA;
                const int sl = is_a ? s : s - SA;
                if (!((is_a ? a_issued : b_issued) & (1u << sl))) continue;
                uint64_t* bar = is_a ? &a_full[sl] : &b_full[sl];
                const uint32_t par = ((is_a ? a_par : b_par) >> sl) & 1u;
                const uint64_t t0 = ptx::globaltimer_ns();
                while (!ptx::mbar_try_wait(bar, par)) {
                    if (ptx::globaltimer_ns() - t0 > limit) {
                        fail(kErrDrainTimeout);
                        break;
                    }
                }
            }
        } else if (warp > Cfg::CTRL_WARP0 && warp <= Cfg::CTRL_WARP0 + Cfg::ND && lane == 0) {
            // ------------------------------------------------------------ MMA issuers
            // One thread per accumulator buffer, in different warps: half-chunk g (N-half
            // g mod 2 of k-chunk g / 2) goes to issuer g mod ND and buffer g mod ND.
            // tcgen05.mma issue stalls while the tensor pipe's queue is full, so a single
            // issuer's waits and commits would leave the pipe idle; with ND issuers each has
            // ND half-chunks of tensor work to do them in while the others keep it fed.
            const int j = warp - (Cfg::CTRL_WARP0 + 1);
            constexpr uint32_t idesc = ptx::make_idesc(false, false, false, Cfg::BM, Cfg::HALF_N);
            int ts = 0, bs = 0;
            uint32_t tph = 0, bph = 0, gc = 0;  // gc counts k-chunks
            bool issued_any = false;
            for (int u = blockIdx.x; u < num_units; u += gridDim.x) {
                UnitDesc ud;
                get_unit<Cfg>(p, u, ud);
                const int nsteps = ud.s1 - ud.s0;
                for (int i = 0; i < nsteps; i += KC) {
                    const int c = nsteps - i < KC ? nsteps - i : KC;  // k-steps in this chunk
                    int tsj[KC], bsj[KC];
                    uint32_t tpj[KC], bpj[KC];
#pragma unroll
                    for (int jj = 0; jj < KC; ++jj) {
                        tsj[jj] = ts;
                        bsj[jj] = bs;
                        tpj[jj] = tph;
                        bpj[jj] = bph;
                        if (jj < c) {
                            if (++ts == ST) {
                                ts = 0;
                                tph ^= 1u;
                            }
                            if (++bs == SB) {
                                bs = 0;
                                bph ^= 1u;
                            }
                        }
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint32_t g = 2 * gc + h;
                        if (g % Cfg::ND != static_cast<uint32_t>(j)) continue;
                        bool ok = true;
#pragma unroll
                        for (int jj = 0; jj < KC; ++jj) {
                            if (jj < c)
                                ok = ok && ptx::mbar_wait(&t_full[tsj[jj]], tpj[jj], abort_flag, limit) &&
                                     ptx::mbar_wait(&b_full[bsj[jj]], bpj[jj], abort_flag, limit);
                        }
                        ok = ok && ptx::mbar_wait(&d_empty[j], ((g / Cfg::ND) & 1u) ^ 1u, abort_flag, limit);
                        if (!ok) {
                            fail(kErrMmaTimeout);
                            goto mma_done;
                        }
                        ptx::tc_fence_after();
                        {
                            const uint32_t d = tmem_base + j * Cfg::HALF_N;
                            // rows 128 h .. 128 h + 127 of the [256 n][64 k] B stage of step jj of the chunk
                            auto bd = [&](int jj, int kk) -> uint64_t {
                                return ptx::make_smem_desc(ptx::smem_u32(b_base + bsj[jj] * Cfg::B_STAGE) +
                                                               h * (Cfg::HALF_N * 128) + kk * 32,
                                                           16, 1024, ptx::kLayoutSW128);
                            };
                            auto a_hi = [&](int jj) -> uint32_t {
                                return tmem_base + Cfg::TMEM_OPERAND0 + tsj[jj] * 64;
                            };
                            // the chunk's lo products into a fresh accumulator ...
#pragma unroll
                            for (int jj = 0; jj < KC; ++jj) {
                                if (jj < c) {
#pragma unroll
                                    for (int kk = 0; kk < 4; ++kk)
                                        ptx::umma_f16_ts(d, a_hi(jj) + 32 + kk * 8, bd(jj, kk), idesc,
                                                         (jj > 0 || kk > 0) ? 1u : 0u);
                                }
                            }
                            // ... scaled by 2^-11 under the first hi product, then the other hi products
                            ptx::umma_f16_ts_scale11(d, a_hi(0), bd(0, 0), idesc);
#pragma unroll
                            for (int jj = 0; jj < KC; ++jj) {
                                if (jj < c) {
#pragma unroll
                                    for (int kk = (jj == 0 ? 1 : 0); kk < 4; ++kk)
                                        ptx::umma_f16_ts(d, a_hi(jj) + kk * 8, bd(jj, kk), idesc, 1u);
                                }
                            }
                        }
                        issued_any = true;
                        ptx::umma_commit(&d_full[j]);
#pragma unroll
                        for (int jj = 0; jj < KC; ++jj) {
                            if (jj < c) {
                                ptx::umma_commit(&t_empty[tsj[jj]]);
                                ptx::umma_commit(&b_empty[bsj[jj]]);
                            }
                        }
                    }
                    ++gc;
                }
            }
        mma_done:
            // Wait for every MMA this thread issued before tensor memory is released.
            if (issued_any) {
                ptx::umma_commit(&drain_bar[j]);
                const uint64_t t0 = ptx::globaltimer_ns();
                while (!ptx::mbar_try_wait(&drain_bar[j], 0)) {
                    if (ptx::globaltimer_ns() - t0 > limit) {
                        fail(kErrDrainTimeout);
                        break;
                    }
                }
            }
        }
    }

    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == Cfg::CTRL_WARP0) ptx::tmem_dealloc(tmem_base, Cfg::TMEM_COLS);
}

template <bool A_KMAJOR, int KC, int SV>
__global__ void __launch_bounds__(640, 1) shgemm_tm_kernel(const __grid_constant__ TileGemmParams p) {
    tm_kernel_body<A_KMAJOR, KC, SV>(p);
}

}  // namespace shgemm_b200
