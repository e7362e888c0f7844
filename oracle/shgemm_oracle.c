/*
 * CPU restatement of the reference SHGEMM algorithm -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the oracle the CUDA path is checked against. Only tests/, the
 * smoke check and bench.py's CPU-baseline leg may load it; the product library
 * never links or calls it.
 *
 * Parity status: "parity unpinned" with respect to the reference's own outputs.
 * The reference keeps its numerics in the un-vendored wmma_extension "tcec"
 * module (call sites src/utils.hpp:15-17, src/wmmae_shgemm.hpp:17,24-31,83-84,
 * src/shgemm.cu:87-99); its submodules are empty, so it cannot be compiled, and
 * its tests hold no golden values (the test/ programs only print errors). What IS pinned:
 * the element conversions below are checked bit-for-bit against independent
 * implementations (numpy's IEEE binary16 cast and exact rational rounding) by
 * tests/test_oracle.py with the fixtures in tests/golden/, and both GEMM modes are
 * checked bit-for-bit against a restatement in exact rational arithmetic
 * (tests/test_oracle_exact.py) on inputs whose fragment sums FP64 holds exactly.
 *
 * Algorithm restated (reference file:line):
 *  - split of the FP32 operand, src/wmmae_shgemm.hpp:30-31:
 *        hi = T(v);  lo = T(2^11 * (v - float(hi)))
 *    T = IEEE binary16 round-to-nearest-even (overflow -> inf, gradual
 *    underflow), or TF32 round-to-nearest-ties-away (the behaviour of the
 *    documented cvt.rna.tf32.f32 conversion used by wmma's tf32 cast).
 *  - accumulation, src/wmmae_shgemm.hpp:86-124: for every k-fragment the hi
 *    product is formed from a zero accumulator and added to the running FP32
 *    sum with a round-to-nearest FP32 add; the lo product is accumulated over
 *    the whole k range.  `chunk` is the k-fragment length (16 for fp16 and 8
 *    for tf32 in the reference; the B200 kernel's k-chunk when modelling it).
 *    Products of split values are exact in FP64; a fragment sum is formed in
 *    FP64 and rounded once to FP32. The FP64 sum is exact while the products'
 *    bits span at most ~49 bits (a 2^27 spread of magnitudes); beyond that it
 *    carries a 2^-53 relative error, far below the FP32 rounding it feeds.
 *    That is oracle_shgemm, the idealised form. oracle_shgemm_tcmodel models
 *    the tensor core's accumulation as the reference meets it instead: each
 *    hi fragment sum truncated (rounded toward zero) to FP32 before its
 *    round-to-nearest add, and lo kept in an FP32 accumulator across all k
 *    that takes each fragment's sum with truncation. oracle_shgemm_b200model
 *    models this library's kernels (not the reference) down to the MMA
 *    instruction: per drain one accumulator goes through the lo fragments, then
 *    the hi fragments with the 2^-11 input scale, each MMA aligning its terms
 *    to the largest and keeping `align_bits` bits with truncation, and the drain
 *    is added with round to nearest.
 *  - fold, tcec store_matrix_sync at src/shgemm.cu:87-99: c = hi + lo * 2^-11.
 *  - epilogue, src/dmem_accessor.hpp:267-271 (beta != 0) and 199-214
 *    (beta == 0, C is not read): alpha * c + beta * C.
 *  - op_c == op_t stores C transposed (src/dmem_accessor.hpp:338-356).
 * Matrices are column-major with BLAS op semantics (include/shgemm/shgemm.hpp:105-119).
 */
#include <stdint.h>
#include <stddef.h>
#include <string.h>
#include <stdlib.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OP_N 0
#define OP_T 1
#define TC_FP16 0
#define TC_TF32 1

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* IEEE binary32 -> binary16, round to nearest even, with subnormals. */
uint16_t oracle_f32_to_f16_bits(float f) {
    const uint32_t x = f2u(f);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) {
        return (uint16_t)(sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u));
    }
    if (ax >= 0x477ff000u) { /* >= 65520 rounds to infinity */
        return (uint16_t)(sign | 0x7c00u);
    }
    if (ax >= 0x38800000u) { /* normal binary16 range, >= 2^-14 */
        const uint32_t e = (ax >> 23) - 127u + 15u;
        const uint32_t mant = ax & 0x7fffffu;
        uint32_t h = (e << 10) | (mant >> 13);
        const uint32_t rem = mant & 0x1fffu;
        if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1u;
        return (uint16_t)(sign | h);
    }
    if (ax < 0x00800000u) { /* binary32 subnormal or zero: far below 2^-25 */
        return (uint16_t)sign;
    }
    /* binary16 subnormal: quantum 2^-24 */
    const int E = (int)(ax >> 23) - 127;
    const uint32_t M = (ax & 0x7fffffu) | 0x800000u;
    const int shift = -(E + 1); /* value / 2^-24 = M * 2^(E+1) */
    if (shift > 24) return (uint16_t)sign;
    uint32_t q = M >> shift;
    const uint32_t rem = M & ((1u << shift) - 1u);
    const uint32_t half = 1u << (shift - 1);
    if (rem > half || (rem == half && (q & 1u))) q += 1u;
    return (uint16_t)(sign | q);
}

float oracle_f16_bits_to_f32(uint16_t h) {
    const uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    const uint32_t e = (h >> 10) & 0x1fu;
    const uint32_t m = h & 0x3ffu;
    if (e == 0x1fu) return u2f(sign | 0x7f800000u | (m << 13));
    if (e != 0) return u2f(sign | ((e - 15u + 127u) << 23) | (m << 13));
    /* subnormal: m * 2^-24, exact in binary32 */
    const float v = (float)m * 5.9604644775390625e-8f;
    return sign ? -v : v;
}

/* TF32: 8-bit exponent, 10-bit mantissa, round to nearest, ties away from zero. */
float oracle_round_tf32(float f) {
    uint32_t x = f2u(f);
    if ((x & 0x7f800000u) == 0x7f800000u) return f;
    x = (x + 0x1000u) & 0xffffe000u;
    return u2f(x);
}

float oracle_round_f16(float f) { return oracle_f16_bits_to_f32(oracle_f32_to_f16_bits(f)); }

static inline float round_tc(int tc, float v) {
    return tc == TC_FP16 ? oracle_round_f16(v) : oracle_round_tf32(v);
}

/* Split of one FP32 value (src/wmmae_shgemm.hpp:30-31), scale 2^11. */
void oracle_split(int tc, const float* v, size_t n, float* hi, float* lo) {
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
        const float h = round_tc(tc, v[i]);
        hi[i] = h;
        lo[i] = round_tc(tc, (v[i] - h) * 2048.0f);
    }
}

/* Element (i, kk) of op(A), A column-major m x k (op_n) or k x m (op_t). */
static inline size_t a_index(int op, size_t i, size_t kk, size_t ld) {
    return op == OP_N ? i + kk * ld : kk + i * ld;
}
/* Element (kk, j) of op(B). */
static inline size_t b_index(int op, size_t kk, size_t j, size_t ld) {
    return op == OP_N ? kk + j * ld : j + kk * ld;
}
static inline size_t c_index(int op, size_t i, size_t j, size_t ld) {
    return op == OP_N ? i + j * ld : j + i * ld;
}

/*
 * The GEMM loops below work on register blocks of RB rows of op(A) by CB columns of
 * op(B). Every element of C still takes its products in k order through the same
 * operations as a loop over one element (no reassociation; no contraction, the file is
 * compiled with -ffp-contract=off), so the blocking changes speed only: the RB rows of a
 * block sit in vector lanes. op(A) is packed in row blocks, element (i, kk) at
 * ((i / RB) * k + kk) * RB + i % RB, rows past m zero; op(B) as [n][k] rows (k
 * contiguous), columns past n zero. The block kernels are compiled for AVX-512, AVX2 and
 * baseline x86-64 and the loader picks one for the host (IEEE operations: the same
 * results on each). They are called from the OpenMP loops, not inlined into them, so that
 * each clone holds the whole k loop.
 */
#define RB 4
#define CB 4
#define HOT __attribute__((noinline, target_clones("arch=x86-64-v4", "arch=x86-64-v3", "default")))

static size_t round_up_sz(size_t x, size_t q) { return (x + q - 1) / q * q; }

static void pack_a_blocked(int op, size_t m, size_t k, const float* A, size_t lda, float* out) {
    const size_t mb = round_up_sz(m, RB) / RB;
#pragma omp parallel for schedule(static)
    for (size_t ib = 0; ib < mb; ib++)
        for (size_t kk = 0; kk < k; kk++)
            for (size_t r = 0; r < RB; r++) {
                const size_t i = ib * RB + r;
                out[(ib * k + kk) * RB + r] = i < m ? A[a_index(op, i, kk, lda)] : 0.0f;
            }
}

static void pack_b_f16(int op, size_t k, size_t n, size_t n_pad, const uint16_t* B, size_t ldb, float* out) {
#pragma omp parallel for schedule(static)
    for (size_t j = 0; j < n_pad; j++)
        for (size_t kk = 0; kk < k; kk++)
            out[j * k + kk] = j < n ? oracle_f16_bits_to_f32(B[b_index(op, kk, j, ldb)]) : 0.0f;
}

static inline float epilogue(float acc, float alpha, float beta, const float* c) {
    if (beta == 0.0f) return acc * alpha;
    return fmaf(acc, alpha, beta * (*c));
}

/* Operands of one GEMM in the blocked layouts (hi/lo only for the split forms). */
typedef struct {
    float *a, *ahi, *alo, *b;
    size_t mb, nb;
} packed_t;

static void packed_free(packed_t* p) {
    free(p->a);
    free(p->ahi);
    free(p->alo);
    free(p->b);
}

/* Packs op(A) and op(B); with tc >= 0 also splits op(A). Returns 0 on success. */
static int packed_make(packed_t* p, int tc, int op_a, int op_b, size_t m, size_t n, size_t k, const float* A,
                       size_t lda, const uint16_t* B, size_t ldb) {
    const size_t mp = round_up_sz(m, RB), np = round_up_sz(n, CB);
    memset(p, 0, sizeof(*p));
    p->mb = mp / RB;
    p->nb = np / CB;
    p->a = (float*)malloc(sizeof(float) * (mp * k + 1));
    p->b = (float*)malloc(sizeof(float) * (np * k + 1));
    if (tc >= 0) {
        p->ahi = (float*)malloc(sizeof(float) * (mp * k + 1));
        p->alo = (float*)malloc(sizeof(float) * (mp * k + 1));
    }
    if (!p->a || !p->b || (tc >= 0 && (!p->ahi || !p->alo))) {
        packed_free(p);
        return 1;
    }
    pack_a_blocked(op_a, m, k, A, lda, p->a);
    if (tc >= 0) oracle_split(tc, p->a, mp * k, p->ahi, p->alo);
    pack_b_f16(op_b, k, n, np, B, ldb, p->b);
    return 0;
}

/* One vector per block column: RB lanes of FP32 or FP64 (GCC vector extensions; on a
 * host without wide registers the compiler splits them). Lane arithmetic is the scalar
 * IEEE operation, conversions round to nearest like a (float) cast. */
typedef float vf_t __attribute__((vector_size(RB * sizeof(float))));
typedef double vd_t __attribute__((vector_size(RB * sizeof(double))));
typedef int32_t vi_t __attribute__((vector_size(RB * sizeof(int32_t))));

static inline __attribute__((always_inline)) vf_t load_vf(const float* p) {
    vf_t v;
    memcpy(&v, p, sizeof(v));
    return v;
}

/* Each lane of a double vector rounded toward zero to FP32 (the tensor core's truncating
 * accumulation is modelled as exact products and sums rounded this way): round to
 * nearest, and where that moved away from zero to a finite value, step one unit back
 * toward zero (the bit pattern minus one, for either sign). NaN lanes compare false and
 * stay; a lane that rounds to infinity stays infinite. */
static inline __attribute__((always_inline)) vf_t rz_vf(vd_t d) {
    const vf_t f = __builtin_convertvector(d, vf_t);
    const vd_t back = __builtin_convertvector(f, vd_t);
    const vd_t inf = (vd_t){0} + (double)INFINITY;
    const __typeof__(back > d) away = ((back > d) & (d >= 0)) | ((back < d) & (d < 0));
    const __typeof__(back > d) finite = (back < inf) & (back > -inf);
    const vi_t step = __builtin_convertvector(away & finite, vi_t); /* -1 where it moves */
    vi_t bits;
    memcpy(&bits, &f, sizeof(bits));
    bits += step;
    vf_t out;
    memcpy(&out, &bits, sizeof(out));
    return out;
}

/* Idealised accumulation of one block (oracle_shgemm): per k-fragment the hi sum in FP64,
 * rounded once and added with a round-to-nearest FP32 add; lo summed in FP64 over all k. */
HOT static void block_ideal(const float* restrict ah, const float* restrict al, const float* restrict b, size_t k,
                            size_t chunk, float out[CB][RB]) {
    vf_t acc[CB];
    vd_t lo[CB];
    for (int c = 0; c < CB; c++) {
        acc[c] = (vf_t){0};
        lo[c] = (vd_t){0};
    }
    for (size_t k0 = 0; k0 < k; k0 += chunk) {
        const size_t k1 = (k0 + chunk < k) ? k0 + chunk : k;
        vd_t s[CB];
        for (int c = 0; c < CB; c++) s[c] = (vd_t){0};
        for (size_t kk = k0; kk < k1; kk++) {
            const vd_t h = __builtin_convertvector(load_vf(ah + kk * RB), vd_t);
            const vd_t l = __builtin_convertvector(load_vf(al + kk * RB), vd_t);
            for (int c = 0; c < CB; c++) {
                const double bv = (double)b[c * k + kk];
                s[c] += h * bv;
                lo[c] += l * bv;
            }
        }
        for (int c = 0; c < CB; c++) acc[c] = acc[c] + __builtin_convertvector(s[c], vf_t);
    }
    for (int c = 0; c < CB; c++) {
        const vf_t r = acc[c] + __builtin_convertvector(lo[c], vf_t) * (1.0f / 2048.0f);
        memcpy(out[c], &r, sizeof(r));
    }
}

/* Tensor-core model of one block (oracle_shgemm_tcmodel): per k-fragment the hi sum
 * truncated to FP32 and added with a round-to-nearest FP32 add; the fragment's lo sum
 * added to an FP32 lo accumulator with truncation. */
HOT static void block_tcmodel(const float* restrict ah, const float* restrict al, const float* restrict b, size_t k,
                              size_t chunk, float out[CB][RB]) {
    vf_t acc[CB], lo[CB];
    for (int c = 0; c < CB; c++) acc[c] = lo[c] = (vf_t){0};
    for (size_t k0 = 0; k0 < k; k0 += chunk) {
        const size_t k1 = (k0 + chunk < k) ? k0 + chunk : k;
        vd_t s[CB], t[CB];
        for (int c = 0; c < CB; c++) s[c] = t[c] = (vd_t){0};
        for (size_t kk = k0; kk < k1; kk++) {
            const vd_t h = __builtin_convertvector(load_vf(ah + kk * RB), vd_t);
            const vd_t l = __builtin_convertvector(load_vf(al + kk * RB), vd_t);
            for (int c = 0; c < CB; c++) {
                const double bv = (double)b[c * k + kk];
                s[c] += h * bv;
                t[c] += l * bv;
            }
        }
        for (int c = 0; c < CB; c++) {
            acc[c] = acc[c] + rz_vf(s[c]);
            lo[c] = rz_vf(__builtin_convertvector(lo[c], vd_t) + t[c]);
        }
    }
    for (int c = 0; c < CB; c++) {
        const vf_t r = acc[c] + lo[c] * (1.0f / 2048.0f);
        memcpy(out[c], &r, sizeof(r));
    }
}

typedef int64_t vl_t __attribute__((vector_size(RB * sizeof(int64_t))));

static inline __attribute__((always_inline)) vl_t bits_vd(vd_t x) {
    vl_t b;
    memcpy(&b, &x, sizeof(b));
    return b;
}
static inline __attribute__((always_inline)) vd_t vd_bits(vl_t b) {
    vd_t x;
    memcpy(&x, &b, sizeof(x));
    return x;
}

/* Biased binary exponent of each lane (0 for zero). */
static inline __attribute__((always_inline)) vl_t expo(vd_t x) { return (bits_vd(x) >> 52) & 0x7ff; }

/* One MMA instruction of the model with alignment (align_bits = p > 0). Every term has a
 * nominal exponent: a product a*b the sum of its factors' exponents (the leading bit of the
 * product is one of the two positions above it), the accumulator c its own. E is the largest
 * nominal exponent; every term is truncated toward zero to a multiple of 2^(E - p + 1), the
 * truncated terms are summed exactly (fewer than 2^5 terms of at most p + 2 bits each fit
 * FP64's 53) and the sum is truncated to FP32. With p = 0 the exact sum is truncated instead.
 * Zero terms take no part in E; lanes with a non-finite term give the IEEE sum. pexp holds
 * the products' biased nominal exponents. */
static inline __attribute__((always_inline)) vf_t mma_model(vd_t c, const vd_t* prod, const vl_t* pexp, size_t np,
                                                            int p) {
    if (p <= 0) {
        vd_t s = c;
        for (size_t i = 0; i < np; i++) s += prod[i];
        return rz_vf(s);
    }
    const vl_t abs_mask = (vl_t){0} + 0x7fffffffffffffffLL;
    vl_t ex = expo(c);
    for (size_t i = 0; i < np; i++) {
        const vl_t gt = pexp[i] > ex;
        ex = (pexp[i] & gt) | (ex & ~gt);
    }
    vl_t eq = ex - (p - 1); /* biased exponent of the quantum */
    const vl_t low = eq < 1;
    eq = (eq & ~low) | (((vl_t){0} + 1) & low);
    const vd_t q = vd_bits(eq << 52);
    vd_t s = __builtin_convertvector(__builtin_convertvector(c / q, vl_t), vd_t) * q;
    vd_t plain = c;
    for (size_t i = 0; i < np; i++) {
        s += __builtin_convertvector(__builtin_convertvector(prod[i] / q, vl_t), vd_t) * q;
        plain += prod[i];
    }
    /* lanes with an infinite or NaN term take the IEEE sum (the integer path would not) */
    const vl_t nonfinite = (bits_vd(plain) & abs_mask) >= ((vl_t){0} + 0x7ff0000000000000LL);
    return rz_vf(vd_bits((bits_vd(plain) & nonfinite) | (bits_vd(s) & ~nonfinite)));
}

/* The B200 kernels' accumulation as modelled for one block (oracle_shgemm_b200model): per
 * drain of nfrag fragments of `frag` k, one FP32 accumulator D starts at zero, takes the
 * drain's lo fragments one MMA each (D = mma(D, fragment)), then the first hi fragment with
 * D scaled by 2^-11 (the MMA's scale-input-d) and the other hi fragments; the drain adds D to
 * the FP32 running sum with a round-to-nearest add. Each MMA is mma_model. */
HOT static void block_b200model(const float* restrict ah, const float* restrict al, const float* restrict b,
                                size_t k, size_t frag, size_t nfrag, int align_bits, float out[CB][RB]) {
    vf_t acc[CB];
    for (int c = 0; c < CB; c++) acc[c] = (vf_t){0};
    vd_t prod[CB][16];
    vl_t pexp[CB][16];
    for (size_t k0 = 0; k0 < k; k0 += frag * nfrag) {
        vf_t d[CB];
        for (int c = 0; c < CB; c++) d[c] = (vf_t){0};
        for (int part = 0; part < 2; part++) { /* 0: lo fragments, 1: hi fragments */
            const float* src = part == 0 ? al : ah;
            for (size_t f = 0; f < nfrag; f++) {
                const size_t kb = k0 + f * frag;
                if (kb >= k) break;
                const size_t ke = (kb + frag < k) ? kb + frag : k;
                for (size_t kk = kb; kk < ke; kk++) {
                    const vd_t v = __builtin_convertvector(load_vf(src + kk * RB), vd_t);
                    const vl_t ev = expo(v), v_zero = ev == 0;
                    for (int c = 0; c < CB; c++) {
                        const vd_t bv = (vd_t){0} + (double)b[c * k + kk];
                        const vl_t eb = expo(bv), zero = v_zero | (eb == 0);
                        prod[c][kk - kb] = v * bv;
                        pexp[c][kk - kb] = (ev + eb - 1023) & ~zero; /* a*b's nominal exponent, biased */
                    }
                }
                for (int c = 0; c < CB; c++) {
                    vd_t dd = __builtin_convertvector(d[c], vd_t);
                    if (part == 1 && f == 0) dd *= 1.0 / 2048.0;
                    d[c] = mma_model(dd, prod[c], pexp[c], ke - kb, align_bits);
                }
            }
        }
        for (int c = 0; c < CB; c++) acc[c] = acc[c] + d[c];
    }
    for (int c = 0; c < CB; c++) memcpy(out[c], &acc[c], sizeof(acc[c]));
}

/* The reference's accumulation (block_tcmodel's structure) with each MMA as mma_model:
 * per k-fragment of `frag` (at most 16) k the hi products go through one MMA from a zero
 * accumulator and are added to the FP32 running sum with round to nearest, and the lo
 * products through one MMA on the lo accumulator that runs over all k; then the fold. With
 * align_bits > 0 this is the reference's algorithm on a tensor core that aligns like the
 * calibrated B200 model. */
HOT static void block_tcmodel_aligned(const float* restrict ah, const float* restrict al, const float* restrict b,
                                      size_t k, size_t frag, int align_bits, float out[CB][RB]) {
    vf_t acc[CB], lo[CB];
    for (int c = 0; c < CB; c++) acc[c] = lo[c] = (vf_t){0};
    vd_t ph[CB][16], pl[CB][16];
    vl_t eh[CB][16], el[CB][16];
    for (size_t k0 = 0; k0 < k; k0 += frag) {
        const size_t k1 = (k0 + frag < k) ? k0 + frag : k;
        for (size_t kk = k0; kk < k1; kk++) {
            const vd_t h = __builtin_convertvector(load_vf(ah + kk * RB), vd_t);
            const vd_t l = __builtin_convertvector(load_vf(al + kk * RB), vd_t);
            const vl_t exh = expo(h), exl = expo(l);
            for (int c = 0; c < CB; c++) {
                const vd_t bv = (vd_t){0} + (double)b[c * k + kk];
                const vl_t eb = expo(bv);
                ph[c][kk - k0] = h * bv;
                pl[c][kk - k0] = l * bv;
                eh[c][kk - k0] = (exh + eb - 1023) & ~((exh == 0) | (eb == 0));
                el[c][kk - k0] = (exl + eb - 1023) & ~((exl == 0) | (eb == 0));
            }
        }
        for (int c = 0; c < CB; c++) {
            acc[c] = acc[c] + mma_model((vd_t){0}, ph[c], eh[c], k1 - k0, align_bits);
            lo[c] = mma_model(__builtin_convertvector(lo[c], vd_t), pl[c], el[c], k1 - k0, align_bits);
        }
    }
    for (int c = 0; c < CB; c++) {
        const vf_t r = acc[c] + lo[c] * (1.0f / 2048.0f);
        memcpy(out[c], &r, sizeof(r));
    }
}

static int shgemm_blocked(int tcmodel, int tc, int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                          const float* A, size_t lda, const uint16_t* B, size_t ldb, float beta, float* C,
                          size_t ldc, int op_c, size_t chunk, int align_bits) {
    if (chunk == 0) chunk = (tc == TC_FP16) ? (tcmodel == 2 ? 64 : 16) : (tcmodel == 2 ? 32 : 8);
    if (tcmodel == 2 && ((chunk % ((tc == TC_FP16) ? 16 : 8)) != 0 || align_bits < 0 || align_bits > 40)) return 2;
    if (tcmodel == 1 && (align_bits < 0 || align_bits > 40 || (align_bits > 0 && chunk > 16))) return 2;
    packed_t p;
    if (packed_make(&p, tc, op_a, op_b, m, n, k, A, lda, B, ldb)) return 1;
    /* TF32 compute: the binary16 operand is exact in TF32 (src/utils.hpp:15-17). */
#pragma omp parallel for collapse(2) schedule(static)
    for (size_t jb = 0; jb < p.nb; jb++) {
        for (size_t ib = 0; ib < p.mb; ib++) {
            float out[CB][RB];
            const float* ah = p.ahi + ib * k * RB;
            const float* al = p.alo + ib * k * RB;
            const float* bj = p.b + jb * CB * k;
            if (tcmodel == 2)
                block_b200model(ah, al, bj, k, (tc == TC_FP16) ? 16 : 8, chunk / ((tc == TC_FP16) ? 16 : 8),
                                align_bits, out);
            else if (tcmodel && align_bits > 0)
                block_tcmodel_aligned(ah, al, bj, k, chunk, align_bits, out);
            else if (tcmodel)
                block_tcmodel(ah, al, bj, k, chunk, out);
            else
                block_ideal(ah, al, bj, k, chunk, out);
            for (size_t c = 0; c < CB && jb * CB + c < n; c++)
                for (size_t r = 0; r < RB && ib * RB + r < m; r++) {
                    float* cp = C + c_index(op_c, ib * RB + r, jb * CB + c, ldc);
                    *cp = epilogue(out[c][r], alpha, beta, cp);
                }
        }
    }
    packed_free(&p);
    return 0;
}

/*
 * Restated reference SHGEMM: C = alpha * op(A) * op(B) + beta * C with A FP32
 * and B binary16 (bits). chunk = hi-fragment length. Returns 0 on success.
 * Per element: for each k-fragment, s = sum of hi * b in FP64, acc = acc + (float)s;
 * lo = sum over all k of lo * b in FP64; c = acc + (float)lo * 2^-11; then the epilogue.
 */
int oracle_shgemm(int tc, int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                  const float* A, size_t lda, const uint16_t* B, size_t ldb, float beta,
                  float* C, size_t ldc, int op_c, size_t chunk) {
    return shgemm_blocked(0, tc, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, op_c, chunk, 0);
}

/*
 * Restated reference SHGEMM with the tensor core's accumulation modelled as the
 * reference meets it (src/wmmae_shgemm.hpp:86-124), rather than exactly:
 *  - hi: per k-fragment of `chunk` (16 for fp16, 8 for tf32: one mma_sync), the
 *    product is formed on the tensor core from a zero accumulator -- modelled as
 *    the exact fragment sum rounded toward zero to FP32 -- and added to the FP32
 *    running sum with a round-to-nearest add (src/wmmae_shgemm.hpp:89-97,106-114);
 *  - lo: accumulated on the tensor core across ALL k, D_lo = A_lo B + D_lo
 *    (src/wmmae_shgemm.hpp:116-121) -- modelled as an FP32 accumulator to which
 *    each fragment's exact sum is added with rounding toward zero;
 *  - fold c = hi + lo * 2^-11 (tcec store, call site src/shgemm.cu:87-99), then the
 *    same epilogue as oracle_shgemm.
 * Products of split values with binary16 values are exact in FP64. align_bits = 0 truncates
 * exact sums as above; align_bits > 0 (chunk at most 16) makes each fragment one MMA as
 * oracle_shgemm_b200model models them (alignment to the largest nominal exponent).
 */
int oracle_shgemm_tcmodel(int tc, int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                          const float* A, size_t lda, const uint16_t* B, size_t ldb, float beta,
                          float* C, size_t ldc, int op_c, size_t chunk, int align_bits) {
    return shgemm_blocked(1, tc, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, op_c, chunk,
                          align_bits);
}

/*
 * SHGEMM with the accumulation of this library's B200 kernels modelled (not the reference's):
 * per drain of `chunk` k (0: 64 for binary16, 32 for TF32; a multiple of the 16- or 8-k
 * MMA fragment), the lo fragments and then the hi fragments go through one FP32 accumulator,
 * one modelled MMA instruction per fragment (mma_model: alignment to the largest term with
 * `align_bits` bits kept and truncation, or with align_bits = 0 truncation of the exact sum),
 * the first hi fragment scaling the accumulator by 2^-11, and the drain is added to the
 * running sum with a round-to-nearest add; then the epilogue. Returns 2 when chunk is not a
 * multiple of the fragment or align_bits is outside 0..40.
 */
int oracle_shgemm_b200model(int tc, int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                            const float* A, size_t lda, const uint16_t* B, size_t ldb, float beta,
                            float* C, size_t ldc, int op_c, size_t chunk, int align_bits) {
    return shgemm_blocked(2, tc, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, op_c, chunk,
                          align_bits);
}

/* FP64 dot products of one block, each element over four interleaved partial sums
 * (k = 0, 4, 8, .. / 1, 5, .. / ..; the tail into the first), combined as
 * (s0 + s1) + (s2 + s3). Two of the block's columns per pass. */
HOT static void block_dgemm(const float* restrict a, const float* restrict b, size_t k, double out[CB][RB]) {
    for (int c0 = 0; c0 < CB; c0 += 2) {
        vd_t s[4][2];
        for (int q = 0; q < 4; q++) s[q][0] = s[q][1] = (vd_t){0};
        size_t kk = 0;
        for (; kk + 4 <= k; kk += 4)
            for (int q = 0; q < 4; q++) {
                const vd_t av = __builtin_convertvector(load_vf(a + (kk + q) * RB), vd_t);
                for (int c = 0; c < 2; c++) s[q][c] += av * (double)b[(c0 + c) * k + kk + q];
            }
        for (; kk < k; kk++) {
            const vd_t av = __builtin_convertvector(load_vf(a + kk * RB), vd_t);
            for (int c = 0; c < 2; c++) s[0][c] += av * (double)b[(c0 + c) * k + kk];
        }
        for (int c = 0; c < 2; c++) {
            const vd_t r = (s[0][c] + s[1][c]) + (s[2][c] + s[3][c]);
            memcpy(out[c0 + c], &r, sizeof(r));
        }
    }
}

/*
 * FP64 GEMM of the same FP32 / binary16 inputs (the error reference):
 * C64 = alpha * op(A) * op(B) + beta * Cin, all in double.  Cin may be NULL
 * when beta == 0.  C64 is column-major m x n with leading dimension m.
 */
int oracle_dgemm_ref(int op_a, int op_b, size_t m, size_t n, size_t k, double alpha,
                     const float* A, size_t lda, const uint16_t* B, size_t ldb, double beta,
                     const float* Cin, size_t ldc, int op_c, double* C64) {
    packed_t p;
    if (packed_make(&p, -1, op_a, op_b, m, n, k, A, lda, B, ldb)) return 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (size_t jb = 0; jb < p.nb; jb++) {
        for (size_t ib = 0; ib < p.mb; ib++) {
            double out[CB][RB];
            block_dgemm(p.a + ib * k * RB, p.b + jb * CB * k, k, out);
            for (size_t c = 0; c < CB && jb * CB + c < n; c++)
                for (size_t r = 0; r < RB && ib * RB + r < m; r++) {
                    const size_t i = ib * RB + r, j = jb * CB + c;
                    double s = alpha * out[c][r];
                    if (beta != 0.0) s += beta * (double)Cin[c_index(op_c, i, j, ldc)];
                    C64[i + j * m] = s;
                }
        }
    }
    packed_free(&p);
    return 0;
}

/* Sequential FP32 fused multiply-adds over k for one block. */
HOT static void block_sgemm(const float* restrict a, const float* restrict b, size_t k, float out[CB][RB]) {
    float acc[CB][RB];
    for (int c = 0; c < CB; c++)
        for (int r = 0; r < RB; r++) acc[c][r] = 0.0f;
    for (size_t kk = 0; kk < k; kk++)
        for (int c = 0; c < CB; c++) {
            const float bv = b[c * k + kk];
            for (int r = 0; r < RB; r++) acc[c][r] = fmaf(a[kk * RB + r], bv, acc[c][r]);
        }
    for (int c = 0; c < CB; c++)
        for (int r = 0; r < RB; r++) out[c][r] = acc[c][r];
}

/*
 * Plain FP32 SGEMM of the same inputs (the "SGEMM error" column): sequential
 * FP32 fused multiply-adds over k, then the same epilogue.
 */
int oracle_sgemm(int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                 const float* A, size_t lda, const uint16_t* B, size_t ldb, float beta,
                 float* C, size_t ldc, int op_c) {
    packed_t p;
    if (packed_make(&p, -1, op_a, op_b, m, n, k, A, lda, B, ldb)) return 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (size_t jb = 0; jb < p.nb; jb++) {
        for (size_t ib = 0; ib < p.mb; ib++) {
            float out[CB][RB];
            block_sgemm(p.a + ib * k * RB, p.b + jb * CB * k, k, out);
            for (size_t c = 0; c < CB && jb * CB + c < n; c++)
                for (size_t r = 0; r < RB && ib * RB + r < m; r++) {
                    float* cp = C + c_index(op_c, ib * RB + r, jb * CB + c, ldc);
                    *cp = epilogue(out[c][r], alpha, beta, cp);
                }
        }
    }
    packed_free(&p);
    return 0;
}

/*
 * Plain OpenMP GEMMs in FP32 and FP64 for the timed CPU baseline (not checkers):
 * C = A B, column-major, A m x k (lda), B k x n (ldb), C m x n (ldc), C overwritten.
 * Threads split the columns of C; a column is a sum of columns of A scaled by B's
 * entries, the innermost loop down a column of A (contiguous, vectorised).
 */
#define CPU_GEMM_COLUMN(T, NAME)                                                        \
    HOT static void NAME(size_t m, size_t k, const T* A, size_t lda, const T* bj, T* cj) { \
        for (size_t i = 0; i < m; i++) cj[i] = (T)0;                                    \
        for (size_t kk = 0; kk < k; kk++) {                                             \
            const T b = bj[kk];                                                         \
            const T* ak = A + kk * lda;                                                 \
            for (size_t i = 0; i < m; i++) cj[i] += ak[i] * b;                          \
        }                                                                               \
    }
CPU_GEMM_COLUMN(float, cpu_column_f32)
CPU_GEMM_COLUMN(double, cpu_column_f64)

void oracle_cpu_sgemm(size_t m, size_t n, size_t k, const float* A, size_t lda, const float* B, size_t ldb,
                      float* C, size_t ldc) {
#pragma omp parallel for schedule(dynamic, 4)
    for (size_t j = 0; j < n; j++) cpu_column_f32(m, k, A, lda, B + j * ldb, C + j * ldc);
}

void oracle_cpu_dgemm(size_t m, size_t n, size_t k, const double* A, size_t lda, const double* B, size_t ldb,
                      double* C, size_t ldc) {
#pragma omp parallel for schedule(dynamic, 4)
    for (size_t j = 0; j < n; j++) cpu_column_f64(m, k, A, lda, B + j * ldb, C + j * ldc);
}

/* Number of OpenMP threads the oracle runs with (for the CPU-baseline report). */
int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
