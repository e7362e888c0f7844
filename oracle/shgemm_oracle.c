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
 *    that takes each fragment's sum with truncation.
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

/* Packs op(A) as [m][k] rows and op(B) as [n][k] rows (k contiguous). */
static void pack_a(int op, size_t m, size_t k, const float* A, size_t lda, float* out) {
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < m; i++)
        for (size_t kk = 0; kk < k; kk++) out[i * k + kk] = A[a_index(op, i, kk, lda)];
}
static void pack_b_f16(int op, size_t k, size_t n, const uint16_t* B, size_t ldb, float* out) {
#pragma omp parallel for schedule(static)
    for (size_t j = 0; j < n; j++)
        for (size_t kk = 0; kk < k; kk++) out[j * k + kk] = oracle_f16_bits_to_f32(B[b_index(op, kk, j, ldb)]);
}

static inline float epilogue(float acc, float alpha, float beta, const float* c) {
    if (beta == 0.0f) return acc * alpha;
    return fmaf(acc, alpha, beta * (*c));
}

/*
 * Restated reference SHGEMM: C = alpha * op(A) * op(B) + beta * C with A FP32
 * and B binary16 (bits). chunk = hi-fragment length. Returns 0 on success.
 */
int oracle_shgemm(int tc, int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                  const float* A, size_t lda, const uint16_t* B, size_t ldb, float beta,
                  float* C, size_t ldc, int op_c, size_t chunk) {
    if (chunk == 0) chunk = (tc == TC_FP16) ? 16 : 8;
    float* a = (float*)malloc(sizeof(float) * (m * k + 1));
    float* ahi = (float*)malloc(sizeof(float) * (m * k + 1));
    float* alo = (float*)malloc(sizeof(float) * (m * k + 1));
    float* b = (float*)malloc(sizeof(float) * (n * k + 1));
    if (!a || !ahi || !alo || !b) { free(a); free(ahi); free(alo); free(b); return 1; }
    pack_a(op_a, m, k, A, lda, a);
    oracle_split(tc, a, m * k, ahi, alo);
    pack_b_f16(op_b, k, n, B, ldb, b);
    /* TF32 compute: the binary16 operand is exact in TF32 (src/utils.hpp:15-17). */
#pragma omp parallel for collapse(2) schedule(static)
    for (size_t j = 0; j < n; j++) {
        for (size_t i = 0; i < m; i++) {
            const float* ah = ahi + i * k;
            const float* al = alo + i * k;
            const float* bj = b + j * k;
            float acc = 0.0f;
            double lo = 0.0;
            for (size_t k0 = 0; k0 < k; k0 += chunk) {
                const size_t k1 = (k0 + chunk < k) ? k0 + chunk : k;
                double s = 0.0;
                for (size_t kk = k0; kk < k1; kk++) {
                    s += (double)ah[kk] * (double)bj[kk];
                    lo += (double)al[kk] * (double)bj[kk];
                }
                acc = acc + (float)s;
            }
            const float c = acc + (float)lo * (1.0f / 2048.0f);
            float* cp = C + c_index(op_c, i, j, ldc);
            *cp = epilogue(c, alpha, beta, cp);
        }
    }
    free(a); free(ahi); free(alo); free(b);
    return 0;
}

/* FP32 value of a double rounded toward zero (the tensor core's truncating
 * accumulation is modelled as exact products and sums rounded this way). */
static inline float rz_f32(double d) {
    float f = (float)d; /* round to nearest */
    if (isfinite(f) && fabs((double)f) > fabs(d)) f = nextafterf(f, 0.0f);
    return f;
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
 * Products of split values with binary16 values are exact in FP64.
 */
int oracle_shgemm_tcmodel(int tc, int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                          const float* A, size_t lda, const uint16_t* B, size_t ldb, float beta,
                          float* C, size_t ldc, int op_c, size_t chunk) {
    if (chunk == 0) chunk = (tc == TC_FP16) ? 16 : 8;
    float* a = (float*)malloc(sizeof(float) * (m * k + 1));
    float* ahi = (float*)malloc(sizeof(float) * (m * k + 1));
    float* alo = (float*)malloc(sizeof(float) * (m * k + 1));
    float* b = (float*)malloc(sizeof(float) * (n * k + 1));
    if (!a || !ahi || !alo || !b) { free(a); free(ahi); free(alo); free(b); return 1; }
    pack_a(op_a, m, k, A, lda, a);
    oracle_split(tc, a, m * k, ahi, alo);
    pack_b_f16(op_b, k, n, B, ldb, b);
#pragma omp parallel for collapse(2) schedule(static)
    for (size_t j = 0; j < n; j++) {
        for (size_t i = 0; i < m; i++) {
            const float* ah = ahi + i * k;
            const float* al = alo + i * k;
            const float* bj = b + j * k;
            float acc = 0.0f, lo = 0.0f;
            for (size_t k0 = 0; k0 < k; k0 += chunk) {
                const size_t k1 = (k0 + chunk < k) ? k0 + chunk : k;
                double s = 0.0, t = 0.0;
                for (size_t kk = k0; kk < k1; kk++) {
                    s += (double)ah[kk] * (double)bj[kk];
                    t += (double)al[kk] * (double)bj[kk];
                }
                acc = acc + rz_f32(s);
                lo = rz_f32((double)lo + t);
            }
            const float c = acc + lo * (1.0f / 2048.0f);
            float* cp = C + c_index(op_c, i, j, ldc);
            *cp = epilogue(c, alpha, beta, cp);
        }
    }
    free(a); free(ahi); free(alo); free(b);
    return 0;
}

/*
 * FP64 GEMM of the same FP32 / binary16 inputs (the error reference):
 * C64 = alpha * op(A) * op(B) + beta * Cin, all in double.  Cin may be NULL
 * when beta == 0.  C64 is column-major m x n with leading dimension m.
 */
int oracle_dgemm_ref(int op_a, int op_b, size_t m, size_t n, size_t k, double alpha,
                     const float* A, size_t lda, const uint16_t* B, size_t ldb, double beta,
                     const float* Cin, size_t ldc, int op_c, double* C64) {
    float* a = (float*)malloc(sizeof(float) * (m * k + 1));
    float* b = (float*)malloc(sizeof(float) * (n * k + 1));
    if (!a || !b) { free(a); free(b); return 1; }
    pack_a(op_a, m, k, A, lda, a);
    pack_b_f16(op_b, k, n, B, ldb, b);
#pragma omp parallel for collapse(2) schedule(static)
    for (size_t j = 0; j < n; j++) {
        for (size_t i = 0; i < m; i++) {
            const float* ai = a + i * k;
            const float* bj = b + j * k;
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            size_t kk = 0;
            for (; kk + 4 <= k; kk += 4) {
                s0 += (double)ai[kk] * bj[kk];
                s1 += (double)ai[kk + 1] * bj[kk + 1];
                s2 += (double)ai[kk + 2] * bj[kk + 2];
                s3 += (double)ai[kk + 3] * bj[kk + 3];
            }
            for (; kk < k; kk++) s0 += (double)ai[kk] * bj[kk];
            double s = alpha * ((s0 + s1) + (s2 + s3));
            if (beta != 0.0) s += beta * (double)Cin[c_index(op_c, i, j, ldc)];
            C64[i + j * m] = s;
        }
    }
    free(a); free(b);
    return 0;
}

/*
 * Plain FP32 SGEMM of the same inputs (the "SGEMM error" column): sequential
 * FP32 fused multiply-adds over k, then the same epilogue.
 */
int oracle_sgemm(int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                 const float* A, size_t lda, const uint16_t* B, size_t ldb, float beta,
                 float* C, size_t ldc, int op_c) {
    float* a = (float*)malloc(sizeof(float) * (m * k + 1));
    float* b = (float*)malloc(sizeof(float) * (n * k + 1));
    if (!a || !b) { free(a); free(b); return 1; }
    pack_a(op_a, m, k, A, lda, a);
    pack_b_f16(op_b, k, n, B, ldb, b);
#pragma omp parallel for collapse(2) schedule(static)
    for (size_t j = 0; j < n; j++) {
        for (size_t i = 0; i < m; i++) {
            const float* ai = a + i * k;
            const float* bj = b + j * k;
            float acc = 0.0f;
            for (size_t kk = 0; kk < k; kk++) acc = fmaf(ai[kk], bj[kk], acc);
            float* cp = C + c_index(op_c, i, j, ldc);
            *cp = epilogue(acc, alpha, beta, cp);
        }
    }
    free(a); free(b);
    return 0;
}

/*
 * Plain OpenMP GEMMs in FP32 and FP64 for the timed CPU baseline (not checkers):
 * C = A B, column-major, A m x k (lda), B k x n (ldb), C m x n (ldc), C overwritten.
 * Threads split the columns of C; each walks k in blocks of 256 so the block of A
 * stays in cache, with the innermost loop down a column (contiguous, vectorisable).
 */
#define CPU_GEMM_KB 256
#define CPU_GEMM_BODY(T)                                                           \
    _Pragma("omp parallel for schedule(dynamic, 4)")                               \
    for (size_t j = 0; j < n; j++) {                                               \
        T* cj = C + j * ldc;                                                       \
        for (size_t i = 0; i < m; i++) cj[i] = (T)0;                               \
        for (size_t k0 = 0; k0 < k; k0 += CPU_GEMM_KB) {                           \
            const size_t k1 = (k0 + CPU_GEMM_KB < k) ? k0 + CPU_GEMM_KB : k;       \
            for (size_t kk = k0; kk < k1; kk++) {                                  \
                const T b = B[kk + j * ldb];                                       \
                const T* ak = A + kk * lda;                                        \
                for (size_t i = 0; i < m; i++) cj[i] += ak[i] * b;                 \
            }                                                                      \
        }                                                                          \
    }

void oracle_cpu_sgemm(size_t m, size_t n, size_t k, const float* A, size_t lda, const float* B, size_t ldb,
                      float* C, size_t ldc) {
    CPU_GEMM_BODY(float)
}

void oracle_cpu_dgemm(size_t m, size_t n, size_t k, const double* A, size_t lda, const double* B, size_t ldb,
                      double* C, size_t ldc) {
    CPU_GEMM_BODY(double)
}

/* Number of OpenMP threads the oracle runs with (for the CPU-baseline report). */
int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
