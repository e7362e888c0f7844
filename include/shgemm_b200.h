/*
 * shgemm_b200 -- C ABI of the B200 (sm_100a) SHGEMM library.
 *
 * Plain C types only (pointers, sizes, ints), so any FFI can bind it. Every
 * entry point returns an int status (SHGEMM_STATUS_*). Matrices are
 * column-major with BLAS op semantics; all matrix pointers are device memory
 * owned by the caller; alpha/beta point to host floats read at call time; work
 * is enqueued asynchronously on the handle's CUDA stream.
 *
 * Each entry point names the reference interface it replaces
 * (enp1s0/shgemm, paths relative to that project).
 */
#ifndef SHGEMM_B200_H_
#define SHGEMM_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct shgemm_b200_handle* shgemm_b200_handle_t;
struct shgemm_b200_problem; /* one problem of a grouped launch (below) */

/* operation_t (include/shgemm/shgemm.hpp:36-39) */
enum { SHGEMM_OP_N = 0, SHGEMM_OP_T = 1 };
/* tc_t (include/shgemm/shgemm.hpp:41-44) */
enum { SHGEMM_TC_FP16 = 0, SHGEMM_TC_TF32 = 1 };
/* detail::kernel_level (include/shgemm/shgemm.hpp:30-34) */
enum { SHGEMM_LEVEL_P0 = 0, SHGEMM_LEVEL_P1 = 1, SHGEMM_LEVEL_AUTO = -1 };

enum {
    SHGEMM_STATUS_OK = 0,
    SHGEMM_STATUS_INVALID_VALUE = 1,
    SHGEMM_STATUS_NOT_SUPPORTED = 2,
    SHGEMM_STATUS_ALLOC_FAILED = 3,
    SHGEMM_STATUS_LAUNCH_FAILED = 4,
    SHGEMM_STATUS_TIMEOUT = 5,
    SHGEMM_STATUS_CUDA_ERROR = 6,
    SHGEMM_STATUS_SCRATCH_TOO_SMALL = 7
};

/* Tunables for shgemm_b200_set_config (no reference counterpart; the
 * reference fixes these at compile time in its tile tables, src/shgemm.cu:429-488). */
enum {
    SHGEMM_CFG_SPLIT_K = 2,       /* 0 = automatic, 1 = never split, s > 1 = force s slices */
    SHGEMM_CFG_WAIT_LIMIT_MS = 3, /* bound on every in-kernel wait (default 2000 ms) */
    SHGEMM_CFG_GROUP_M = 4,       /* tile rasterisation group along m (default 8) */
    SHGEMM_CFG_GROUPED_B_FP32 = 5, /* 1: grouped TF32 batches pass B as FP32 values that are
                                      exactly binary16 (a widened copy), loaded without a
                                      conversion; 0 (default): B is binary16 */
    SHGEMM_CFG_AUTOTUNE = 6,       /* 0: heuristic plans only; 1 (default): a shape whose bucket
                                      the autotuner has an entry for uses it; 2: as 1, and a call
                                      with beta == 0 on an untuned bucket tunes it first */
    SHGEMM_CFG_TILE_KERNEL = 7,    /* 0 (default): 128x256 binary16 tiles with a K-major B run the
                                      kernel that keeps hi/lo in tensor memory; 1: always the
                                      shared-memory operand kernel */
    SHGEMM_CFG_K_CHUNK = 8         /* k between FP32 round-to-nearest drains of the tensor-core
                                      accumulator in the tensor-memory kernel: 64 (default) or
                                      128 (measured: ~1.2x the 64-k error on mixed-sign data,
                                      ~2.2x on all-positive data, within 2x FP32 SGEMM's error);
                                      the other kernels always drain every 64 */,
    SHGEMM_CFG_HOST_BLOCK_COLS = 9, /* columns of C per block of shgemm_b200_shgemm_host:
                                      0 (default) = a multiple of 256 giving about 16 blocks */
    SHGEMM_CFG_TM_STAGES = 10,     /* operand ring of the tensor-memory kernel when no tuned entry
                                      applies: 0 (default) = 4 FP32 A + 3 binary16 B stages, 1 = 3 + 4 */
    SHGEMM_CFG_PAIR_TILES = 11     /* when no tuned entry applies: 1 = run the tensor-memory kernel in
                                      CTA pairs (256 x 256 tiles over two SMs, tcgen05 cta_group::2,
                                      half the B traffic per SM), 0 (default) = one CTA per tile */
};

/* ------------------------------------------------------------------------
 * Autotuner. No reference counterpart (the reference fixes its tile tables at
 * compile time, src/shgemm.cu:429-488, and picks one of two levels per call,
 * src/shgemm.cu:643-656). A shape bucket is (compute type, op_a, op_b,
 * floor(log2 m), floor(log2 n), floor(log2 k)); its entry names the tile N,
 * the split-K slice count, the tile rasterisation group and, for the 128 x 256
 * binary16 tiles of the tensor-memory kernel, the operand ring (stage counts) and
 * the k-chunk of the FP32 drain. A 128-k chunk is only chosen when it is faster
 * AND passes an accuracy gate: on sampled blocks of C its relative error against
 * an FP64 product of the same operands is at most 1.25x that of the 64-k chunk.
 * ------------------------------------------------------------------------ */
typedef struct {
    int tile_n;   /* 64, 128 or 256 (binary16); 64 or 128 (TF32) */
    int slices;   /* split-K slices, 1 = none */
    int group_m;  /* tiles along m per rasterisation group */
    float time_us;
    int stages;   /* tensor-memory kernel ring: 0 = 4 FP32 A + 3 binary16 B stages, 1 = 3 + 4 */
    int k_chunk;  /* tensor-memory kernel: k between FP32 drains, 64 or 128 */
    int cta_group; /* tensor-memory kernel: 1 = one CTA per 128 x 256 tile, 2 = CTA pairs (256 x 256) */
} shgemm_b200_tuned_config;

/* Times every candidate configuration on the given operands (C is overwritten with
 * A B: the runs use alpha = 1, beta = 0), stores the fastest for the shape's bucket
 * and returns it in *best. Synchronises the handle's stream; not while capturing.
 * Operands must be TMA-addressable (16-byte aligned, 16-byte leading dimensions).
 * The accuracy gate allocates and frees two small device buffers. */
int shgemm_b200_autotune(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                         const float* a, size_t lda, const void* b, size_t ldb, float* c, size_t ldc,
                         int compute_type, shgemm_b200_tuned_config* best);
/* The entry for a shape's bucket: SHGEMM_STATUS_OK and *cfg, or SHGEMM_STATUS_INVALID_VALUE if none. */
int shgemm_b200_autotune_lookup(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                                int compute_type, shgemm_b200_tuned_config* cfg);
/* Tunes the tile N of grouped launches per n bucket, floor(log2 n), on a real batch
 * (problems as for shgemm_b200_shgemm_grouped; their C is overwritten by the timing
 * runs, which are eager grouped launches on the handle's stream): for every bucket the
 * batch holds, every tile N the kernel allows is timed with the other buckets at their
 * current choice, and the fastest is kept. Later grouped launches of the same compute
 * type, op_a and B format use the entries; buckets without one keep the default rule
 * (the smallest power of two >= n). *tuned (may be NULL) receives the number of
 * buckets tuned. Not while capturing. */
int shgemm_b200_autotune_grouped(shgemm_b200_handle_t handle, int op_a, int op_b, int compute_type, int op_c,
                                 const struct shgemm_b200_problem* problems, int count, int* tuned);
/* The grouped entry for one n bucket: SHGEMM_STATUS_OK and *tile_n, or SHGEMM_STATUS_INVALID_VALUE if none.
 * b_fp32: the B format (SHGEMM_CFG_GROUPED_B_FP32). */
int shgemm_b200_autotune_grouped_lookup(shgemm_b200_handle_t handle, int op_a, int compute_type, int b_fp32, size_t n,
                                        int* tile_n);
/* Writes / reads the table as text, one bucket per line (plain and grouped entries). Loading adds to the table. */
int shgemm_b200_autotune_save(shgemm_b200_handle_t handle, const char* path);
int shgemm_b200_autotune_load(shgemm_b200_handle_t handle, const char* path);
int shgemm_b200_autotune_clear(shgemm_b200_handle_t handle);

/* mtk::shgemm::create (include/shgemm/shgemm.hpp:94; src/shgemm.cu:401-490).
 * Binds the handle to `device` (the reference hard-codes device 0, src/shgemm.cu:419-425),
 * allocates the handle's workspace and error word once. */
int shgemm_b200_create(shgemm_b200_handle_t* handle, int device);

/* mtk::shgemm::destroy (include/shgemm/shgemm.hpp:95; src/shgemm.cu:492-496). */
int shgemm_b200_destroy(shgemm_b200_handle_t handle);

/* mtk::shgemm::set_cuda_stream (include/shgemm/shgemm.hpp:102; src/shgemm.cu:498-503).
 * `cuda_stream` is a cudaStream_t (NULL = legacy default stream). */
int shgemm_b200_set_stream(shgemm_b200_handle_t handle, void* cuda_stream);

/* mtk::shgemm::enable_kernel_level_fixing / disable_kernel_level_fixing
 * (include/shgemm/shgemm.hpp:97-98; src/shgemm.cu:505-515). SHGEMM_LEVEL_AUTO disables. */
int shgemm_b200_set_kernel_level(shgemm_b200_handle_t handle, int level);

/* mtk::shgemm::set_debug_mode (include/shgemm/shgemm.hpp:100; src/shgemm.cu:688-690). */
int shgemm_b200_set_debug_mode(shgemm_b200_handle_t handle, unsigned on);

/* mtk::shgemm::shgemm (include/shgemm/shgemm.hpp:105-119; src/shgemm.cu:517-686):
 * C = alpha * op(A) * op(B) + beta * C, A FP32, B binary16 (`b` points to __half),
 * op_c == SHGEMM_OP_T stores C transposed. TF32 calls with a K-contiguous B whose
 * 128 x 256 tiles fill the GPU and whose widened B (n * round4(k) floats) fits the handle
 * workspace widen B there first and run the TF32 kernel that loads it unconverted
 * (not while capturing). Binary16 calls whose K-contiguous B has columns >= 1 MiB apart
 * (ldb >= 512 Ki) and run on 128 x 256 tiles re-lay B out in the workspace as contiguous
 * 64-deep k-blocks first, when it holds n * round64(k) * 2 bytes besides the split-K
 * partials (a wide column pitch otherwise halves the load rate). *level_out (may be NULL)
 * receives the kernel level used, like the reference's return value. */
int shgemm_b200_shgemm(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                       const float* alpha, const float* a, size_t lda, const void* b, size_t ldb,
                       const float* beta, float* c, size_t ldc, int compute_type, int op_c, int* level_out);

/* mtk::shgemm::shgemm with alpha and beta in DEVICE memory (the reference reads them on the
 * host at call time, src/shgemm.cu:532,600,603; no counterpart there). alpha_dev and beta_dev
 * are 4-byte aligned device addresses of one float each; the kernels read them when they
 * run, so a launch captured in a CUDA graph picks up whatever the caller stored there before
 * each replay. Everything else as shgemm_b200_shgemm, including that C is not read when
 * *beta_dev == 0; autotuning on first use (SHGEMM_CFG_AUTOTUNE = 2) is skipped, since it
 * needs beta == 0 known on the host. */
int shgemm_b200_shgemm_device_scalars(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                                      const float* alpha_dev, const float* a, size_t lda, const void* b, size_t ldb,
                                      const float* beta_dev, float* c, size_t ldc, int compute_type, int op_c,
                                      int* level_out);

/* hsgemm with device-resident alpha and beta: shgemm_b200_shgemm_device_scalars through
 * the transposition identity of include/shgemm/shgemm.hpp:121-157. */
int shgemm_b200_hsgemm_device_scalars(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                                      const float* alpha_dev, const void* a, size_t lda, const float* b, size_t ldb,
                                      const float* beta_dev, float* c, size_t ldc, int compute_type, int op_c,
                                      int* level_out);

/* SHGEMM on host buffers (no reference counterpart: the reference takes device
 * pointers only). Same arguments, status codes and results as shgemm_b200_shgemm,
 * but a, b and c are host addresses. A is copied to the device once; C is then
 * produced in column blocks (SHGEMM_CFG_HOST_BLOCK_COLS) through three device slots,
 * block j's B and C columns going up while block j-1 computes and block j-2's C
 * comes back, so both PCIe directions overlap the tensor work. Host buffers should
 * be page-locked (cudaHostAlloc / cudaHostRegister); pageable memory gives correct
 * results without the overlap. Device staging (A plus three blocks) belongs to the
 * handle and grows when a call needs more, the only allocation this entry point
 * makes (refused with SHGEMM_STATUS_NOT_SUPPORTED while the stream is capturing);
 * shgemm_b200_release_host_staging frees it. Asynchronous like every call here:
 * synchronise the handle's stream before reading c or reusing a or b. */
int shgemm_b200_shgemm_host(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                            const float* alpha, const float* a, size_t lda, const void* b, size_t ldb,
                            const float* beta, float* c, size_t ldc, int compute_type, int op_c, int* level_out);

/* hsgemm on host buffers (A binary16, B FP32): shgemm_b200_shgemm_host through the
 * same transposition identity as shgemm_b200_hsgemm. */
int shgemm_b200_hsgemm_host(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                            const float* alpha, const void* a, size_t lda, const float* b, size_t ldb,
                            const float* beta, float* c, size_t ldc, int compute_type, int op_c, int* level_out);

/* Frees the handle's host-entry staging (after synchronising its streams). */
int shgemm_b200_release_host_staging(shgemm_b200_handle_t handle);

/* mtk::shgemm::hsgemm (include/shgemm/shgemm.hpp:121-157): A binary16, B FP32,
 * computed through the same transposition identity as the reference. */
int shgemm_b200_hsgemm(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                       const float* alpha, const void* a, size_t lda, const float* b, size_t ldb,
                       const float* beta, float* c, size_t ldc, int compute_type, int op_c, int* level_out);

/* ------------------------------------------------------------------------
 * Grouped launches (no reference counterpart; the reference's equivalent is a
 * host loop of shgemm calls, one launch each). Many independent problems
 * C_i = alpha_i op(A_i) op(B_i) + beta_i C_i in ONE persistent launch: a
 * per-problem table of TMA descriptors and a unit list (tiles, longest first)
 * in device memory, built on the host. All problems share op_a, op_b (op_n
 * only), op_c and the compute type; operands must be TMA-addressable (16-byte
 * aligned bases and leading dimensions). Tile N per problem: the smallest of
 * 32/64/128/256 (TF32: up to 128) covering n_i.
 * ------------------------------------------------------------------------ */
typedef struct shgemm_b200_problem {
    size_t m, n, k;
    const float* a;
    size_t lda;
    const void* b; /* binary16 */
    size_t ldb;
    float* c;
    size_t ldc;
    float alpha, beta;
    /* 0: B is given (b, ldb). SHGEMM_OMEGA_RADEMACHER_BLOCKS (binary16 compute only): B is the
     * k x n block-sign operand of omega_seed with entries +1 / -1, generated by the kernel
     * as it goes instead of loaded (b and ldb unused): no Omega in memory and no Omega
     * traffic. The values are those shgemm_b200_generate_omega writes for the same seed with
     * scale 1; scale the sketch through alpha. */
    int b_generated;
    unsigned long long omega_seed;
} shgemm_b200_problem;

/* Enqueues (on the handle's stream) the copy of the batch's tables from the
 * handle's pinned host staging to the device and one grouped kernel launch.
 * Can be captured in a CUDA graph: replaying the graph copies whatever the
 * staging holds, so shgemm_b200_grouped_update + cudaGraphLaunch runs a new
 * batch with the captured launch (up to the captured number of problems).
 * At most 8192 problems and 65536 tiles per batch. */
int shgemm_b200_shgemm_grouped(shgemm_b200_handle_t handle, int op_a, int op_b, int compute_type, int op_c,
                               const shgemm_b200_problem* problems, int count);

/* Rewrites the pinned host staging with a new batch without enqueueing anything
 * (for replaying a captured grouped launch). The batch must use the op_a,
 * compute type and op_c the launch was captured with, and no replay of that
 * launch may still be pending (its copy reads the staging): synchronise first.
 * Every grouped call restages the table, and so does an eager TF32 shgemm call that
 * takes the widened-B route (see shgemm_b200_shgemm): update before each replay. */
int shgemm_b200_grouped_update(shgemm_b200_handle_t handle, int op_a, int op_b, int compute_type, int op_c,
                               const shgemm_b200_problem* problems, int count);

/* Tunables (no reference counterpart). */
int shgemm_b200_set_config(shgemm_b200_handle_t handle, int key, long long value);
int shgemm_b200_get_config(shgemm_b200_handle_t handle, int key, long long* value);

/* Resizes the handle-owned split-K workspace (the reference's w_ptr,
 * src/shgemm.cu:417). Allocation happens here, never inside shgemm calls. */
int shgemm_b200_set_workspace_size(shgemm_b200_handle_t handle, size_t bytes);

/* The handle's workspace: its device address and size in bytes (the reference's
 * w_ptr and max_working_memory_num_elements, include/shgemm/shgemm.hpp:46-92,
 * src/shgemm.cu:417). Valid until the next shgemm_b200_set_workspace_size or
 * shgemm_b200_destroy; calls on the handle overwrite its contents. */
int shgemm_b200_get_workspace(shgemm_b200_handle_t handle, void** ptr, size_t* bytes);

/* The heuristic plan of a call, without a device: the kernel level (0: the smaller tile N,
 * 1: the larger; the reference's choice, src/shgemm.cu:643-656: the large tile when it fills
 * the machine or when split-K will), the tile N, and the deterministic split-K slice count
 * (split when the tiles leave SMs idle, k >= 4096 and the workspace holds >= 2 partials of
 * m x n FP32; the count maximises the busy fraction of num_sms over the waves). Autotuned
 * entries, the widened-B TF32 path and level fixing can override it on a handle. */
int shgemm_b200_plan_preview(int num_sms, size_t m, size_t n, size_t k, int compute_type, size_t workspace_bytes,
                             int* level, int* tile_n, int* slices);

/* Synchronises the handle's stream and reports (then clears) the device-side
 * error word: SHGEMM_STATUS_TIMEOUT when a kernel gave up a bounded wait
 * (*device_code = which role), SHGEMM_STATUS_CUDA_ERROR on a CUDA error.
 * No reference counterpart (the reference checks no launch). */
int shgemm_b200_check_error(shgemm_b200_handle_t handle, int* device_code);

/* Number of kernels this library enqueued since the handle was created. */
int shgemm_b200_get_launch_count(shgemm_b200_handle_t handle, long long* count);

/* Human-readable status name. */
const char* shgemm_b200_status_string(int status);

/* Self-test of the bounded in-kernel wait: launches one CTA that waits on an
 * mbarrier nothing arrives at, with a limit of `limit_us`; the kernel must give
 * up, record the timeout and return. *observed receives the device error code.
 * No reference counterpart. */
int shgemm_b200_selftest_wait_timeout(shgemm_b200_handle_t handle, unsigned limit_us, int* observed);

/* ------------------------------------------------------------------------
 * Evaluation helpers (FP64 on the GPU, used only to measure error; the
 * reference's role for these is mateval, test/shgemm_test.cu:91-100).
 * ------------------------------------------------------------------------ */

/* C64 (m x n, ld = m, column-major) = op(A) * op(B) in FP64 from FP32 A and binary16 B. */
int shgemm_b200_eval_dgemm(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                           const float* a, size_t lda, const void* b, size_t ldb, double* c64);

/* Same with the operand types swapped (A binary16, B FP32), for HSGEMM results. */
int shgemm_b200_eval_dgemm_hs(shgemm_b200_handle_t handle, int op_a, int op_b, size_t m, size_t n, size_t k,
                              const void* a, size_t lda, const float* b, size_t ldb, double* c64);

/* Error of C (op_c layout, ldc) against ref = alpha*C64 + beta*C0 (C0 may be NULL when beta == 0):
 * out[0] = ||C - ref||_F over entries finite in both, out[1] = ||ref||_F over the same,
 * out[2] = max |C - ref| / |ref| over those entries with ref != 0,
 * out[3] = number of entries where C and ref disagree on being finite. */
int shgemm_b200_eval_error(shgemm_b200_handle_t handle, size_t m, size_t n, const float* c, size_t ldc, int op_c,
                           const double* c64, double alpha, double beta, const float* c0, double* out);

/* ------------------------------------------------------------------------
 * Allocation-free entry point. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc -- code running inside an allocator
 * callback, a memory manager that owns all device memory, or a process that
 * reserved its device memory up front -- and so cannot create a handle (whose
 * workspace is allocated). It computes what shgemm_b200_shgemm computes (same
 * kernels, same deterministic split-K), on the current device and the given
 * stream, and allocates nothing: the split-K partials live in a 16 MiB
 * file-scope device array of the library and the error word in another. The
 * driver reserves the arrays on a device when the library's device code is
 * loaded there -- with CUDA's lazy module loading (the default), during the
 * first call on that device -- and keeps them until the process exits.
 * MTK_SHGEMM_KERNEL_LEVEL and MTK_SHGEMM_DEBUG apply as in shgemm_b200_create.
 *  - Limit: m * n <= shgemm_b200_noalloc_scratch_bytes() / 8 (two slices of
 *    FP32 partials); larger problems return SHGEMM_STATUS_SCRATCH_TOO_SMALL.
 *    Operands must be 16-byte aligned with 16-byte aligned leading dimensions
 *    (no staging), else SHGEMM_STATUS_NOT_SUPPORTED.
 *  - The first call on a device sets that device up (resolves the arrays'
 *    device addresses, raises kernel shared-memory limits) and may make the
 *    driver load the library's device code and reserve the arrays. Make it at
 *    start-up, while device memory can still be reserved (before a memory
 *    manager claims the rest, outside allocator callbacks), and before any
 *    stream capture: one warm-up call on each device is enough.
 *  - Every call shares the arrays: calls that overlap on the GPU (different
 *    streams, or different host threads) race on the partials. Serialise them.
 *  - The error word is shared too and sticky: a bounded wait that gave up in any
 *    call stays recorded until shgemm_b200_noalloc_check_error reads and clears
 *    it. Check after each call whose result you depend on.
 * ------------------------------------------------------------------------ */
int shgemm_b200_shgemm_noalloc(void* cuda_stream, int op_a, int op_b, size_t m, size_t n, size_t k,
                               const float* alpha, const float* a, size_t lda, const void* b, size_t ldb,
                               const float* beta, float* c, size_t ldc, int compute_type, int op_c, int* level_out);

/* Size of the allocation-free path's scratch array in bytes. No counterpart in the reference. */
size_t shgemm_b200_noalloc_scratch_bytes(void);

/* Synchronises `cuda_stream` and reports (then clears) the allocation-free path's
 * device error word, as shgemm_b200_check_error does for a handle. No counterpart
 * in the reference. */
int shgemm_b200_noalloc_check_error(void* cuda_stream, int* device_code);

/* ------------------------------------------------------------------------
 * Sketch generation and the sketch server. No counterpart in the reference
 * (whose sketches are host loops of shgemm calls).
 * ------------------------------------------------------------------------ */

/* Distribution of a generated sketch operand Omega. RADEMACHER_BLOCKS: random signs from one
 * 64-bit hash per 64 consecutive entries of a column: entry (r, c) is negative when bit
 * b(r mod 64) of splitmix64(seed * 0x9E3779B97F4A7C15 + c * ceil(k / 64) + r / 64 + 1) is set,
 * b(i) = 32 (i / 32) + (i / 2 mod 16) + 16 (i mod 2) -- adjacent entries take bits 16 apart,
 * so a 32-bit word of two binary16 values is one shift and one mask. This is the stream
 * grouped launches can generate in the kernel instead of loading Omega. */
enum { SHGEMM_OMEGA_GAUSSIAN = 0, SHGEMM_OMEGA_RADEMACHER = 1, SHGEMM_OMEGA_RADEMACHER_BLOCKS = 2 };

/* Writes Omega (k x cols, column-major, leading dimension ld elements) on `cuda_stream`:
 * entry (r, c) = scale * g rounded to binary16. GAUSSIAN: entries 2i and 2i + 1 of a column
 * are the cosine and sine normals of one Box-Muller pair from the splitmix64 counter hash of
 * (seed, c * k + 2i). RADEMACHER: a random sign from the hash of (seed, c * k + r).
 * fp32 = 0 stores binary16; fp32 = 1 stores the same binary16 values widened to FP32 (the B
 * operand of a TF32 batch with SHGEMM_CFG_GROUPED_B_FP32). */
int shgemm_b200_generate_omega(void* cuda_stream, void* dst, size_t ld, size_t k, size_t cols, int dist,
                               unsigned long long seed, float scale, int fp32);

/* One Omega of a batch, with the arguments of shgemm_b200_generate_omega. */
struct shgemm_b200_omega_job {
    void* dst;
    size_t ld;
    size_t k;
    size_t cols;
    unsigned long long seed;
    float scale;
    int dist;
};

/* Writes `count` Omegas, each exactly as shgemm_b200_generate_omega would, in one launch per 64
 * jobs on `cuda_stream` (the sketch server generates all draws of a batch this way). fp32 applies
 * to every job. */
int shgemm_b200_generate_omega_batch(void* cuda_stream, const struct shgemm_b200_omega_job* jobs, int count,
                                     int fp32);

typedef struct shgemm_b200_server* shgemm_b200_server_t;

typedef struct {
    size_t hbm_budget_bytes; /* admission budget: A + Omega + Y of every admitted request */
    int compute_type;        /* SHGEMM_TC_FP16 or SHGEMM_TC_TF32 */
    int max_batch;           /* requests per grouped launch (<= 8192; 0: 512) */
    int streams;             /* grouped launches in flight at once (1..8; 0: 3) */
    int auto_release;        /* 1: a completed request's Y is freed at once (throughput runs) */
} shgemm_b200_server_config;

/* One sketch request: Y = A [Omega_1 ... Omega_draws], A m x k FP32 column-major
 * (op_n, 16-byte aligned with lda a multiple of 4, device memory the caller keeps
 * unchanged until the request completes). Omega_j (k x n) is what
 * shgemm_b200_generate_omega writes for seed omega_seed * 1099511628211 + j.
 * Y is m x (draws n), column-major with ld m, allocated by the server inside the budget. */
typedef struct {
    size_t m, n, k;
    const float* a;
    size_t lda;
    int draws;
    int omega_dist;          /* SHGEMM_OMEGA_* */
    float omega_scale;       /* e.g. 1/sqrt(n) */
    unsigned long long omega_seed;
} shgemm_b200_sketch_request;

enum { SHGEMM_REQ_QUEUED = 0, SHGEMM_REQ_ADMITTED = 1, SHGEMM_REQ_RUNNING = 2, SHGEMM_REQ_DONE = 3,
       SHGEMM_REQ_FAILED = 4, SHGEMM_REQ_UNKNOWN = 5 };

typedef struct {
    unsigned long long submitted, completed, failed, batches;
    double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> completion observed, completed requests */
    double flops_completed;                 /* sum of 2 m (draws n) k */
    double span_s;                          /* first submit -> last completion */
    size_t peak_resident_bytes;             /* max over time of the admitted A + Omega + Y bytes */
    size_t resident_bytes;
    unsigned long long queued, in_flight;   /* now */
    /* Device-side timing (CUDA events on the server's streams), completed batches only:
     * kernel_busy_s = time during which at least one grouped SHGEMM launch was running
     * (the union of their intervals), omega_s = summed time of the Omega generation. */
    double kernel_busy_s, omega_s;
    unsigned long long launches;            /* kernels enqueued: grouped launches + Omega generations */
} shgemm_b200_server_stats;

/* Starts a server thread on `device` that admits requests first-come first-served
 * while their A + Omega + Y bytes fit the budget, generates their Omega draws,
 * batches the admitted requests into grouped launches on up to `streams` streams
 * (so a new batch starts while earlier ones finish) and records each completion.
 * Omega and Y live in one device arena of the budget's size allocated here. */
int shgemm_b200_server_create(shgemm_b200_server_t* server, int device, const shgemm_b200_server_config* config);
int shgemm_b200_server_destroy(shgemm_b200_server_t server);
/* Queues a request (returns at once). SHGEMM_STATUS_NOT_SUPPORTED if it can never fit the budget. */
int shgemm_b200_server_submit(shgemm_b200_server_t server, const shgemm_b200_sketch_request* request,
                              unsigned long long* ticket);
/* State of a request; when done, *y / *ldy give its result and *latency_ms the
 * submit-to-completion time. Any output pointer may be NULL. */
int shgemm_b200_server_poll(shgemm_b200_server_t server, unsigned long long ticket, int* state, float** y,
                            size_t* ldy, double* latency_ms);
/* Waits (up to timeout_ms) until the request is done or failed. */
int shgemm_b200_server_wait(shgemm_b200_server_t server, unsigned long long ticket, double timeout_ms, int* state);
/* Waits (up to timeout_ms) until every submitted request is done or failed. */
int shgemm_b200_server_drain(shgemm_b200_server_t server, double timeout_ms);
/* Returns a completed request's Y to the budget (not needed with auto_release). */
int shgemm_b200_server_release(shgemm_b200_server_t server, unsigned long long ticket);
int shgemm_b200_server_get_stats(shgemm_b200_server_t server, shgemm_b200_server_stats* stats);
/* Forgets the latency samples and counters (not the requests in flight). */
int shgemm_b200_server_reset_stats(shgemm_b200_server_t server);

#ifdef __cplusplus
}
#endif

#endif /* SHGEMM_B200_H_ */
