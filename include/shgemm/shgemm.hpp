// mtk::shgemm -- source-compatible C++ API of the reference library
// (enp1s0/shgemm include/shgemm/shgemm.hpp), implemented on B200 (sm_100a)
// by libshgemm_b200 through the C ABI in shgemm_b200.h.
//
// Names, signatures and semantics follow the reference: column-major BLAS
// operands, host-side alpha/beta pointers, asynchronous execution on the
// handle's CUDA stream. The handle's internals differ (the reference keeps a
// table of kernel slots, include/shgemm/shgemm.hpp:46-92); it stays copyable by
// value and keeps the fields user code may touch.
#ifndef __SHEGMM_SHGEMM_HPP__
#define __SHEGMM_SHGEMM_HPP__
#include <cstddef>
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace mtk {
namespace shgemm {
namespace detail {
// include/shgemm/shgemm.hpp:30-34
enum kernel_level {
	P0 = 0, // Small
	P1 = 1, // Large
	num_levels
};
} // namespace detail

// include/shgemm/shgemm.hpp:36-39
enum operation_t {
	op_n,
	op_t
};

// include/shgemm/shgemm.hpp:41-44
enum tc_t {
	fp16,
	tf32
};

// include/shgemm/shgemm.hpp:46-92 (contents re-designed; copyable by value)
struct shgemmHandle_t {
	cudaStream_t cuda_stream = 0;
	unsigned debug_mode = 0;
	detail::kernel_level fixed_lernel_level = detail::num_levels;
	// Split-K workspace owned by the handle (the reference's w_ptr, src/shgemm.cu:417).
	std::size_t max_working_memory_num_elements = 0;
	float* w_ptr = nullptr;
	// Opaque shgemm_b200_handle_t.
	void* impl = nullptr;
};

// include/shgemm/shgemm.hpp:94-102
void create(shgemmHandle_t& handle);
void destroy(shgemmHandle_t& handle);

void enable_kernel_level_fixing(shgemmHandle_t& handle, const detail::kernel_level kernel_level);
void disable_kernel_level_fixing(shgemmHandle_t& handle);

void set_debug_mode(shgemmHandle_t& handle, const unsigned on);

void set_cuda_stream(shgemmHandle_t& handle, cudaStream_t const cuda_stream);

// main function (include/shgemm/shgemm.hpp:105-119)
mtk::shgemm::detail::kernel_level shgemm(
		const shgemmHandle_t handle,
		const operation_t op_a,
		const operation_t op_b,
		const std::size_t m,
		const std::size_t n,
		const std::size_t k,
		const float* const alpha_ptr,
		const float* const a_ptr, const std::size_t lda,
		const half * const b_ptr, const std::size_t ldb,
		const float* const beta_ptr,
		float* const c_ptr, const std::size_t ldc,
		const tc_t compute_type,
		const operation_t op_c = op_n
		);

// include/shgemm/shgemm.hpp:121-157: C = A B with A binary16 and B FP32, computed
// as C^T = B^T A^T so that the FP32 operand is the split one.
inline mtk::shgemm::detail::kernel_level hsgemm(
		const shgemmHandle_t handle,
		const operation_t op_a,
		const operation_t op_b,
		const std::size_t m,
		const std::size_t n,
		const std::size_t k,
		const float* const alpha_ptr,
		const half * const a_ptr, const std::size_t lda,
		const float* const b_ptr, const std::size_t ldb,
		const float* const beta_ptr,
		float* const c_ptr, const std::size_t ldc,
		const tc_t compute_type,
		const operation_t op_c = op_n
		) {
	const auto inv_op = [](const mtk::shgemm::operation_t op) {
		return op == op_n ? op_t : op_n;
	};
	return shgemm(handle, inv_op(op_b), inv_op(op_a), n, m, k, alpha_ptr, b_ptr, ldb, a_ptr, lda, beta_ptr,
			c_ptr, ldc, compute_type, inv_op(op_c));
}

// Status of the last call made through this thread (0 = success; codes of shgemm_b200.h).
int get_last_status();

} // namespace shgemm
} // namespace mtk
#endif
