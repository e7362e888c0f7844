// mtk::shgemm C++ API (include/shgemm/shgemm.hpp) over the C ABI.
// Semantics of the reference's src/shgemm.cu:401-690: create binds a device and
// its workspace, set_cuda_stream/level fixing/debug mode update the handle, and
// shgemm returns the kernel level used. The reference aborts only in create
// (CUTF_CHECK_ERROR, src/shgemm.cu:361-364,424-425); here create throws on
// failure and every call's status is kept for get_last_status().
#include <shgemm/shgemm.hpp>

#include <cstdlib>
#include <stdexcept>
#include <string>

#include "shgemm_b200.h"

namespace {
thread_local int g_last_status = SHGEMM_STATUS_OK;

shgemm_b200_handle_t impl(const mtk::shgemm::shgemmHandle_t& h) {
	return static_cast<shgemm_b200_handle_t>(h.impl);
}
}  // namespace

int mtk::shgemm::get_last_status() { return g_last_status; }

void mtk::shgemm::create(mtk::shgemm::shgemmHandle_t& handle) {
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
	shgemm_b200_handle_t h = nullptr;
	const int st = shgemm_b200_create(&h, dev);
	g_last_status = st;
	if (st != SHGEMM_STATUS_OK) {
		throw std::runtime_error(std::string("mtk::shgemm::create: ") + shgemm_b200_status_string(st));
	}
	handle.impl = h;
	handle.cuda_stream = 0;
	handle.fixed_lernel_level = mtk::shgemm::detail::num_levels;
	handle.debug_mode = 0;
	const char* dbg = std::getenv("MTK_SHGEMM_DEBUG");
	if (dbg && dbg[0] == '1') handle.debug_mode = 1;
	const char* kl = std::getenv("MTK_SHGEMM_KERNEL_LEVEL");
	if (kl && (kl[0] == '0' || kl[0] == '1') && kl[1] == '\0') {
		handle.fixed_lernel_level = static_cast<mtk::shgemm::detail::kernel_level>(kl[0] - '0');
	}
	// The handle's live workspace, like the reference's cudaMalloc'd w_ptr (src/shgemm.cu:417).
	void* w = nullptr;
	std::size_t w_bytes = 0;
	if (shgemm_b200_get_workspace(h, &w, &w_bytes) != SHGEMM_STATUS_OK) w_bytes = 0;
	handle.w_ptr = w_bytes ? static_cast<float*>(w) : nullptr;
	handle.max_working_memory_num_elements = handle.w_ptr ? w_bytes / sizeof(float) : 0;
}

void mtk::shgemm::destroy(mtk::shgemm::shgemmHandle_t& handle) {
	if (handle.impl) g_last_status = shgemm_b200_destroy(impl(handle));
	handle.impl = nullptr;
}

void mtk::shgemm::set_cuda_stream(mtk::shgemm::shgemmHandle_t& handle, cudaStream_t const cuda_stream) {
	handle.cuda_stream = cuda_stream;
}

void mtk::shgemm::enable_kernel_level_fixing(mtk::shgemm::shgemmHandle_t& handle,
                                             const mtk::shgemm::detail::kernel_level kernel_level) {
	handle.fixed_lernel_level = kernel_level;
}

void mtk::shgemm::disable_kernel_level_fixing(mtk::shgemm::shgemmHandle_t& handle) {
	handle.fixed_lernel_level = mtk::shgemm::detail::num_levels;
}

void mtk::shgemm::set_debug_mode(mtk::shgemm::shgemmHandle_t& handle, const unsigned on) {
	handle.debug_mode = on;
}

mtk::shgemm::detail::kernel_level mtk::shgemm::shgemm(
		const mtk::shgemm::shgemmHandle_t handle, const mtk::shgemm::operation_t op_a,
		const mtk::shgemm::operation_t op_b, const std::size_t m, const std::size_t n, const std::size_t k,
		const float* const alpha_ptr, const float* const a_ptr, const std::size_t lda, const half* const b_ptr,
		const std::size_t ldb, const float* const beta_ptr, float* const c_ptr, const std::size_t ldc,
		const mtk::shgemm::tc_t compute_type, const mtk::shgemm::operation_t op_c) {
	shgemm_b200_handle_t h = impl(handle);
	if (!h) {
		g_last_status = SHGEMM_STATUS_INVALID_VALUE;
		return mtk::shgemm::detail::num_levels;
	}
	// The handle travels by value, as in the reference: apply its stream and
	// settings to the implementation before the call.
	shgemm_b200_set_stream(h, handle.cuda_stream);
	shgemm_b200_set_debug_mode(h, handle.debug_mode);
	shgemm_b200_set_kernel_level(h, handle.fixed_lernel_level >= mtk::shgemm::detail::num_levels
	                                    ? SHGEMM_LEVEL_AUTO
	                                    : static_cast<int>(handle.fixed_lernel_level));
	int level = SHGEMM_LEVEL_P0;
	const int st = shgemm_b200_shgemm(h, op_a == op_n ? SHGEMM_OP_N : SHGEMM_OP_T,
	                                  op_b == op_n ? SHGEMM_OP_N : SHGEMM_OP_T, m, n, k, alpha_ptr, a_ptr, lda,
	                                  b_ptr, ldb, beta_ptr, c_ptr, ldc,
	                                  compute_type == fp16 ? SHGEMM_TC_FP16 : SHGEMM_TC_TF32,
	                                  op_c == op_n ? SHGEMM_OP_N : SHGEMM_OP_T, &level);
	g_last_status = st;
	if (st != SHGEMM_STATUS_OK) return mtk::shgemm::detail::num_levels;
	return static_cast<mtk::shgemm::detail::kernel_level>(level);
}
