// Drop-in check of the C++ API: the reference's README usage (create,
// set_cuda_stream, shgemm, hsgemm, destroy), unchanged, against an FP64 host
// product. Prints one line per call: name, level, relative Frobenius error.
#include <shgemm/shgemm.hpp>

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

static double rel_err(const std::vector<float>& c, const std::vector<double>& ref) {
	double num = 0, den = 0;
	for (size_t i = 0; i < c.size(); ++i) {
		num += (c[i] - ref[i]) * (c[i] - ref[i]);
		den += ref[i] * ref[i];
	}
	return std::sqrt(num / den);
}

int main() {
	const std::size_t m = 192, n = 160, k = 320;
	std::mt19937 gen(7);
	std::uniform_real_distribution<float> dist(-1.f, 1.f);
	std::vector<float> a(m * k), b32(k * n);
	std::vector<half> b16(k * n);
	for (auto& v : a) v = dist(gen);
	for (size_t i = 0; i < b16.size(); ++i) {
		b16[i] = __float2half(dist(gen));
		b32[i] = __half2float(b16[i]);
	}
	std::vector<double> ref(m * n, 0.0);
	for (size_t j = 0; j < n; ++j)
		for (size_t kk = 0; kk < k; ++kk)
			for (size_t i = 0; i < m; ++i) ref[i + j * m] += double(a[i + kk * m]) * double(b32[kk + j * k]);

	float *da, *dc, *db32;
	half* db16;
	cudaMalloc(&da, a.size() * 4);
	cudaMalloc(&db16, b16.size() * 2);
	cudaMalloc(&db32, b32.size() * 4);
	cudaMalloc(&dc, m * n * 4);
	cudaMemcpy(da, a.data(), a.size() * 4, cudaMemcpyHostToDevice);
	cudaMemcpy(db16, b16.data(), b16.size() * 2, cudaMemcpyHostToDevice);
	cudaMemcpy(db32, b32.data(), b32.size() * 4, cudaMemcpyHostToDevice);
	cudaStream_t stream;
	cudaStreamCreate(&stream);

	mtk::shgemm::shgemmHandle_t shgemm_handle;
	mtk::shgemm::create(shgemm_handle);
	mtk::shgemm::set_cuda_stream(shgemm_handle, stream);

	const float alpha = 1.0f, beta = 0.0f;
	int failures = 0;
	// The handle exposes its live workspace, as the reference's w_ptr does (src/shgemm.cu:417).
	{
		cudaPointerAttributes attr{};
		const bool dev_mem = shgemm_handle.w_ptr != nullptr &&
		                     cudaPointerGetAttributes(&attr, shgemm_handle.w_ptr) == cudaSuccess &&
		                     attr.type == cudaMemoryTypeDevice;
		std::printf("workspace w_ptr=%p elements=%zu device=%d\n", static_cast<void*>(shgemm_handle.w_ptr),
				shgemm_handle.max_working_memory_num_elements, dev_mem ? 1 : 0);
		failures += (!dev_mem || shgemm_handle.max_working_memory_num_elements == 0);
	}
	for (const auto compute_type : {mtk::shgemm::fp16, mtk::shgemm::tf32}) {
		// SHGEMM (A = float, B = half)
		const auto level = mtk::shgemm::shgemm(shgemm_handle, mtk::shgemm::op_n, mtk::shgemm::op_n, m, n, k, &alpha,
				da, m, db16, k, &beta, dc, m, compute_type);
		cudaStreamSynchronize(stream);
		std::vector<float> c(m * n);
		cudaMemcpy(c.data(), dc, c.size() * 4, cudaMemcpyDeviceToHost);
		const double e = rel_err(c, ref);
		std::printf("shgemm %s level=%d rel_err=%.3e status=%d\n", compute_type == mtk::shgemm::fp16 ? "fp16" : "tf32",
				static_cast<int>(level), e, mtk::shgemm::get_last_status());
		failures += (e > 1e-6 || mtk::shgemm::get_last_status() != 0);

		// HSGEMM (A = half, B = float): C^T (n x m) = B^T A^T with B^T = a^T and A^T = b32^T
		// computed as hsgemm(op_t, op_t, n, m, k, b16 (k x n), a (m x k))
		const auto level2 = mtk::shgemm::hsgemm(shgemm_handle, mtk::shgemm::op_t, mtk::shgemm::op_t, n, m, k, &alpha,
				db16, k, da, m, &beta, dc, n, compute_type);
		cudaStreamSynchronize(stream);
		cudaMemcpy(c.data(), dc, c.size() * 4, cudaMemcpyDeviceToHost);
		std::vector<float> ct(m * n);  // transpose back: dc holds C^T (n x m, ld n)
		for (size_t i = 0; i < m; ++i)
			for (size_t j = 0; j < n; ++j) ct[i + j * m] = c[j + i * n];
		const double e2 = rel_err(ct, ref);
		std::printf("hsgemm %s level=%d rel_err=%.3e status=%d\n", compute_type == mtk::shgemm::fp16 ? "fp16" : "tf32",
				static_cast<int>(level2), e2, mtk::shgemm::get_last_status());
		failures += (e2 > 1e-6 || mtk::shgemm::get_last_status() != 0);
	}
	mtk::shgemm::destroy(shgemm_handle);
	cudaStreamDestroy(stream);
	cudaFree(da);
	cudaFree(db16);
	cudaFree(db32);
	cudaFree(dc);
	std::printf("%s\n", failures ? "FAIL" : "OK");
	return failures ? 1 : 0;
}
