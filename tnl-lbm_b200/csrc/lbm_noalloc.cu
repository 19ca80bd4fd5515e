// Allocation-free sums of a macro field (declared in include/tnl_lbm_b200.h as
// lbm_macro_sums_noalloc).
//
// Why it exists: some callers cannot allocate device memory at the point where
// they want the sums.  A host application that has handed the whole device to
// its own pool allocator forbids stray allocations from libraries, and a
// real-time loop cannot afford the implicit synchronisation an allocation can
// bring.  The
// regular path (lbm_step with LBM_STEP_SUMS) keeps its per-block partial sums
// in a buffer the handle allocates.  This entry point does the same reduction
// with its scratch in a file-scope device array instead, so a call allocates
// nothing: the caller passes the macro field and a device buffer for the six
// results, both already allocated.
//
// Scratch: g_sums_scratch, LBM_NOALLOC_SCRATCH_DOUBLES doubles (96 KiB) per
// GPU that loads this library, held until the process exits.  It holds the
// partial sums of at most LBM_NOALLOC_MAX_BLOCKS blocks; the reduction uses a
// fixed grid of that many blocks with a grid-stride loop, so the lattice size
// is bounded only by LBM_NOALLOC_MAX_SITES.  Every block writes all of its
// partials before the finishing block reads them, so nothing has to be
// cleared between calls.  Each GPU has its own copy of the array, so calls on
// different devices may overlap; all calls on one device share its copy, and
// calls whose kernels overlap on that GPU (different streams, or several host
// threads) race on it and must be serialised by the caller.  The device
// address is resolved once per device and kept for the life of the process:
// after cudaDeviceReset the module is reloaded and the array may move, so the
// entry point must not be used across a device reset.
#include <cstdint>
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/tnl_lbm_b200.h"

namespace {

constexpr int SUMS = 6;	 // sum rho, rho*vx, rho*vy, rho*vz, rho*|u|^2, non-finite count
constexpr int THREADS = 256;

static_assert(LBM_NOALLOC_SCRATCH_DOUBLES == SUMS * LBM_NOALLOC_MAX_BLOCKS, "scratch size");

// the scratch the reduction kernels use; host code only ever passes the device
// address obtained from cudaGetSymbolAddress, never the symbol itself
static __device__ __align__(256) double g_sums_scratch[LBM_NOALLOC_SCRATCH_DOUBLES];

// per-device address of g_sums_scratch, resolved on the first call on a device
double* g_scratch_addr[64] = {nullptr};
std::mutex g_setup_mutex;

__device__ __forceinline__ double block_sum(double v, double* sh)
{
	sh[threadIdx.x] = v;
	__syncthreads();
	for (int s = THREADS / 2; s > 0; s >>= 1) {
		if ((int) threadIdx.x < s)
			sh[threadIdx.x] += sh[threadIdx.x + s];
		__syncthreads();
	}
	const double r = sh[0];
	__syncthreads();
	return r;
}

// per-block partial sums of the macro field m = [4][n] (rho, vx, vy, vz);
// partials[k * gridDim.x + blockIdx.x]
template <typename R>
__global__ void __launch_bounds__(THREADS) macro_partials(const R* __restrict__ m, long long n, double* __restrict__ partials)
{
	__shared__ double sh[THREADS];
	double v[SUMS] = {0, 0, 0, 0, 0, 0};
	for (long long i = blockIdx.x * (long long) THREADS + threadIdx.x; i < n; i += (long long) gridDim.x * THREADS) {
		const double rho = (double) m[i], vx = (double) m[n + i], vy = (double) m[2 * n + i], vz = (double) m[3 * n + i];
		v[0] += rho;
		v[1] += rho * vx;
		v[2] += rho * vy;
		v[3] += rho * vz;
		v[4] += rho * (vx * vx + vy * vy + vz * vz);
		v[5] += isfinite(rho) ? 0.0 : 1.0;
	}
	for (int k = 0; k < SUMS; k++) {
		const double r = block_sum(v[k], sh);
		if (threadIdx.x == 0)
			partials[k * gridDim.x + blockIdx.x] = r;
	}
}

// one block: fixed-order sum of the partials of nblocks blocks into out[6]
__global__ void __launch_bounds__(THREADS) finish_partials(const double* __restrict__ partials, int nblocks, double* __restrict__ out)
{
	__shared__ double sh[THREADS];
	for (int k = 0; k < SUMS; k++) {
		double v = 0;
		for (int b = threadIdx.x; b < nblocks; b += THREADS)
			v += partials[k * nblocks + b];
		const double r = block_sum(v, sh);
		if (threadIdx.x == 0)
			out[k] = r;
	}
}

}  // namespace

namespace lbm {
// records the message returned by lbm_last_error() (lbm_abi.cu)
int record_error(int code, const char* msg);
}  // namespace lbm

namespace {
int reject(int code, const char* fmt, long long a = 0, long long b = 0)
{
	char msg[256];
	snprintf(msg, sizeof(msg), fmt, a, b);
	return lbm::record_error(code, msg);
}
}  // namespace

extern "C" {

LBM_API int lbm_macro_sums_noalloc(const void* macro, int dtype, int64_t nsites, double* out, void* stream)
{
	if (!macro || !out)
		return reject(LBM_ERR_INVALID, "lbm_macro_sums_noalloc: null macro field or output pointer");
	if (dtype != LBM_DTYPE_F64 && dtype != LBM_DTYPE_F32)
		return reject(LBM_ERR_INVALID, "lbm_macro_sums_noalloc: dtype %lld, expected LBM_DTYPE_F64 or LBM_DTYPE_F32", dtype);
	if (nsites <= 0)
		return reject(LBM_ERR_INVALID, "lbm_macro_sums_noalloc: nsites must be positive (got %lld)", (long long) nsites);
	if (nsites > LBM_NOALLOC_MAX_SITES)
		return reject(LBM_ERR_SIZE, "lbm_macro_sums_noalloc: %lld sites exceed the maximum of %lld", (long long) nsites,
					  (long long) LBM_NOALLOC_MAX_SITES);
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
		return reject(LBM_ERR_CUDA, "lbm_macro_sums_noalloc: no usable current CUDA device");
	// set-up, once per device with that device current: the device address of
	// the scratch array, and the three reduction kernels loaded together with
	// it (with lazy module loading, the CUDA 12 default, a kernel is otherwise
	// loaded at its first launch, which could fall into a later capture)
	double* scratch = nullptr;
	{
		std::lock_guard<std::mutex> lock(g_setup_mutex);
		if (!g_scratch_addr[dev]) {
			void* ptr = nullptr;
			cudaError_t e = cudaGetSymbolAddress(&ptr, g_sums_scratch);
			if (e != cudaSuccess || !ptr)
				return reject(LBM_ERR_CUDA, "lbm_macro_sums_noalloc: cudaGetSymbolAddress of the scratch array failed (error %lld)",
							  (long long) e);
			cudaFuncAttributes attr;
			const void* kernels[3] = {(const void*) macro_partials<double>, (const void*) macro_partials<float>,
									  (const void*) finish_partials};
			for (const void* k : kernels) {
				e = cudaFuncGetAttributes(&attr, k);
				if (e != cudaSuccess)
					return reject(LBM_ERR_CUDA, "lbm_macro_sums_noalloc: loading the reduction kernels failed (error %lld)",
								  (long long) e);
			}
			g_scratch_addr[dev] = (double*) ptr;
		}
		scratch = g_scratch_addr[dev];
	}
	long long blocks = (nsites + THREADS - 1) / THREADS;
	if (blocks > LBM_NOALLOC_MAX_BLOCKS)
		blocks = LBM_NOALLOC_MAX_BLOCKS;
	cudaStream_t st = (cudaStream_t) stream;
	if (dtype == LBM_DTYPE_F64)
		macro_partials<double><<<(unsigned) blocks, THREADS, 0, st>>>((const double*) macro, nsites, scratch);
	else
		macro_partials<float><<<(unsigned) blocks, THREADS, 0, st>>>((const float*) macro, nsites, scratch);
	finish_partials<<<1, THREADS, 0, st>>>(scratch, (int) blocks, out);
	const cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess)
		return reject(LBM_ERR_CUDA, "lbm_macro_sums_noalloc: reduction launch failed (error %lld)", (long long) e);
	return LBM_OK;
}

}  // extern "C"
