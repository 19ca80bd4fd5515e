// FP64 reductions of the hot path: the deterministic finish of the per-block
// partial sums written by the step kernels, and the velocity-gradient
// (enstrophy) sum over the macro field.
//
// Reference: TNL::Algorithms::reduce over dmacro in the Taylor-Green probe
// (sim_NSE/sim_4.cu:257-301) with the central-difference gradient of
// computeGradVel (sim_4.cu:21-54), and the NaN scan of
// State::AfterSimUpdate (include/lbm3d/state.hpp:1469-1492).
#include "aa_kernels.cuh"
#include "launch.h"

namespace lbm {

// Two-stage deterministic finish of the per-block partial sums, stored as
// partials[k][nblocks].  Stage 1: FINISH_BLOCKS blocks, each summing a fixed
// contiguous chunk of every quantity in a fixed order; stage 2: one block
// summing the stage-1 results.  The result does not depend on scheduling.
constexpr int FINISH_THREADS = 256;
constexpr int FINISH_BLOCKS = 296;

__device__ __forceinline__ double block_sum(double v, double* sh)
{
	sh[threadIdx.x] = v;
	__syncthreads();
	for (int s = FINISH_THREADS / 2; s > 0; s >>= 1) {
		if ((int) threadIdx.x < s)
			sh[threadIdx.x] += sh[threadIdx.x + s];
		__syncthreads();
	}
	const double r = sh[0];
	__syncthreads();
	return r;
}

__global__ void __launch_bounds__(FINISH_THREADS) finish_stage1(const double* __restrict__ partials, long long nblocks,
																double* __restrict__ stage)
{
	__shared__ double sh[FINISH_THREADS];
	const long long chunk = (nblocks + gridDim.x - 1) / gridDim.x;
	const long long b0 = blockIdx.x * chunk;
	const long long b1 = b0 + chunk < nblocks ? b0 + chunk : nblocks;
	for (int k = 0; k < NRED; k++) {
		double v = 0;
		for (long long b = b0 + threadIdx.x; b < b1; b += FINISH_THREADS)
			v += partials[k * nblocks + b];
		const double r = block_sum(v, sh);
		if (threadIdx.x == 0)
			stage[k * gridDim.x + blockIdx.x] = r;
	}
}

__global__ void __launch_bounds__(FINISH_THREADS) finish_stage2(const double* __restrict__ stage, int nstage,
																double* __restrict__ out)
{
	__shared__ double sh[FINISH_THREADS];
	for (int k = 0; k < NRED; k++) {
		double v = 0;
		for (int b = threadIdx.x; b < nstage; b += FINISH_THREADS)
			v += stage[k * nstage + b];
		const double r = block_sum(v, sh);
		if (threadIdx.x == 0)
			out[k] = r;
	}
}

long long finish_scratch_doubles()
{
	return (long long) FINISH_BLOCKS * NRED;
}

cudaError_t finish_sums(const double* partials, long long nblocks, double* stage, double* out, cudaStream_t st)
{
	finish_stage1<<<FINISH_BLOCKS, FINISH_THREADS, 0, st>>>(partials, nblocks, stage);
	finish_stage2<<<1, FINISH_THREADS, 0, st>>>(stage, FINISH_BLOCKS, out);
	return cudaGetLastError();
}

// rho * |grad u|^2 per site with periodic central differences
// (sim_4.cu:21-54, :279-298); partial sums per block in slot 0, the other
// slots hold zero so that finish_sums can be reused
template <typename R>
__global__ void enstrophy_kernel(const R* __restrict__ m, int X, int Y, int Z, double* __restrict__ partials)
{
	const int x = blockIdx.x * blockDim.x + threadIdx.x;
	const int y = blockIdx.y;
	const int z = blockIdx.z;
	double red[NRED] = {0, 0, 0, 0, 0, 0};
	if (x < X) {
		const long long n = (long long) X * Y * Z;
		auto at = [&](int c, int xx, int yy, int zz) -> double
		{
			return (double) m[c * n + ((long long) zz * Y + yy) * X + xx];
		};
		const int xp = x == X - 1 ? 0 : x + 1, xm = x == 0 ? X - 1 : x - 1;
		const int yp = y == Y - 1 ? 0 : y + 1, ym = y == 0 ? Y - 1 : y - 1;
		const int zp = z == Z - 1 ? 0 : z + 1, zm = z == 0 ? Z - 1 : z - 1;
		double g2 = 0;
		for (int c = 1; c <= 3; c++) {
			const double gx = 0.5 * (at(c, xp, y, z) - at(c, xm, y, z));
			const double gy = 0.5 * (at(c, x, yp, z) - at(c, x, ym, z));
			const double gz = 0.5 * (at(c, x, y, zp) - at(c, x, y, zm));
			g2 += gx * gx + gy * gy + gz * gz;
		}
		red[0] = at(0, x, y, z) * g2;
	}
	block_reduce_store<R>(red, partials);
}

cudaError_t enstrophy_partials(const void* macro, int compute_size, int X, int Y, int Z, double* partials, long long* nblocks,
							   cudaStream_t st)
{
	const int bx = 128;
	dim3 grid((X + bx - 1) / bx, Y, Z);
	*nblocks = (long long) grid.x * grid.y * grid.z;
	if (compute_size == 8)
		enstrophy_kernel<double><<<grid, bx, 0, st>>>((const double*) macro, X, Y, Z, partials);
	else
		enstrophy_kernel<float><<<grid, bx, 0, st>>>((const float*) macro, X, Y, Z, partials);
	return cudaGetLastError();
}

}  // namespace lbm
