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

// one block; each thread accumulates a strided subset of the partials in a
// fixed order, then a fixed tree combines them, so the result does not depend
// on scheduling
__global__ void finish_sums_kernel(const double* __restrict__ partials, long long nblocks, double* __restrict__ out)
{
	__shared__ double acc[256][NRED];
	double v[NRED] = {0, 0, 0, 0, 0, 0};
	for (long long b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
		for (int k = 0; k < NRED; k++)
			v[k] += partials[b * NRED + k];
#pragma unroll
	for (int k = 0; k < NRED; k++)
		acc[threadIdx.x][k] = v[k];
	__syncthreads();
	for (int s = blockDim.x / 2; s > 0; s >>= 1) {
		if ((int) threadIdx.x < s)
#pragma unroll
			for (int k = 0; k < NRED; k++)
				acc[threadIdx.x][k] += acc[threadIdx.x + s][k];
		__syncthreads();
	}
	if (threadIdx.x < NRED)
		out[threadIdx.x] = acc[0][threadIdx.x];
}

cudaError_t finish_sums(const double* partials, long long nblocks, double* out, cudaStream_t st)
{
	finish_sums_kernel<<<1, 256, 0, st>>>(partials, nblocks, out);
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
