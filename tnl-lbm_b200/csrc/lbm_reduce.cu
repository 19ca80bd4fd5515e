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

// Deterministic finish of the partial sums, stored as partials[k][nslots], in
// one launch.  FINISH_BLOCKS blocks each sum a fixed contiguous chunk of every
// quantity in a fixed order and store the block results in stage; the block
// that arrives last on the arrival counter sums the stage in a fixed order,
// writes out[NRED] (device or mapped host memory) and resets the counter for
// the next launch.  The result does not depend on scheduling.
constexpr int FINISH_THREADS = 256;
constexpr int FINISH_BLOCKS = 296;
constexpr int FINISH_WARPS = FINISH_THREADS / 32;

// sums of NRED values over the block, valid in thread 0
__device__ __forceinline__ void block_sums(double (&v)[NRED], double (*sh)[NRED])
{
#pragma unroll
	for (int k = 0; k < NRED; k++)
#pragma unroll
		for (int off = 16; off > 0; off >>= 1)
			v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (lane == 0)
#pragma unroll
		for (int k = 0; k < NRED; k++)
			sh[warp][k] = v[k];
	__syncthreads();
	if (threadIdx.x == 0)
#pragma unroll
		for (int k = 0; k < NRED; k++) {
			double acc = 0;
			for (int w = 0; w < FINISH_WARPS; w++)
				acc += sh[w][k];
			v[k] = acc;
		}
}

__global__ void __launch_bounds__(FINISH_THREADS) finish_kernel(const double* __restrict__ partials, long long nslots,
																double* __restrict__ stage, unsigned* __restrict__ arrived,
																double* __restrict__ out, double mass_offset)
{
	__shared__ double sh[FINISH_WARPS][NRED];
	__shared__ bool last;
	// launched as a programmatic dependent of the step that wrote the
	// partials: wait until that grid has completed and its writes are visible
	asm volatile("griddepcontrol.wait;" ::: "memory");
	const long long chunk = (nslots + gridDim.x - 1) / gridDim.x;
	const long long b0 = blockIdx.x * chunk;
	const long long b1 = b0 + chunk < nslots ? b0 + chunk : nslots;
	// the quantities innermost: the NRED loads of a slot go out together (the
	// order of each quantity's additions is unchanged)
	double v[NRED] = {0, 0, 0, 0, 0, 0};
	for (long long b = b0 + threadIdx.x; b < b1; b += FINISH_THREADS)
#pragma unroll
		for (int k = 0; k < NRED; k++)
			v[k] += __ldcs(partials + k * nslots + b);
	block_sums(v, sh);
	if (threadIdx.x == 0) {
#pragma unroll
		for (int k = 0; k < NRED; k++)
			stage[k * FINISH_BLOCKS + blockIdx.x] = v[k];
		__threadfence();
		last = atomicAdd(arrived, 1u) == gridDim.x - 1;
	}
	__syncthreads();
	if (!last)
		return;
	__threadfence();
	__syncthreads();  // sh is reused
#pragma unroll
	for (int k = 0; k < NRED; k++)
		v[k] = 0;
	for (int b = threadIdx.x; b < (int) gridDim.x; b += FINISH_THREADS)
#pragma unroll
		for (int k = 0; k < NRED; k++)
			v[k] += __ldcg(stage + k * FINISH_BLOCKS + b);
	block_sums(v, sh);
	if (threadIdx.x == 0) {
		v[0] += mass_offset;
#pragma unroll
		for (int k = 0; k < NRED; k++)
			out[k] = v[k];
		*arrived = 0;
		__threadfence_system();
	}
}

long long finish_scratch_doubles()
{
	return (long long) FINISH_BLOCKS * NRED;
}

cudaError_t finish_sums(const double* partials, long long nslots, double* stage, unsigned* arrived, double* out, cudaStream_t st,
						double mass_offset)
{
	// programmatic dependent launch: where the finish follows the kernel that
	// wrote the partials on the same stream, its grid is scheduled while that
	// kernel's last blocks run (the observation step kernels trigger it when
	// they start) and waits in griddepcontrol.wait; after a wait on another
	// stream's event (the sums of lbm_step, on the finish stream) it starts as
	// an ordinary launch
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(FINISH_BLOCKS);
	cfg.blockDim = dim3(FINISH_THREADS);
	cfg.dynamicSmemBytes = 0;
	cfg.stream = st;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, finish_kernel, partials, nslots, stage, arrived, out, mass_offset);
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
