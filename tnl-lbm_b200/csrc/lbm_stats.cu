// Running per-site velocity statistics of D3Q27_MACRO_Mean
// (include/lbm3d/d3q27/macro.h:89-180): after every step, the mean velocity
// by the moving-average update m[n+1] = m[n] + (v - m[n]) / (n+1), and the
// co-moment S_ab[n+1] = S_ab[n] + (v_a - m_a[n+1]) (v_b - m_b[n]) of the
// Welford-type online covariance (Cov(a, b) = S_ab / (n+1)), from the macro
// field the step wrote.  Fields: stats[9][sites] = m_x, m_y, m_z, S_xx, S_yy,
// S_zz, S_xy, S_xz, S_yz in the compute type, as the reference keeps them in
// its macro array.
#include <cuda_runtime.h>

#include "launch.h"

namespace {

template <typename R>
__global__ void stats_update_kernel(const R* __restrict__ macro, R* __restrict__ st, long long n, int counter)
{
	const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const R vx = macro[n + i], vy = macro[2 * n + i], vz = macro[3 * n + i];
	const R denominator = R(1) / R(counter + 1);
	const R mx_old = st[i], my_old = st[n + i], mz_old = st[2 * n + i];
	const R dx = vx - mx_old, dy = vy - my_old, dz = vz - mz_old;
	const R mx = mx_old + dx * denominator;
	const R my = my_old + dy * denominator;
	const R mz = mz_old + dz * denominator;
	const R ex = vx - mx, ey = vy - my, ez = vz - mz;
	st[i] = mx;
	st[n + i] = my;
	st[2 * n + i] = mz;
	st[3 * n + i] += ex * dx;
	st[4 * n + i] += ey * dy;
	st[5 * n + i] += ez * dz;
	st[6 * n + i] += ex * dy;
	st[7 * n + i] += ex * dz;
	st[8 * n + i] += ey * dz;
}

}  // namespace

namespace lbm {

cudaError_t stats_update(const void* macro, void* stats, int compute_size, long long n, int counter, cudaStream_t st)
{
	const int bs = 256;
	const unsigned nb = (unsigned) ((n + bs - 1) / bs);
	if (compute_size == 8)
		stats_update_kernel<double><<<nb, bs, 0, st>>>((const double*) macro, (double*) stats, n, counter);
	else
		stats_update_kernel<float><<<nb, bs, 0, st>>>((const float*) macro, (float*) stats, n, counter);
	return cudaGetLastError();
}

}  // namespace lbm
