// A-B pull step (streaming_AB.h:12-58): every site reads direction q from site
// x - c_q of the input buffer, applies the boundary condition and the
// collision, and writes its 27 post-collision values to its own site of the
// output buffer; the host swaps the buffers after every step
// (lbm.hpp:314-322).
//
// Reading only the previous step's buffer makes every site type of
// D3Q27_BC_All free of cross-site ordering, so this step also provides the
// types the in-place A-A step cannot: GEO_INFLOW_BB_LEFT (bc.h:143-165),
// GEO_OUTFLOW_RIGHT (bc.h:73-74, 191-194) and GEO_OUTFLOW_RIGHT_INTERP
// (bc.h:195-200 with streamingInterpRight, streaming_AB.h:209-242).
// Neighbour indices follow kernelInitIndices of a single block
// (kernels.h:21-28, 48-55): periodic sites wrap, other sites clamp to the
// lattice (there is no ghost layer in the A-B scheme).
#pragma once

#include "aa_kernels.cuh"

namespace lbm {

// neighbour offsets of the A-B step (kernels.h:5-57 without AA_PATTERN)
__device__ __forceinline__ Offsets ab_offsets(uint8_t geo, int x, int y, int z, int X, int Y, int Z, int sy, int sz)
{
	if (geo == GEO_PERIODIC)
		return neighbour_offsets(true, x, y, z, X, Y, Z, sy, sz);
	Offsets o;
	o.x[0] = x == 0 ? 0 : -1;
	o.x[1] = 0;
	o.x[2] = x == X - 1 ? 0 : 1;
	o.y[0] = y == 0 ? 0 : -(long long) sy;
	o.y[1] = 0;
	o.y[2] = y == Y - 1 ? 0 : (long long) sy;
	o.z[0] = z == 0 ? 0 : -(long long) sz;
	o.z[1] = 0;
	o.z[2] = z == Z - 1 ? 0 : (long long) sz;
	if (geo == GEO_OUTFLOW_RIGHT)  // pull from x - 1 in every direction (bc.h:73-74)
		o.x[1] = o.x[2] = o.x[0];
	return o;
}

// pull streaming (streaming_AB.h:22-49)
template <typename S>
__device__ __forceinline__ void ab_read(const typename S::T* __restrict__ f, long long sq, long long base, const Offsets& o,
										typename S::R* v)
{
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			v[q] = S::template load<q>(f + q * sq + base + o.x[1 - cx(q)] + o.y[1 - cy(q)] + o.z[1 - cz(q)]);
		}
	);
}

// streaming of an interpolated right outlet (streaming_AB.h:209-242): the
// directions that leave through x = X-1 backwards (c_x = -1) are taken as a
// blend of sites x - 1 and x weighted by the lattice speed of sound
template <typename S>
__device__ __forceinline__ void ab_read_interp(const typename S::T* __restrict__ f, long long sq, long long base,
											   const Offsets& o, typename S::R* v)
{
	using R = typename S::R;
	const R cs = R(0.5773502691896257);
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			const typename S::T* p = f + q * sq + base + o.y[1 - cy(q)] + o.z[1 - cz(q)];
			if constexpr (cx(q) == -1)
				v[q] = cs * S::template load<q>(p + o.x[0]) + (R(1) - cs) * S::template load<q>(p);
			else
				v[q] = S::template load<q>(p + o.x[1 - cx(q)]);
		}
	);
}

// pre-collision part of the A-B step for one site (bc.h:60-403); returns
// whether the site collides (bc.h:406-412)
template <typename S, typename R, typename T>
__device__ __forceinline__ bool ab_boundary(Site<R>& s, uint8_t geo, const StepArgs<T, R>& a, long long base, int z, int y)
{
	switch (geo) {
		case GEO_INFLOW_BB_LEFT: {
			// bounce-back of the site's own outgoing populations with the inlet
			// velocity (kernel-struct density rho = 1)
			const long long prof = (long long) z * a.Y + y;
			s.vx = a.in_vx ? a.in_vx[prof] : R(0);
			s.vy = a.in_vy ? a.in_vy[prof] : R(0);
			s.vz = a.in_vz ? a.in_vz[prof] : R(0);
			static_for<27>(
				[&](auto Qc)
				{
					constexpr int q = decltype(Qc)::value;
					if constexpr (cx(q) == 1) {
						constexpr int m = opp(q);
						const R cmu = R(cx(m)) * s.vx + R(cy(m)) * s.vy + R(cz(m)) * s.vz;
						s.f[q] = S::template load<m>(a.f + m * a.sq + base) - R(2) * R(weight(q)) * R(1) * R(3) * cmu;
					}
				}
			);
			density_velocity(s, a.p);
			return true;
		}
		case GEO_OUTFLOW_RIGHT:
			density_velocity(s, a.p);
			s.rho = R(1);
			s.ir = R(1);
			return true;
		case GEO_OUTFLOW_RIGHT_INTERP: {
			density_velocity(s, a.p);
			// setEquilibriumDecomposition(KS, 1) (common.h:95-124)
			R e1[27], er[27];
			set_equilibrium(e1, a.p.eq, R(1), s.vx, s.vy, s.vz);
			set_equilibrium(er, a.p.eq, s.rho, s.vx, s.vy, s.vz);
#pragma unroll
			for (int q = 0; q < 27; q++)
				s.f[q] += e1[q] - er[q];
			s.rho = R(1);
			s.ir = R(1);
			return true;
		}
		default:
			return apply_boundary(s, geo, a, z, y);
	}
}

template <typename S, int COLL, int CUMF, bool OUT, int MINB>
__global__ void __launch_bounds__(128, MINB)
	ab_step_kernel(const StepArgs<typename S::T, typename S::R> a, typename S::T* __restrict__ fout)
{
	using R = typename S::R;
	const int x = blockIdx.x * blockDim.x + threadIdx.x;
	const int y = blockIdx.y * blockDim.y + threadIdx.y;
	const int z = blockIdx.z;
	const bool active = x < a.X && y < a.Y;
	Site<R> s;
	long long base = 0, site = 0;
	bool coll = false, write = false;
	if (active) {
		base = (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + x;
		site = ((long long) z * a.Y + y) * a.X + x;
		const uint8_t geo = a.map ? a.map[site] : (uint8_t) GEO_PERIODIC;
		if (geo == GEO_NOTHING) {
			s.rho = R(1);
			s.vx = s.vy = s.vz = R(0);
		}
		else {
			const Offsets o = ab_offsets(geo, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
			if (geo == GEO_OUTFLOW_RIGHT_INTERP)
				ab_read_interp<S>(a.f, a.sq, base, o, s.f);
			else
				ab_read<S>(a.f, a.sq, base, o, s.f);
			coll = ab_boundary<S>(s, geo, a, base, z, y);
			write = true;
		}
	}
	if constexpr (OUT)
		step_outputs(a, active, site, s);
	if (write) {
		if (coll)
			collide<R, COLL, CUMF>(s, a.p);
		static_for<27>(
			[&](auto Qc)
			{
				constexpr int q = decltype(Qc)::value;
				S::template store<q>(fout + q * a.sq + base, s.f[q]);
			}
		);
	}
}

}  // namespace lbm
