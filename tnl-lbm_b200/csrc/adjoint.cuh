// Discrete adjoint of the A-A step with the SRT collision and a per-site body
// force (the control), for gradients of an objective on the final state.
//
// One A-A step is a map of the population memory M_n -> M_{n+1} that is
// block-diagonal over sites: site x reads 27 locations R_q(x) and writes 27
// locations W_q(x), and {R_q(x)} = {W_q(x)} as sets (streaming_AA.h:12-116);
// locations no site touches (ghost slots nobody writes, GEO_NOTHING sites)
// map to themselves.  The adjoint step therefore has the same access pattern:
// each thread gathers the adjoint of its 27 outputs from W_q(x), applies the
// transposed Jacobian of its per-site update at the primal state M_n, and
// scatters the result to R_q(x), in place and race-free.  No linearisation
// error: the result is the exact gradient of the discrete FP update, up to
// rounding.
//
// Per-site update (GEO type from the map, bc.h:85-412) and its transpose:
//   FLUID, PERIODIC  rho = sum f, u = (sum c f + F/2) / rho (common.h:17-50),
//                    out = f + (feq - f)/tau + (1 - 1/(2 tau)) S feq with
//                    S_q = 3 (c_q - u).F / rho (col_srt.h:14-105)
//   WALL             out_q = f_opp(q) (full-way bounce-back, bc.h:201-221)
//   INFLOW           out = feq(1, u_inlet): no dependence on f or F
//   OUTFLOW_EQ       out = feq(1, u(f)) (bc.h:186-190)
//   SYM_*            mirror copy of one half of the directions (bc.h:222-293)
// With rho and u held fixed, the SRT transpose is the reference's adjoint
// collision (col_srt_adjoint.h:50-109, eq_adjoint.h:13-27): at rho = 1 and
// F = 0 both give f*_j + (sum_q f*_q w_q (feq_rho + feq_v)(q; c_j) - f*_j)/tau.
// The equilibrium is the second-order one (D3Q27_EQ, eq.h).
#pragma once

#include "aa_kernels.cuh"

namespace lbm {

// resident blocks per SM of the adjoint step (register cap 65536 / (128 n))
#ifndef ADJ_STEP_MINB
#define ADJ_STEP_MINB 4
#endif

template <typename T, typename R>
struct AdjArgs
{
	T* f;			   // primal populations (the step's input, or the state to observe)
	double* lam;	   // adjoint populations, FP64 whatever the storage, same layout (element strides) as f
	long long sq;
	int sy, sz, x0;
	int X, Y, Z;
	const uint8_t* map;	 // null: every site periodic
	const R* in_vx;		 // inlet profiles [Z][Y] (GEO_INFLOW) or null
	const R* in_vy;
	const R* in_vz;
	const double* force;  // per-site body force [3][Z][Y][X] or null (uniform p.fx..fz)
	double* grad;	  // d objective / d force, [3][Z][Y][X], accumulated
	CollParams<R> p;
};

// location of the value that direction q of a site reads (R_q) or writes
// (W_q) in the A-A step of the given parity
template <bool ODD, int q>
__device__ __forceinline__ long long aa_read_loc(long long sq, long long base, const Offsets& o)
{
	if constexpr (ODD)
		return opp(q) * sq + base + o.x[1 - cx(q)] + o.y[1 - cy(q)] + o.z[1 - cz(q)];
	else
		return q * sq + base;
}
template <bool ODD, int q>
__device__ __forceinline__ long long aa_write_loc(long long sq, long long base, const Offsets& o)
{
	if constexpr (ODD)
		return q * sq + base + o.x[1 + cx(q)] + o.y[1 + cy(q)] + o.z[1 + cz(q)];
	else
		return opp(q) * sq + base;
}

// collision constants of one site: the per-site force replaces the uniform one
template <typename T, typename R>
__device__ __forceinline__ CollParams<R> site_params(const AdjArgs<T, R>& a, long long site, long long nsites)
{
	CollParams<R> p = a.p;
	if (a.force) {
		p.fx = (R) a.force[site];
		p.fy = (R) a.force[nsites + site];
		p.fz = (R) a.force[2 * nsites + site];
		p.hfx = R(0.5) * p.fx;
		p.hfy = R(0.5) * p.fy;
		p.hfz = R(0.5) * p.fz;
	}
	return p;
}

// d feq_q(rho, u) / d u_a of the second-order equilibrium, contracted with a
// per-direction weight: adds l_q * d feq_q / d u to (bx, by, bz)
template <int q, typename R>
__device__ __forceinline__ void add_dfeq_du(R lq, R rho, R vx, R vy, R vz, R& bx, R& by, R& bz)
{
	const R cu = R(cx(q)) * vx + R(cy(q)) * vy + R(cz(q)) * vz;
	const R s = lq * R(weight(q)) * rho;
	const R g = R(3) + R(9) * cu;
	bx += s * (g * R(cx(q)) - R(3) * vx);
	by += s * (g * R(cy(q)) - R(3) * vy);
	bz += s * (g * R(cz(q)) - R(3) * vz);
}

// 8-byte asynchronous copy global -> shared (cp.async, cached in L1)
__device__ __forceinline__ void copy8_async(double* dst, const double* src)
{
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned) __cvta_generic_to_shared(dst)), "l"(src)
				 : "memory");
}

// primal moments and collision constants of one site, in FP64: the
// transpose is evaluated in FP64 at the primal's values (the FP32 primal's
// moments and constants converted exactly), so that the adjoint carries no
// FP32 rounding whatever the storage
struct AdjSite
{
	double rho, ir, vx, vy, vz;
	double fx, fy, fz;		  // the site's body force
	double inv_tau, srt_force;  // 1/tau, 1 - 1/(2 tau)
};

template <typename R>
__device__ __forceinline__ AdjSite adj_site(const Site<R>& s, const CollParams<R>& p)
{
	AdjSite m;
	m.rho = (double) s.rho;
	m.ir = s.rho == R(0) ? 1.0 : (double) s.ir;
	m.vx = (double) s.vx;
	m.vy = (double) s.vy;
	m.vz = (double) s.vz;
	m.fx = (double) p.fx;
	m.fy = (double) p.fy;
	m.fz = (double) p.fz;
	m.inv_tau = (double) p.inv_tau;
	m.srt_force = (double) p.srt_force;
	return m;
}

// transpose of the SRT update with body force at one site, in place: l <-
// J^T l, and the force gradient dF += (d out / d F)^T l
__device__ __forceinline__ void srt_vjp(const AdjSite& m, double* l, double* dF)
{
	const double rho = m.rho, ir = m.ir;
	const double vx = m.vx, vy = m.vy, vz = m.vz;
	const double usq = vx * vx + vy * vy + vz * vz;
	const double it = m.inv_tau, k = m.srt_force;
	double A = 0, bx = 0, by = 0, bz = 0, hx = 0, hy = 0, hz = 0;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			const double feq = eq_second<q>(rho, vx, vy, vz, usq);
			const double S = 3.0 * ((cx(q) - vx) * m.fx + (cy(q) - vy) * m.fy + (cz(q) - vz) * m.fz) * ir;
			const double lq = l[q];
			A += lq * feq;
			// d feq / d u weighted by (it + k S)
			add_dfeq_du<q>(lq * (it + k * S), rho, vx, vy, vz, bx, by, bz);
			// k feq dS/du = -3 k feq F / rho ; k feq dS/dF_a = 3 k feq (c_a - u_a) / rho
			const double lf = lq * feq;
			hx += lf * (cx(q) - vx);
			hy += lf * (cy(q) - vy);
			hz += lf * (cz(q) - vz);
		}
	);
	// sum_q l_q feq_q, used by the density derivative and the dS/du term
	const double sum_lf = A;
	A = it * sum_lf * ir;
	bx -= 3.0 * k * sum_lf * m.fx * ir;
	by -= 3.0 * k * sum_lf * m.fy * ir;
	bz -= 3.0 * k * sum_lf * m.fz * ir;
	const double omit = 1.0 - it;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int j = decltype(Qc)::value;
			l[j] = omit * l[j] + A + (bx * (cx(j) - vx) + by * (cy(j) - vy) + bz * (cz(j) - vz)) * ir;
		}
	);
	// d out / d F: through u (du/dF = 1 / (2 rho)) and through S directly
	const double half_ir = 0.5 * ir, three_k_ir = 3.0 * k * ir;
	dF[0] += bx * half_ir + three_k_ir * hx;
	dF[1] += by * half_ir + three_k_ir * hy;
	dF[2] += bz * half_ir + three_k_ir * hz;
}

// transpose of out = feq(1, u(f)) (GEO_OUTFLOW_EQ), in place
__device__ __forceinline__ void outflow_eq_vjp(const AdjSite& m, double* l, double* dF)
{
	const double ir = m.ir, vx = m.vx, vy = m.vy, vz = m.vz;
	double bx = 0, by = 0, bz = 0;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			add_dfeq_du<q>(l[q], 1.0, vx, vy, vz, bx, by, bz);
		}
	);
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int j = decltype(Qc)::value;
			l[j] = (bx * (cx(j) - vx) + by * (cy(j) - vy) + bz * (cz(j) - vz)) * ir;
		}
	);
	const double half_ir = 0.5 * ir;
	dF[0] += bx * half_ir;
	dF[1] += by * half_ir;
	dF[2] += bz * half_ir;
}

// transpose of the mirror copy of a symmetry plane (see symmetry(),
// aa_kernels.cuh), in place: the directions whose component along the normal
// equals `side` hand their adjoint to their mirror image (which is never one
// of them) and become zero
__device__ __forceinline__ void symmetry_vjp(double* l, int axis, int side)
{
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (cx(q) != 0) {
				constexpr int m = dir(-cx(q), cy(q), cz(q));
				if (axis == 0 && cx(q) == side) {
					l[m] += l[q];
					l[q] = 0.0;
				}
			}
			if constexpr (cy(q) != 0) {
				constexpr int m = dir(cx(q), -cy(q), cz(q));
				if (axis == 1 && cy(q) == side) {
					l[m] += l[q];
					l[q] = 0.0;
				}
			}
			if constexpr (cz(q) != 0) {
				constexpr int m = dir(cx(q), cy(q), -cz(q));
				if (axis == 2 && cz(q) == side) {
					l[m] += l[q];
					l[q] = 0.0;
				}
			}
		}
	);
}

// Primal A-A step with SRT collision and a per-site force: the per-site code
// of aa_step_kernel (GENERAL, COLL_SRT) with the site's force in place of the
// uniform one.  With a uniform force field it is the production SRT step.
template <typename S, bool ODD>
__global__ void __launch_bounds__(128) adj_primal_kernel(const AdjArgs<typename S::T, typename S::R> a)
{
	using R = typename S::R;
	const int x = blockIdx.x * blockDim.x + threadIdx.x;
	const int y = blockIdx.y, z = blockIdx.z;
	if (x >= a.X)
		return;
	const long long nsites = (long long) a.X * a.Y * a.Z;
	const long long site = ((long long) z * a.Y + y) * a.X + x;
	const uint8_t geo = a.map ? a.map[site] : (uint8_t) GEO_PERIODIC;
	if (geo == GEO_NOTHING)
		return;
	StepArgs<typename S::T, R> sa{};
	sa.Y = a.Y;
	sa.in_vx = a.in_vx;
	sa.in_vy = a.in_vy;
	sa.in_vz = a.in_vz;
	sa.p = site_params(a, site, nsites);
	const long long base = (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + x;
	const Offsets o = neighbour_offsets(geo == GEO_PERIODIC, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
	Site<R> s;
	aa_read<S, ODD>(a.f, a.sq, base, o, s.f);
	if (apply_boundary(s, geo, sa, z, y))
		collide<R, COLL_SRT, 0>(s, sa.p);
	aa_write<S, ODD>(a.f, a.sq, base, o, s.f);
}

// Adjoint of one A-A step: lam (adjoint of the step's output) is replaced in
// place by the adjoint of its input, with f the step's primal input; grad
// accumulates the force gradient of this step.  The adjoint values of a site
// are gathered from its write locations, transformed in place in FP64 and
// scattered to its read locations; the addresses are formed again for the
// scatter instead of being kept in registers across the transform.  Blocks of
// 128 threads (the shared array has one row per thread).
template <typename S, bool ODD>
__global__ void __launch_bounds__(128, ADJ_STEP_MINB) adj_step_kernel(const AdjArgs<typename S::T, typename S::R> a)
{
	using R = typename S::R;
	const int x = blockIdx.x * blockDim.x + threadIdx.x;
	const int y = blockIdx.y, z = blockIdx.z;
	if (x >= a.X)
		return;
	const long long nsites = (long long) a.X * a.Y * a.Z;
	const long long site = ((long long) z * a.Y + y) * a.X + x;
	const uint8_t geo = a.map ? a.map[site] : (uint8_t) GEO_PERIODIC;
	if (geo == GEO_NOTHING)
		return;
	const long long base = (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + x;
	// the site's 27 adjoint values live in shared memory (27 doubles per
	// thread, an odd stride: no bank conflicts beyond the two wavefronts of a
	// 64-bit access), not in registers: 54 registers fewer per thread and so
	// more resident warps for this memory-bound step
	__shared__ double lsh[128 * 27];
	double* const l = lsh + threadIdx.x * 27;
	// the primal populations of the sites whose transpose needs the moments
	// are loaded before the adjoint values, so that both sets of loads are in
	// flight together
	const bool primal = geo != GEO_WALL && geo != GEO_INFLOW && !(geo >= GEO_SYM_TOP && geo <= GEO_SYM_FRONT);
	Site<R> s;
	{
		const Offsets o = neighbour_offsets(geo == GEO_PERIODIC, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
		// the adjoint values go straight to shared memory (asynchronous copies,
		// no registers), and the primal loads are in flight with them
		static_for<27>(
			[&](auto Qc)
			{
				constexpr int q = decltype(Qc)::value;
				copy8_async(l + q, a.lam + aa_write_loc<ODD, q>(a.sq, base, o));
			}
		);
		asm volatile("cp.async.commit_group;" ::: "memory");
		if (primal)
			aa_read<S, ODD>(a.f, a.sq, base, o, s.f);
		// each thread reads only its own row of lsh: the wait makes this
		// thread's copies visible to it, no block barrier is needed
		asm volatile("cp.async.wait_group 0;" ::: "memory");
	}
	double dF[3] = {0, 0, 0};
	switch (geo) {
		case GEO_WALL:
			// full-way bounce-back swaps opposite directions: its transpose too
			static_for<13>(
				[&](auto Qc)
				{
					constexpr int q = 2 * decltype(Qc)::value + 1;
					const double t = l[q];
					l[q] = l[opp(q)];
					l[opp(q)] = t;
				}
			);
			break;
		case GEO_INFLOW:
			static_for<27>(
				[&](auto Qc)
				{
					constexpr int q = decltype(Qc)::value;
					l[q] = 0.0;
				}
			);
			break;
		case GEO_SYM_TOP:
		case GEO_SYM_BOTTOM:
		case GEO_SYM_LEFT:
		case GEO_SYM_RIGHT:
		case GEO_SYM_BACK:
		case GEO_SYM_FRONT: {
			const int axis = geo <= GEO_SYM_BOTTOM ? 2 : (geo <= GEO_SYM_RIGHT ? 0 : 1);
			const int side = (geo == GEO_SYM_TOP || geo == GEO_SYM_RIGHT || geo == GEO_SYM_FRONT) ? -1 : 1;
			symmetry_vjp(l, axis, side);
			break;
		}
		default: {	// FLUID, PERIODIC, OUTFLOW_EQ: need the primal moments
			const CollParams<R> p = site_params(a, site, nsites);
			density_velocity(s, p);
			const AdjSite m = adj_site(s, p);
			if (geo == GEO_OUTFLOW_EQ)
				outflow_eq_vjp(m, l, dF);
			else
				srt_vjp(m, l, dF);
		}
	}
	{
		const Offsets o = neighbour_offsets(geo == GEO_PERIODIC, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
		static_for<27>(
			[&](auto Qc)
			{
				constexpr int q = decltype(Qc)::value;
				a.lam[aa_read_loc<ODD, q>(a.sq, base, o)] = l[q];
			}
		);
	}
	if (a.grad && a.force && (dF[0] != 0.0 || dF[1] != 0.0 || dF[2] != 0.0)) {
		a.grad[site] += dF[0];
		a.grad[nsites + site] += dF[1];
		a.grad[2 * nsites + site] += dF[2];
	}
}

// Objective on the state f (the input of a step of the given parity):
// J = sum_i 1/2 [w_rho (rho_i - rho*_i)^2 + |u_i - u*_i|^2] at the sample
// sites, with rho and u the moments that step computes (density_velocity).
// Writes the per-sample terms to loss[i]; with lam set, adds seed * dJ/df to
// lam at the read locations and seed * dJ/dF to grad.  Sample sites are
// distinct fluid sites.
template <typename S, bool ODD>
__global__ void adj_objective_kernel(const AdjArgs<typename S::T, typename S::R> a, const long long* __restrict__ samples,
									 const double* __restrict__ target, int nsamples, double w_rho, double seed,
									 double* __restrict__ loss)
{
	using R = typename S::R;
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nsamples)
		return;
	const long long site = samples[i];
	const long long nsites = (long long) a.X * a.Y * a.Z;
	const int x = (int) (site % a.X);
	const int y = (int) ((site / a.X) % a.Y);
	const int z = (int) (site / ((long long) a.X * a.Y));
	const uint8_t geo = a.map ? a.map[site] : (uint8_t) GEO_PERIODIC;
	const CollParams<R> p = site_params(a, site, nsites);
	const long long base = (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + x;
	const Offsets o = neighbour_offsets(geo == GEO_PERIODIC, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
	Site<R> s;
	aa_read<S, ODD>(a.f, a.sq, base, o, s.f);
	density_velocity(s, p);
	const double drho = (double) s.rho - target[4 * i + 0];
	const double dvx = (double) s.vx - target[4 * i + 1];
	const double dvy = (double) s.vy - target[4 * i + 2];
	const double dvz = (double) s.vz - target[4 * i + 3];
	loss[i] = 0.5 * (w_rho * drho * drho + dvx * dvx + dvy * dvy + dvz * dvz);
	if (!a.lam)
		return;
	const double ir = (double) s.ir, vx = (double) s.vx, vy = (double) s.vy, vz = (double) s.vz;
	const double ex = seed * dvx, ey = seed * dvy, ez = seed * dvz, er = seed * w_rho * drho;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			const double d = er + (ex * (cx(q) - vx) + ey * (cy(q) - vy) + ez * (cz(q) - vz)) * ir;
			a.lam[aa_read_loc<ODD, q>(a.sq, base, o)] += d;
		}
	);
	if (a.grad && a.force) {
		const double h = 0.5 / (double) s.rho;
		a.grad[site] += seed * dvx * h;
		a.grad[nsites + site] += seed * dvy * h;
		a.grad[2 * nsites + site] += seed * dvz * h;
	}
}

}  // namespace lbm
