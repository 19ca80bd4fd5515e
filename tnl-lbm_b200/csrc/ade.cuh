// D3Q7 advection-diffusion (ADE) coupled to the D3Q27 flow step.
//
// The reference's coupled kernel (include/lbm3d/kernels.h:114-196) updates, in
// one pass per site, the flow populations and then the scalar's seven
// populations, advected with the site's flow velocity (the velocity after the
// flow boundary treatment, which the collision leaves unchanged).  Here the same
// fusion is one kernel (ade_step_kernel): the flow part is the direct step's
// per-site code, the scalar part reads and writes its seven populations with the
// same A-A pattern and the same neighbour offsets, so a site's registers of the
// flow update are dead before the scalar needs its own.
//
// Scalar populations are stored in the compute type, seven slot rows per
// lattice row with the flow lattice's row pitch and x offset; the coupling is
// offered for the FP64 and FP32 storage formats, whose element is the compute
// type's size.
//
// Operators (include/lbm3d/d3q7/): equilibrium eq.h:17-54 (c_s^2 = 1/4,
// w_0 = 1/4, w_q = 1/8), collisions col_srt.h, col_mrt.h, col_clbm.h with
// omega = 1 / (1/2 + 4 D), D the diffusion coefficient of the site
// (lbm_data.h:231-239), boundary conditions bc.h:66-211.  Site types whose A-A
// update reads a slot that another site writes in the same pass
// (GEO_OUTFLOW_RIGHT, GEO_OUTFLOW_PE, which pull from x - 1 and x - 2) and the
// phase-transfer types (GEO_TRANSFER_*, which need the transfer direction
// arrays and read neighbour slots) are rejected by lbm_ade_set_map.
#pragma once

#include "aa_kernels.cuh"

namespace lbm {

// ADE site types of D3Q7_BC_All (include/lbm3d/d3q7/bc.h:17-36)
enum AdeGeo : uint8_t
{
	ADE_FLUID = 0,
	ADE_WALL = 1,
	ADE_WALL_BODY = 2,
	ADE_SOLID = 3,
	ADE_TRANSFER_FS = 4,
	ADE_TRANSFER_SF = 5,
	ADE_TRANSFER_SW = 6,
	ADE_INFLOW = 7,
	ADE_OUTFLOW_RIGHT = 8,
	ADE_PERIODIC = 9,
	ADE_NOTHING = 10,
	ADE_OUTFLOW_PE = 11,
	ADE_SYM_TOP = 12,
	ADE_SYM_BOTTOM = 13,
	ADE_SYM_LEFT = 14,
	ADE_SYM_RIGHT = 15,
	ADE_SYM_BACK = 16,
	ADE_SYM_FRONT = 17
};

__host__ __device__ constexpr bool ade_type_supported(uint8_t g)
{
	return g <= ADE_SOLID || g == ADE_INFLOW || g == ADE_PERIODIC || g == ADE_NOTHING || (g >= ADE_SYM_TOP && g <= ADE_SYM_FRONT);
}

enum AdeColl : int
{
	ADE_SRT = 0,
	ADE_MRT = 1,
	ADE_CLBM = 2
};

template <typename R>
struct AdeArgs
{
	R* g;				  // scalar populations, slot q of site (x, y, z) at
						  // q * sq + (z + 1) * sz + (y + 1) * sy + x0 + x
	long long sq;
	int sy, sz;
	const uint8_t* map;	  // ADE site types [Z][Y][X]
	const R* dcoef;		  // per-site diffusion coefficient [Z][Y][X], or null
	R D;				  // diffusion coefficient when dcoef is null
	R inflow_phi;		  // phi of GEO_INFLOW sites (ADE_Data_ConstInflow, lbm_data.h:248-262)
	R* phi;				  // macro output [Z][Y][X] of observation steps, or null
	int coll;			  // AdeColl
};

// second-order equilibrium of direction Q (eq.h:17-25, 27-53)
template <int Q, typename R>
__device__ __forceinline__ R ade_feq(R phi, R vx, R vy, R vz)
{
	const R w = Q == 0 ? R(0.25) : R(0.125);
	const R cu = R(cx(Q)) * vx + R(cy(Q)) * vy + R(cz(Q)) * vz;
	return w * phi * (R(1) - R(2) * (vx * vx + vy * vy + vz * vz) + R(4) * cu + R(8) * cu * cu);
}

template <typename R>
__device__ __forceinline__ R ade_phi(const R (&g)[7])
{
	R phi = 0;
#pragma unroll
	for (int q = 0; q < 7; q++)
		phi += g[q];
	return phi;
}

template <typename R>
__device__ __forceinline__ void ade_equilibrium(R (&g)[7], R phi, R vx, R vy, R vz)
{
	static_for<7>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			g[q] = ade_feq<q>(phi, vx, vy, vz);
		}
	);
}

// collisions: col_srt.h:12-25, col_mrt.h:12-49, col_clbm.h:14-83 (the
// higher-order relaxation rates of the central-moment variant are 1)
template <typename R>
__device__ __forceinline__ void ade_collide(R (&g)[7], R phi, R vx, R vy, R vz, R D, int coll)
{
	const R omega = R(1) / (R(0.5) + R(4) * D);
	if (coll == ADE_SRT) {
		static_for<7>(
			[&](auto Qc)
			{
				constexpr int q = decltype(Qc)::value;
				g[q] += omega * (ade_feq<q>(phi, vx, vy, vz) - g[q]);
			}
		);
		return;
	}
	const R cs2 = R(0.25);
	R m100, m010, m001, m200, m020, m002;
	if (coll == ADE_MRT) {
		m100 = phi * vx + g[2] - g[1];
		m010 = phi * vy + g[4] - g[3];
		m001 = phi * vz + g[6] - g[5];
		m200 = phi * (vx * vx + cs2) - g[2] - g[1];
		m020 = phi * (vy * vy + cs2) - g[4] - g[3];
		m002 = phi * (vz * vz + cs2) - g[6] - g[5];
	}
	else {	// central moments
		m100 = phi * vx + g[2] - g[1];
		m010 = phi * vy + g[4] - g[3];
		m001 = phi * vz + g[6] - g[5];
		m200 = phi * (cs2 - vx * vx) + R(2) * vx * (g[1] - g[2]) - g[2] - g[1];
		m020 = phi * (cs2 - vy * vy) + R(2) * vy * (g[3] - g[4]) - g[4] - g[3];
		m002 = phi * (cs2 - vz * vz) + R(2) * vz * (g[5] - g[6]) - g[6] - g[5];
	}
	m100 *= omega;
	m010 *= omega;
	m001 *= omega;
	if (coll == ADE_MRT) {
		g[0] += -m200 - m020 - m002;
		g[1] += R(0.5) * (m200 + m100);
		g[3] += R(0.5) * (m020 + m010);
		g[5] += R(0.5) * (m002 + m001);
		g[2] += R(0.5) * (m200 - m100);
		g[4] += R(0.5) * (m020 - m010);
		g[6] += R(0.5) * (m002 - m001);
	}
	else {
		g[0] += -R(2) * (m100 * vx + m010 * vy + m001 * vz) - m200 - m020 - m002;
		g[1] += m100 * vx + R(0.5) * (m200 + m100);
		g[3] += m010 * vy + R(0.5) * (m020 + m010);
		g[5] += m001 * vz + R(0.5) * (m002 + m001);
		g[2] += m100 * vx + R(0.5) * (m200 - m100);
		g[4] += m010 * vy + R(0.5) * (m020 - m010);
		g[6] += m001 * vz + R(0.5) * (m002 - m001);
	}
}

// pre-collision part of D3Q7_BC_All (bc.h:66-193) for the supported types
// (after the read); returns whether the site collides (bc.h:196-201)
template <typename R>
__device__ __forceinline__ bool ade_boundary(R (&g)[7], R& phi, uint8_t geo, R vx, R vy, R vz, R inflow_phi)
{
	switch (geo) {
		case ADE_INFLOW:
			phi = inflow_phi;
			ade_equilibrium(g, phi, vx, vy, vz);
			return false;
		case ADE_WALL:
		case ADE_WALL_BODY: {
			phi = ade_phi(g);
			R t = g[2];
			g[2] = g[1];
			g[1] = t;
			t = g[4];
			g[4] = g[3];
			g[3] = t;
			t = g[6];
			g[6] = g[5];
			g[5] = t;
			if (geo == ADE_WALL_BODY) {
				g[0] = -g[0] + R(2) * R(0.25) * phi;
#pragma unroll
				for (int q = 1; q < 7; q++)
					g[q] = -g[q] + R(2) * R(0.125) * phi;
			}
			return false;
		}
		case ADE_SYM_TOP:
			g[6] = g[5];
			phi = ade_phi(g);
			return false;
		case ADE_SYM_BOTTOM:
			g[5] = g[6];
			phi = ade_phi(g);
			return false;
		case ADE_SYM_LEFT:
			g[1] = g[2];
			phi = ade_phi(g);
			return false;
		case ADE_SYM_RIGHT:
			g[2] = g[1];
			phi = ade_phi(g);
			return false;
		case ADE_SYM_BACK:
			g[3] = g[4];
			phi = ade_phi(g);
			return false;
		case ADE_SYM_FRONT:
			g[4] = g[3];
			phi = ade_phi(g);
			return false;
		default:  // FLUID, SOLID, PERIODIC
			phi = ade_phi(g);
			return true;
	}
}

// A-A read / write of the seven scalar populations (d3q7/streaming_AA.h),
// the first seven directions of the D3Q27 order
template <bool ODD, typename R>
__device__ __forceinline__ void ade_read(const R* __restrict__ g, long long sq, long long base, const Offsets& o, R (&v)[7])
{
	static_for<7>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (ODD)
				v[q] = g[opp(q) * sq + base + o.x[1 - cx(q)] + o.y[1 - cy(q)] + o.z[1 - cz(q)]];
			else
				v[q] = g[q * sq + base];
		}
	);
}

template <bool ODD, typename R>
__device__ __forceinline__ void ade_write(R* __restrict__ g, long long sq, long long base, const Offsets& o, const R (&v)[7])
{
	static_for<7>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (ODD)
				g[q * sq + base + o.x[1 + cx(q)] + o.y[1 + cy(q)] + o.z[1 + cz(q)]] = v[q];
			else
				g[opp(q) * sq + base] = v[q];
		}
	);
}

#ifndef ADE_EARLY_READ
#define ADE_EARLY_READ 1
#endif

// Coupled update of site (x, y, z): the direct kernel's flow update, then the
// scalar's.  OUT: every thread of the warp calls it (outputs are warp-wide).
template <typename S, int COLL, int CUMF, bool ODD, bool GENERAL, bool OUT>
__device__ __forceinline__ void ade_site_update(const StepArgs<typename S::T, typename S::R>& a, const AdeArgs<typename S::R>& d,
												int x, int y, int z)
{
	using R = typename S::R;
	const bool active = x < a.X && y < a.Y;

	Site<R> s;
	Offsets o;
	long long base = 0, site = 0;
	bool coll = false, write = false;
	uint8_t ag = ADE_NOTHING;
	R g[7];
	if (active) {
		base = (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + x;
		site = ((long long) z * a.Y + y) * a.X + x;
		uint8_t geo = GEO_PERIODIC;
		if constexpr (GENERAL)
			geo = a.map[site];
		// the scalar uses the flow site's neighbour indices (kernels.h:155-156)
		const bool wrap = !GENERAL || geo == GEO_PERIODIC;
		o = neighbour_offsets(wrap, wrap && a.zwrap, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
#if ADE_EARLY_READ
		// the scalar's loads go out together with the flow's, so that both are
		// in flight at once
		ag = d.map[site];
		if (ag != ADE_NOTHING) {
			const bool w = !GENERAL || geo == GEO_PERIODIC;
			const Offsets od = neighbour_offsets(w, w && a.zwrap, x, y, z, a.X, a.Y, a.Z, d.sy, d.sz);
			ade_read<ODD>(d.g, d.sq, (long long) (z + 1) * d.sz + (long long) (y + 1) * d.sy + a.x0 + x, od, g);
		}
#endif
		if (GENERAL && geo == GEO_NOTHING) {
			s.rho = R(1);
			s.vx = s.vy = s.vz = R(0);
		}
		else {
			aa_read<S, ODD>(a.f, a.sq, base, o, s.f);
			if constexpr (GENERAL)
				coll = apply_boundary(s, geo, a, z, y);
			else {
				density_velocity(s, a.p);
				coll = true;
			}
			write = true;
		}
	}
	if constexpr (OUT)
		step_outputs(a, active, site, s);
	else
		__syncwarp();  // keeps the scheduler from overlapping the read with the collision (no spills)
	if (write) {
		if (coll)
			collide<R, COLL, CUMF>(s, a.p);
		aa_write<S, ODD>(a.f, a.sq, base, o, s.f);
	}
	if (!active)
		return;

	// scalar part (kernels.h:170-195), velocity of the flow site
	R phi = 0;
	if (ag != ADE_NOTHING || !ADE_EARLY_READ) {
		const bool w = !GENERAL || (a.map ? a.map[site] == GEO_PERIODIC : true);
		const Offsets od = neighbour_offsets(w, w && a.zwrap, x, y, z, a.X, a.Y, a.Z, d.sy, d.sz);
		const long long based = (long long) (z + 1) * d.sz + (long long) (y + 1) * d.sy + a.x0 + x;
#if !ADE_EARLY_READ
		ag = d.map[site];
		if (ag != ADE_NOTHING)
			ade_read<ODD>(d.g, d.sq, based, od, g);
#endif
		if (ag != ADE_NOTHING) {
			if (ade_boundary(g, phi, ag, s.vx, s.vy, s.vz, d.inflow_phi))
				ade_collide(g, phi, s.vx, s.vy, s.vz, d.dcoef ? d.dcoef[site] : d.D, d.coll);
			ade_write<ODD>(d.g, d.sq, based, od, g);
		}
	}
	if (OUT && d.phi)
		d.phi[site] = phi;
}

// Coupled step: one thread per site.
template <typename S, int COLL, int CUMF, bool ODD, bool GENERAL, bool OUT, int MINB>
__global__ void __launch_bounds__(128, MINB)
	ade_step_kernel(const StepArgs<typename S::T, typename S::R> a, const AdeArgs<typename S::R> d)
{
	ade_site_update<S, COLL, CUMF, ODD, GENERAL, OUT>(a, d, blockIdx.x * blockDim.x + threadIdx.x,
													  blockIdx.y * blockDim.y + threadIdx.y, blockIdx.z);
}

}  // namespace lbm
