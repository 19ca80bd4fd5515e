// Two-site coupled flow + D3Q7 scalar step (the pair step of pair.cuh with the
// scalar of ade.cuh) for FP32 storage and the cumulant collision.
//
// One launch per plain step over a work list in z-plane order, as
// aa_pair_work_kernel: a tile of 256 x-sites of a row takes the two-site
// update of the groups whose flow sites are all GEO_FLUID (or all
// GEO_PERIODIC) and whose scalar sites all collide without a boundary rewrite
// (ADE_FLUID, ADE_SOLID, ADE_PERIODIC); a chunk of 128 listed sites takes the
// one-site coupled update of ade_site_update.  The scalar of a pair is read
// with the flow's x offsets and its own y and z offsets, collides with the
// pair's flow velocity (kernels.h:170-195) on packed FP32, and is written
// back with the same A-A pattern.  Observation steps run the one-site kernel.
#pragma once

#include "ade.cuh"
#include "pair.cuh"

namespace lbm {

// A-A read / write of the seven scalar populations of sites (x, x + 1), with
// the addresses of PairAt / PairSlots (pair.cuh) over the scalar's slot rows
template <bool ODD>
__device__ __forceinline__ void ade_pair_read_at(const PairAt& at, const PairSlots& ps, F2 (&v)[7])
{
	static_for<7>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (!ODD)
				v[q] = F2(*reinterpret_cast<const float2*>(at.P[1] + ps.b[q]));
			else {
				// direction q of site x comes from slot opp(q) of site x - c_q
				const float* c = reinterpret_cast<const float*>(at.P[1 - cz(q)] + at.oy[1 - cy(q)] + ps.b[opp(q)]);
				if constexpr (cx(q) == 0)
					v[q] = F2(*reinterpret_cast<const float2*>(c));
				else if constexpr (cx(q) > 0)
					v[q] = F2(c[at.left], c[0]);
				else
					v[q] = F2(c[1], c[1 + at.right]);
			}
		}
	);
}

template <bool ODD>
__device__ __forceinline__ void ade_pair_write_at(const PairAt& at, const PairSlots& ps, const F2 (&v)[7])
{
	static_for<7>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (!ODD)
				*reinterpret_cast<float2*>(at.P[1] + ps.b[opp(q)]) = v[q].v;
			else {
				// direction q of site x goes to slot q of site x + c_q
				float* c = reinterpret_cast<float*>(at.P[1 + cz(q)] + at.oy[1 + cy(q)] + ps.b[q]);
				if constexpr (cx(q) == 0)
					*reinterpret_cast<float2*>(c) = v[q].v;
				else if constexpr (cx(q) > 0) {
					c[1] = v[q].v.x;
					c[1 + at.right] = v[q].v.y;
				}
				else {
					c[at.left] = v[q].v.x;
					c[0] = v[q].v.y;
				}
			}
		}
	);
}

// The coupled update of the pair (x, x + 1) of row (y, z) if its group is a
// pair group (groups[] of the coupled step); every thread of the warp calls
// it.  Flow and scalar addresses are plane pointers plus 32-bit slot offsets
// (ps: the flow's 27 slot rows, psd: the scalar's 7), as in pair_update.
template <typename S, int CUMF, bool ODD>
__device__ __forceinline__ void ade_pair_update(const StepArgs<typename S::T, float>& a, const CollParams<F2>& p2,
												const PairSlots& ps, const PairSlots& psd, const AdeArgs<float>& d,
												const uint8_t* __restrict__ groups, int x, int y, int z)
{
	bool act = x < a.X && y < a.Y;
	Site<F2> s;
	F2 g[7];
	PairAt at, atd;
	long long site = 0;
	if (act) {
		const long long row = (long long) z * a.Y + y;
		const int gx = (a.X + PAIR_GROUP - 1) / PAIR_GROUP;
		const uint8_t gf = groups[row * gx + x / PAIR_GROUP];
		act = gf != PAIR_GROUP_REST;
		if (act) {
			const bool wrap = gf == PAIR_GROUP_PERIODIC;
			site = row * a.X + x;
			at = pair_at(a, x, y, z, wrap);
			// the scalar's rows are the flow's, x0 alike
			atd = pair_at_of(reinterpret_cast<char*>(d.g), (long long) sizeof(float), d.sy, d.sz, a.x0, a.X, a.Y, a.Z, x, y,
							 z, wrap, a.zwrap != 0);
			pair_read_at<S, ODD>(at, ps, s);
			ade_pair_read_at<ODD>(atd, psd, g);
			density_velocity(s, p2);
		}
	}
	__syncwarp();  // keeps the collision after the loads (fewer live registers)
	if (!act)
		return;
	collide_cumulant<F2, CUMF>(s, p2);
	pair_write_at<S, ODD>(at, ps, s);
	// the scalar, advected with the pair's flow velocity (unchanged by the collision)
	const F2 phi = ade_phi(g);
	const F2 D = d.dcoef ? F2(d.dcoef[site], d.dcoef[site + 1]) : F2(d.D);
	ade_collide(g, phi, s.vx, s.vy, s.vz, D, d.coll);
	ade_pair_write_at<ODD>(atd, psd, g);
}

// One plain coupled step over the work list (items as aa_pair_work_kernel's).
template <typename S, int CUMF, bool ODD, int MINB>
__global__ void __launch_bounds__(128, MINB)
	ade_pair_work_kernel(const StepArgs<typename S::T, float> a, const CollParams<F2> p2, const PairSlots ps,
						 const PairSlots psd, const AdeArgs<float> d, const uint8_t* __restrict__ groups,
						 const unsigned* __restrict__ work, const unsigned long long* __restrict__ rest, long long nrest,
						 int tiles_x)
{
	const unsigned w = work[blockIdx.x];
	if (w & PAIR_WORK_REST) {
		const long long i = (long long) (w & ~PAIR_WORK_REST) * 128 + threadIdx.x;
		// threads past the list take x = X: no site, but every thread of the
		// warp reaches the update's warp fence
		int x = a.X, y = 0, z = 0;
		if (i < nrest) {
			const unsigned long long e = rest[i];
			const unsigned row = (unsigned) (e >> 32);
			x = (int) (e & 0xffffffffu);
			y = (int) (row % (unsigned) a.Y);
			z = (int) (row / (unsigned) a.Y);
		}
		ade_site_update<S, COLL_CUM, CUMF, ODD, true, false>(a, d, x, y, z);
	}
	else {
		const unsigned row = w / (unsigned) tiles_x;
		const int x = (int) (w - row * (unsigned) tiles_x) * 256 + 2 * (int) threadIdx.x;
		ade_pair_update<S, CUMF, ODD>(a, p2, ps, psd, d, groups, x, (int) (row % (unsigned) a.Y), (int) (row / (unsigned) a.Y));
	}
}

// resident blocks per SM: the coupled pair holds 34 packed values.  The even
// step at 5 (96 registers, 32-36 bytes of spills) ran the duct with a scalar
// at 20.05 GLUPS against 19.05 at 4; the odd step spills 200+ bytes at 5 and
// stays at 4 (128 registers, no spills)
#ifndef ADE_PAIR_MINB_EVEN
#define ADE_PAIR_MINB_EVEN 5
#endif
#ifndef ADE_PAIR_MINB_ODD
#define ADE_PAIR_MINB_ODD 4
#endif

// One plain coupled step through ade_pair_work_kernel; cudaErrorNotSupported
// for what it does not cover (other collisions, no map, observation steps, no
// work list).
template <typename S>
cudaError_t ade_pair_step(const StepLaunch& L)
{
	using T = typename S::T;
	static_assert(sizeof(T) == 4 && sizeof(typename S::R) == 4, "FP32 storage");
	const AdeLaunch* A = L.ade;
	if (!A || L.coll != COLL_CUM || !L.map || L.macro || L.partials || A->phi || !A->pair_groups || !A->pair_work.work
		|| A->pair_work.nwork < 1)
		return cudaErrorNotSupported;
	if ((L.g.x0 | L.g.sq | L.g.sy | L.g.sz | A->sy | A->sz) & 1)
		return cudaErrorNotSupported;
	if (L.cum_flags != 0 && L.cum_flags != CUM_ANTIALIAS && L.cum_flags != (CUM_2017 | CUM_ANTIALIAS))
		return cudaErrorInvalidValue;
	StepArgs<T, float> a;
	a.f = (T*) L.g.f;
	a.sq = L.g.sq;
	a.sy = L.g.sy;
	a.sz = L.g.sz;
	a.x0 = L.g.x0;
	a.X = L.g.X;
	a.Y = L.g.Y;
	a.Z = L.g.Z;
	a.map = L.map;
	a.in_vx = (const float*) L.inflow[0];
	a.in_vy = (const float*) L.inflow[1];
	a.in_vz = (const float*) L.inflow[2];
	a.macro = nullptr;
	a.partials = nullptr;
	a.zwrap = L.distributed_z ? 0 : 1;
	a.p = make_coll_params<float>(L.p);
	const CollParams<F2> p2 = make_coll_params<F2>(L.p);
	AdeArgs<float> d;
	d.g = (float*) A->g;
	d.sq = A->sq;
	d.sy = A->sy;
	d.sz = A->sz;
	d.map = A->map;
	d.dcoef = (const float*) A->dcoef;
	d.D = (float) A->D;
	d.inflow_phi = (float) A->inflow_phi;
	d.phi = nullptr;
	d.coll = A->coll;
	// every slot offset of a lattice row fits 32 bits (the scalar's rows are
	// as long as the flow's)
	if (27ll * L.g.sq * (long long) sizeof(T) >= (1ll << 31) || 27ll * A->sq * (long long) sizeof(float) >= (1ll << 31))
		return cudaErrorNotSupported;
	const PairSlots ps = make_pair_slots(L.g.sq, (int) sizeof(T));
	const PairSlots psd = make_pair_slots(A->sq, (int) sizeof(float));
	const PairWork& W = A->pair_work;
	const dim3 grid((unsigned) W.nwork), block(128);
	if (L.blocks_out)
		*L.blocks_out = (long long) W.nwork * 4;
	if (L.dry_run)
		return cudaSuccess;
	const int tiles_x = ((L.g.X + 1) / 2 + 127) / 128;
#define LBM_ADE_PAIR(CUMF)                                                                                             \
	do {                                                                                                               \
		if (L.odd)                                                                                                     \
			ade_pair_work_kernel<S, CUMF, true, ADE_PAIR_MINB_ODD>                                                         \
				<<<grid, block, 0, L.stream>>>(a, p2, ps, psd, d, A->pair_groups, W.work, W.rest, W.nrest, tiles_x);            \
		else                                                                                                           \
			ade_pair_work_kernel<S, CUMF, false, ADE_PAIR_MINB_EVEN>                                                        \
				<<<grid, block, 0, L.stream>>>(a, p2, ps, psd, d, A->pair_groups, W.work, W.rest, W.nrest, tiles_x);            \
	} while (0)
	switch (L.cum_flags) {
		case 0:
			LBM_ADE_PAIR(0);
			break;
		case CUM_ANTIALIAS:
			LBM_ADE_PAIR(CUM_ANTIALIAS);
			break;
		default:
			LBM_ADE_PAIR(CUM_2017 | CUM_ANTIALIAS);
			break;
	}
#undef LBM_ADE_PAIR
	return cudaGetLastError();
}

}  // namespace lbm
