// A-A stepping kernels for sm_100a (even and odd step of the fused
// stream + boundary + collide update), initialisation, layout conversion and
// the FP64 reductions.
//
// Data layout in HBM (one allocation per lattice):
//   populations  slot-major SoA: index(q, x, y, z) = q*sq + (z+1)*sz + (y+1)*sy + x0 + x
//                x fastest.  One ghost layer of sites surrounds the lattice
//                (x = -1 .. X, y = -1 .. Y, z = -1 .. Z), which the reference's
//                A-A kernel assumes (include/lbm3d/kernels.h:30-37).  x0 pads
//                the row so that interior x = 0 starts on a 128-byte boundary;
//                sy is a multiple of 128 bytes, so every row of every
//                direction is a coalesced, 128-byte-aligned stream.
//   map          uint8 [Z][Y][X] GEO values (general kernels only)
//   macro        compute type [4][Z][Y][X] (rho, vx, vy, vz)
//
// A-A pattern (include/lbm3d/d3q27/streaming_AA.h:12-116):
//   even step  read slot q of the site, write direction q into slot opp(q)
//              of the same site;
//   odd step   read direction q from slot opp(q) of site x - c_q, write
//              direction q into slot q of site x + c_q.
// In both steps a thread writes exactly the 27 locations it read, and no
// other thread touches them, so the update runs in place without races.
#pragma once

#include <cstdint>
#include <type_traits>
#include <utility>

#include "collision.cuh"

namespace lbm {

template <int... Is, typename F>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Is...>, F&& f)
{
	(f(std::integral_constant<int, Is>{}), ...);
}
// compile-time loop: f receives std::integral_constant<int, i> for i = 0..N-1
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f)
{
	static_for_impl(std::make_integer_sequence<int, N>{}, f);
}

// number of FP64 reduction quantities per block: sum rho, rho*vx, rho*vy,
// rho*vz, rho*|u|^2 and the count of non-finite densities
constexpr int NRED = 6;

template <typename T, typename R>
struct StepArgs
{
	T* f;
	long long sq;
	int sy, sz, x0;
	int X, Y, Z;
	const uint8_t* map;	 // general kernels only
	const R* in_vx;
	const R* in_vy;
	const R* in_vz;
	R* macro;		   // [4][Z][Y][X] or null
	double* partials;  // [NRED][slots] or null
	int zwrap;		   // 0: distributed along z, periodic sites do not wrap in z
	CollParams<R> p;
};

// Offsets (in elements) of the neighbour sites; periodic sites wrap, all
// other sites reach into the ghost layer (kernels.h:21-37).
struct Offsets
{
	long long x[3], y[3], z[3];
};

// wrap_z = false: a lattice distributed along z (a slab of a larger lattice,
// kernelInitIndices with distributed.z(), kernels.h:21-37) reaches its z
// neighbours through the ghost layer, which the halo exchange fills
__device__ __forceinline__ Offsets neighbour_offsets(bool wrap, bool wrap_z, int x, int y, int z, int X, int Y, int Z, int sy,
													int sz)
{
	Offsets o;
	o.x[0] = (wrap && x == 0) ? (X - 1) : -1;
	o.x[1] = 0;
	o.x[2] = (wrap && x == X - 1) ? -(X - 1) : 1;
	o.y[0] = (long long) ((wrap && y == 0) ? (Y - 1) : -1) * sy;
	o.y[1] = 0;
	o.y[2] = (long long) ((wrap && y == Y - 1) ? -(Y - 1) : 1) * sy;
	o.z[0] = (long long) ((wrap_z && z == 0) ? (Z - 1) : -1) * sz;
	o.z[1] = 0;
	o.z[2] = (long long) ((wrap_z && z == Z - 1) ? -(Z - 1) : 1) * sz;
	return o;
}

__device__ __forceinline__ Offsets neighbour_offsets(bool wrap, int x, int y, int z, int X, int Y, int Z, int sy, int sz)
{
	return neighbour_offsets(wrap, wrap, x, y, z, X, Y, Z, sy, sz);
}

// A-A read of the 27 populations (streaming_AA.h:79-116)
template <typename S, bool ODD>
__device__ __forceinline__ void aa_read(const typename S::T* __restrict__ f, long long sq, long long base, const Offsets& o,
										typename S::R* v)
{
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (ODD)
				v[q] = S::template load<opp(q)>(f + opp(q) * sq + base + o.x[1 - cx(q)] + o.y[1 - cy(q)] + o.z[1 - cz(q)]);
			else
				v[q] = S::template load<q>(f + q * sq + base);
		}
	);
}

// A-A write of the 27 populations (streaming_AA.h:12-76)
template <typename S, bool ODD>
__device__ __forceinline__ void aa_write(typename S::T* __restrict__ f, long long sq, long long base, const Offsets& o,
										 const typename S::R* v)
{
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (ODD)
				S::template store<q>(f + q * sq + base + o.x[1 + cx(q)] + o.y[1 + cy(q)] + o.z[1 + cz(q)], v[q]);
			else
				S::template store<opp(q)>(f + opp(q) * sq + base, v[q]);
		}
	);
}

// mirror copy of a symmetry plane (bc.h:222-293): directions whose component
// along the plane normal equals `side` take the value of their mirror image.
// One code path for all six GEO_SYM_* types, selected at run time: axis 0/1/2
// = x/y/z; the sources (component -side) are never overwritten.
template <typename R>
__device__ __forceinline__ void symmetry(R* f, int axis, int side)
{
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (cx(q) != 0) {
				constexpr int m = dir(-cx(q), cy(q), cz(q));
				if (axis == 0 && cx(q) == side)
					f[q] = f[m];
			}
			if constexpr (cy(q) != 0) {
				constexpr int m = dir(cx(q), -cy(q), cz(q));
				if (axis == 1 && cy(q) == side)
					f[q] = f[m];
			}
			if constexpr (cz(q) != 0) {
				constexpr int m = dir(cx(q), cy(q), -cz(q));
				if (axis == 2 && cz(q) == side)
					f[q] = f[m];
			}
		}
	);
}

// density of a left inlet from the populations that stream in from the
// interior (bc.h:97-110)
template <typename R>
__device__ __forceinline__ R inlet_density(const R* f, R vx)
{
	return R(1) / (R(1) - vx)
		 * ((f[ZZZ] + (((f[ZPP] + f[ZMM]) + (f[ZPM] + f[ZMP])) + ((f[ZPZ] + f[ZMZ]) + (f[ZZP] + f[ZZM]))))
			+ R(2) * (f[MZZ] + (((f[MPP] + f[MMM]) + (f[MPM] + f[MMP])) + ((f[MPZ] + f[MMZ]) + (f[MZP] + f[MZM])))));
}

// moment-based velocity inlet of Eichler et al. (bc.h:91-142)
template <typename R>
__device__ __forceinline__ void inlet_moments(Site<R>& s)
{
	R* f = s.f;
	s.rho = inlet_density(f, s.vx);
	const R rho = s.rho, vx = s.vx, vy = s.vy, vz = s.vz;
	const R third = R(1.0 / 3.0), ninth = R(1.0 / 9.0);
	const R m100 = rho * vx, m010 = rho * vy, m001 = rho * vz;
	const R m011 = rho * (vy * vz);
	const R m020 = third * rho + rho * (vy * vy);
	const R m002 = third * rho + rho * (vz * vz);
	const R m021 = third * rho * vz + rho * ((vy * vy) * vz);
	const R m012 = third * rho * vy + rho * (vy * (vz * vz));
	const R m022 = ninth * rho + third * rho * (vy * vy + vz * vz) + rho * (vy * vy) * (vz * vz);
	f[PZZ] = m100 + (m022 - (m020 + m002)) + f[MZZ] + (((f[ZPP] + f[ZMM]) + (f[ZPM] + f[ZMP])) + ((f[ZZP] + f[ZZM]) + (f[ZPZ] + f[ZMZ])))
		   + R(2) * (((f[MPP] + f[MMM]) + (f[MPM] + f[MMP])) + ((f[MPZ] + f[MMZ]) + (f[MZP] + f[MZM])));
	f[PPZ] = R(0.5) * ((m020 - m022) + (m010 - m012)) - (f[MPZ] + f[ZPZ]);
	f[PMZ] = R(0.5) * ((m020 - m022) + (m012 - m010)) - (f[MMZ] + f[ZMZ]);
	f[PZP] = R(0.5) * ((m002 - m022) + (m001 - m021)) - (f[MZP] + f[ZZP]);
	f[PZM] = R(0.5) * ((m002 - m022) + (m021 - m001)) - (f[MZM] + f[ZZM]);
	f[PPP] = R(0.25) * ((m022 + m011) + (m021 + m012)) - (f[MPP] + f[ZPP]);
	f[PPM] = R(0.25) * ((m022 - m011) + (m012 - m021)) - (f[MPM] + f[ZPM]);
	f[PMP] = R(0.25) * ((m022 - m011) + (m021 - m012)) - (f[MMP] + f[ZMP]);
	f[PMM] = R(0.25) * ((m022 + m011) - (m021 + m012)) - (f[MMM] + f[ZMM]);
}

// Pre-collision part of D3Q27_BC_All for one site (bc.h:85-403) for the site
// types that are free of cross-site ordering in the A-A pattern: fills rho and
// u, rewrites the populations a boundary prescribes, and returns whether the
// site collides (bc.h:406-412).
template <typename R, typename T>
__device__ __forceinline__ bool apply_boundary(Site<R>& s, uint8_t geo, const StepArgs<T, R>& a, int z, int y)
{
	const long long prof = (long long) z * a.Y + y;
	switch (geo) {
		case GEO_INFLOW:
			s.vx = a.in_vx ? a.in_vx[prof] : R(0);
			s.vy = a.in_vy ? a.in_vy[prof] : R(0);
			s.vz = a.in_vz ? a.in_vz[prof] : R(0);
			s.rho = R(1);
			set_equilibrium(s.f, a.p.eq, s.rho, s.vx, s.vy, s.vz);
			return false;
		case GEO_INFLOW_LEFT:
			s.vx = a.in_vx ? a.in_vx[prof] : R(0);
			s.vy = a.in_vy ? a.in_vy[prof] : R(0);
			s.vz = a.in_vz ? a.in_vz[prof] : R(0);
			inlet_moments(s);
			s.ir = rcp(s.rho);
			return true;
		case GEO_INFLOW_EQ_LEFT:
			s.vx = a.in_vx ? a.in_vx[prof] : R(0);
			s.vy = a.in_vy ? a.in_vy[prof] : R(0);
			s.vz = a.in_vz ? a.in_vz[prof] : R(0);
			s.rho = inlet_density(s.f, s.vx);
			set_equilibrium(s.f, a.p.eq, s.rho, s.vx, s.vy, s.vz);
			return false;
		case GEO_OUTFLOW_EQ:
			density_velocity(s, a.p);
			s.rho = R(1);
			set_equilibrium(s.f, a.p.eq, s.rho, s.vx, s.vy, s.vz);
			return false;
		case GEO_WALL:
			// full-way bounce-back (bc.h:201-221)
			s.rho = R(1);
			s.vx = s.vy = s.vz = R(0);
#pragma unroll
			for (int q = 1; q < 27; q += 2) {
				const R t = s.f[q];
				s.f[q] = s.f[q + 1];
				s.f[q + 1] = t;
			}
			return false;
		case GEO_SYM_TOP:
		case GEO_SYM_BOTTOM:
		case GEO_SYM_LEFT:
		case GEO_SYM_RIGHT:
		case GEO_SYM_BACK:
		case GEO_SYM_FRONT: {
			// TOP/BOTTOM: z, LEFT/RIGHT: x, BACK/FRONT: y; the overwritten side
			// is -1 for TOP, RIGHT, FRONT and +1 for BOTTOM, LEFT, BACK
			const int axis = geo <= GEO_SYM_BOTTOM ? 2 : (geo <= GEO_SYM_RIGHT ? 0 : 1);
			const int side = (geo == GEO_SYM_TOP || geo == GEO_SYM_RIGHT || geo == GEO_SYM_FRONT) ? -1 : 1;
			symmetry(s.f, axis, side);
			density_velocity(s, a.p);
			return false;
		}
		default:  // GEO_FLUID, GEO_PERIODIC
			density_velocity(s, a.p);
			return true;
	}
}

// Per-warp FP64 sums of the NRED quantities of one step, stored as
// partials[k][slot] with one slot per warp of the launch.  No shared memory
// and no barrier: a warp leaves as soon as its own sums are stored, so the
// observation step keeps as many loads in flight as the plain step.  The
// butterfly halves the set of values each warp lane carries at every level
// (8 slots, the last two zero: 4 + 2 + 1 exchanges), then finishes with two
// plain levels, 9 64-bit shuffles in all instead of 5 per quantity; lane 4q
// ends with the warp sum of quantity q.  The order of the additions is fixed.
// Requires blockDim.x to be a multiple of 32, so that a warp is one row of
// the block.  The warp's slot is `slot` of `nslots` (partials[k * nslots +
// slot]); the two-argument form numbers the warps of the launch from 0.
__device__ __forceinline__ void warp_reduce_store(const double (&v)[NRED], double* partials, long long slot, long long nslots)
{
	constexpr unsigned FULL = 0xffffffffu;
	const int tid = threadIdx.x + blockDim.x * threadIdx.y;
	const int lane = tid & 31;
	const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
	double a[4];
#pragma unroll
	for (int i = 0; i < 4; i++) {
		const double lo = v[i];
		const double hi = i + 4 < NRED ? v[(i + 4) % NRED] : 0.0;
		a[i] = (h16 ? hi : lo) + __shfl_xor_sync(FULL, h16 ? lo : hi, 16);
	}
	double b[2];
#pragma unroll
	for (int i = 0; i < 2; i++)
		b[i] = (h8 ? a[i + 2] : a[i]) + __shfl_xor_sync(FULL, h8 ? a[i] : a[i + 2], 8);
	double c = (h4 ? b[1] : b[0]) + __shfl_xor_sync(FULL, h4 ? b[0] : b[1], 4);
	c += __shfl_xor_sync(FULL, c, 2);
	c += __shfl_xor_sync(FULL, c, 1);
	const int q = (h16 ? 4 : 0) + (h8 ? 2 : 0) + (h4 ? 1 : 0);
	if ((lane & 3) == 0 && q < NRED)
		partials[q * nslots + slot] = c;
}
__device__ __forceinline__ void warp_reduce_store(const double (&v)[NRED], double* partials)
{
	const int wpb = (blockDim.x * blockDim.y) >> 5;
	const long long nslots = (long long) gridDim.x * gridDim.y * gridDim.z * wpb;
	const long long block = blockIdx.x + (long long) gridDim.x * (blockIdx.y + (long long) gridDim.y * blockIdx.z);
	const int warp = (threadIdx.x + blockDim.x * threadIdx.y) >> 5;
	warp_reduce_store(v, partials, block * wpb + warp, nslots);
}

// Lets the grid launched after this one as a programmatic dependent (the
// finish kernel of the sums) be scheduled once every block of this grid has
// started; the dependent still waits for this grid's completion
// (griddepcontrol.wait) before it reads anything.
__device__ __forceinline__ void launch_dependents()
{
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Outputs of an observation step for one site: the macro field and the
// per-warp FP64 sums.  Every lane of the warp calls it (lanes past the
// lattice edge with active = false).  The step kernels call it between the
// boundary treatment and the collision: the collision changes neither the
// density nor the velocity, and the registers of the sums are free again
// before the collision needs the most.
template <typename T, typename R>
__device__ __forceinline__ void step_outputs(const StepArgs<T, R>& a, bool active, long long site, const Site<R>& s)
{
	if (active && a.macro) {
		const long long n = (long long) a.X * a.Y * a.Z;
		a.macro[site] = s.rho;
		a.macro[n + site] = s.vx;
		a.macro[2 * n + site] = s.vy;
		a.macro[3 * n + site] = s.vz;
	}
	if (a.partials) {
		double red[NRED] = {0, 0, 0, 0, 0, 0};
		if (active) {
			const double rho = (double) s.rho, vx = (double) s.vx, vy = (double) s.vy, vz = (double) s.vz;
			red[0] = rho;
			red[1] = rho * vx;
			red[2] = rho * vy;
			red[3] = rho * vz;
			red[4] = rho * (vx * vx + vy * vy + vz * vz);
			red[5] = isfinite(rho) ? 0.0 : 1.0;
		}
		warp_reduce_store(red, a.partials);
	}
}

template <typename R>
__device__ __forceinline__ void block_reduce_store(double (&v)[NRED], double* partials)
{
	// warp level
#pragma unroll
	for (int k = 0; k < NRED; k++)
#pragma unroll
		for (int off = 16; off > 0; off >>= 1)
			v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
	__shared__ double red[32][NRED];
	const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
	const int nthreads = blockDim.x * blockDim.y * blockDim.z;
	const int lane = tid & 31, warp = tid >> 5, nwarps = (nthreads + 31) >> 5;
	if (lane == 0)
#pragma unroll
		for (int k = 0; k < NRED; k++)
			red[warp][k] = v[k];
	__syncthreads();
	if (tid < NRED) {
		double acc = 0;
		for (int w = 0; w < nwarps; w++)
			acc += red[w][tid];
		// structure of arrays: partials[k][block], so that the finish kernels
		// read each quantity with coalesced loads
		const long long nblocks = (long long) gridDim.x * gridDim.y * gridDim.z;
		const long long block = blockIdx.x + (long long) gridDim.x * (blockIdx.y + (long long) gridDim.y * blockIdx.z);
		partials[tid * nblocks + block] = acc;
	}
}

// One A-A step over the whole lattice.  OUT = true compiles the macro-field
// output and the FP64 partial sums (used on observation steps only), so the
// plain step carries none of their registers.  GENERAL = false: every site is
// periodic (no map read).  GENERAL = true: per-site GEO type from the map with
// the boundary conditions of D3Q27_BC_All (bc.h:60-422) that are free of
// cross-site ordering in the A-A pattern.
// The per-site step of the direct kernel with the collision as a functor
// collide(Site<R>&): the COLL slot of cudaLBMKernel (kernels.h:59-112), so
// that the built-in collisions and a user's collision (plugin.cuh) run the
// same streaming, boundary treatment and outputs.
template <typename S, bool ODD, bool GENERAL, bool OUT, typename Collide>
__device__ __forceinline__ void aa_step_site(const StepArgs<typename S::T, typename S::R>& a, Collide&& collide)
{
	using R = typename S::R;
	const int x = blockIdx.x * blockDim.x + threadIdx.x;
	const int y = blockIdx.y * blockDim.y + threadIdx.y;
	const int z = blockIdx.z;
	const bool active = x < a.X && y < a.Y;

	Site<R> s;
	Offsets o;
	long long base = 0, site = 0;
	bool coll = false, write = false;
	if (active) {
		base = (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + x;
		site = ((long long) z * a.Y + y) * a.X + x;
		uint8_t geo = GEO_PERIODIC;
		if constexpr (GENERAL)
			geo = a.map[site];
		if (GENERAL && geo == GEO_NOTHING) {
			s.rho = R(1);
			s.vx = s.vy = s.vz = R(0);
		}
		else {
			const bool wrap = !GENERAL || geo == GEO_PERIODIC;
			o = neighbour_offsets(wrap, wrap && a.zwrap, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
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
	if (write) {
		if (coll)
			collide(s);
		aa_write<S, ODD>(a.f, a.sq, base, o, s.f);
	}
}

template <typename S, int COLL, int CUMF, bool ODD, bool GENERAL, bool OUT, int MINB>
__global__ void __launch_bounds__(128, MINB) aa_step_kernel(const StepArgs<typename S::T, typename S::R> a)
{
	using R = typename S::R;
	if constexpr (OUT)
		launch_dependents();
	aa_step_site<S, ODD, GENERAL, OUT>(a, [&](Site<R>& s) { collide<R, COLL, CUMF>(s, a.p); });
}

// Split step for lattices with a map: the host sorts the lattice's tiles of
// 128 consecutive x-sites of one row into tiles whose sites are all
// GEO_FLUID and tiles holding any other type (or lying partly outside the
// lattice), and runs one launch over each list.  The fluid-only launch reads
// no map and takes no boundary branch; with the duct's inlet, outlet and wall
// rims about half of the tiles are fluid-only.  Both launches update disjoint
// sites with the per-site code of aa_step_kernel, so the results are those of
// the direct kernel.
template <typename S, int COLL, int CUMF, bool ODD, bool INTERIOR, int MINB>
__global__ void __launch_bounds__(128, MINB)
	aa_split_kernel(const StepArgs<typename S::T, typename S::R> a, const unsigned* __restrict__ tiles, int tiles_x)
{
	using R = typename S::R;
	const unsigned t = tiles[blockIdx.x];
	const unsigned row = t / (unsigned) tiles_x;
	const int x = (int) (t - row * (unsigned) tiles_x) * 128 + (int) threadIdx.x;
	const int y = (int) (row % (unsigned) a.Y);
	const int z = (int) (row / (unsigned) a.Y);
	if (x >= a.X)
		return;	 // the last tile of a row can be partial (never a fluid-only tile)
	const long long base = (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + x;
	Site<R> s;
	if constexpr (INTERIOR) {
		const Offsets o = neighbour_offsets(false, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
		aa_read<S, ODD>(a.f, a.sq, base, o, s.f);
		density_velocity(s, a.p);
		collide<R, COLL, CUMF>(s, a.p);
		aa_write<S, ODD>(a.f, a.sq, base, o, s.f);
	}
	else {
		const long long site = ((long long) z * a.Y + y) * a.X + x;
		const uint8_t geo = a.map[site];
		if (geo == GEO_NOTHING)
			return;
		const Offsets o = neighbour_offsets(geo == GEO_PERIODIC, geo == GEO_PERIODIC && a.zwrap, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
		aa_read<S, ODD>(a.f, a.sq, base, o, s.f);
		if (apply_boundary(s, geo, a, z, y))
			collide<R, COLL, CUMF>(s, a.p);
		aa_write<S, ODD>(a.f, a.sq, base, o, s.f);
	}
}

}  // namespace lbm
