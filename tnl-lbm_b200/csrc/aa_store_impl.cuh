// Kernel instantiations for one population storage format.  Included by
// aa_store_<format>.cu, which defines LBM_TILE_MINB (resident blocks of the
// tile kernel) and names the storage type in LBM_DEFINE_STORAGE_OPS.
#pragma once

#include <cstring>

#include "aa_kernels.cuh"
#include "ab_kernels.cuh"
#include "coll_params.cuh"
#include "aa_tile.cuh"
#include "ade.cuh"
#include "ensemble.cuh"
#include "launch.h"

namespace lbm {


// Resident 128-thread blocks per SM requested from the compiler for the
// direct step kernel; __launch_bounds__(128, n) caps registers at
// 65536 / (128 n): 4 -> 128, 5 -> 102 (96 used), 6 -> 85 (80 used).  The
// values are the largest n at which the instantiations compile without (or
// with a few bytes of) register spills (-Xptxas -v on sm_100a): more
// resident warps keep more HBM requests in flight.  The observation variant
// (OUT) needs no more registers than the plain step: its outputs are written
// before the collision.  The FP64 kernels need twice the registers per value.
//
// FP64 arithmetic: 4 blocks (128 registers, up to 24 bytes of spills) for
// MRT and the default and anti-aliased cumulant, 3 (168 registers, up to 68
// bytes) for SRT, BGK and the Geier-2017 cumulant, which spill 140-500 bytes
// at 4.  Against 2 blocks (the full 256 registers, of which these kernels use
// 110-150), duct: cumulant 14.5 -> 15.3, SRT 11.7 -> 13.6, BGK 13.1 -> 14.5,
// MRT 14.3 -> 15.2 GLUPS; 256^3 Taylor-Green vortex (Geier 2017) 10.7 -> 12.9.
template <typename R, int COLL, int CUMF, bool ODD, bool GENERAL, bool OUT>
constexpr int direct_minb()
{
	if (sizeof(R) == 8)
		return COLL == COLL_SRT || COLL == COLL_BGK || (COLL == COLL_CUM && (CUMF & CUM_2017)) ? 3 : 4;
	if (!ODD && GENERAL)
		return 6;  // the even general step keeps no neighbour offsets: 80 registers
	if (COLL == COLL_CUM || COLL == COLL_MRT)
		return 5;
	return 4;  // SRT and BGK spill at 5
}

// resident blocks of the coupled flow + scalar step: as the direct step's,
// and 2 with FP64 arithmetic (the scalar's seven values on top of the flow's)
template <typename R, int COLL, int CUMF, bool ODD, bool GENERAL, bool OUT>
constexpr int ade_minb()
{
	return sizeof(R) == 8 ? 2 : direct_minb<R, COLL, CUMF, ODD, GENERAL, OUT>();
}

// resident blocks of the A-B step; its observation variant spills at 5.  In
// FP64, 3 blocks (168 registers, 56-144 bytes of spills; the step uses about
// 200 at 2): duct cumulant 11.8 -> 13.8, SRT 11.6 -> 13.7 GLUPS
template <typename R, int COLL, int CUMF, bool OUT>
constexpr int ab_minb()
{
	if (sizeof(R) == 8)
		return 3;
	if (OUT)
		return 4;
	return direct_minb<R, COLL, CUMF, true, true, false>();
}

#ifndef SPLIT_MINB_FLUID
#define SPLIT_MINB_FLUID 5
#endif

#ifndef ENS_MINB128
#define ENS_MINB128 5
#endif

// resident 128-thread blocks per SM of the persistent two-site ensemble kernel
#ifndef ENS_PAIR_MINB
#define ENS_PAIR_MINB 4
#endif

// Resident blocks per SM for the fluid-only launch of the split step (no map,
// no boundary branch): the largest counts without register spills.
template <typename R, int COLL, bool ODD>
constexpr int split_minb()
{
	if (sizeof(R) == 8)
		return 2;
	if (COLL == COLL_SRT || COLL == COLL_BGK)
		return 4;
	return SPLIT_MINB_FLUID;
}

template <typename S>
struct StorageUnit
{
	using T = typename S::T;
	using R = typename S::R;

	static constexpr int TILE_X = 128;
	static constexpr int TILE_STAGES = 3;

	template <int COLL, int CUMF, bool ODD, bool GENERAL>
	static cudaError_t launch_tile(const StepLaunch& L, const StepArgs<T, R>& a)
	{
		auto kern = aa_tile_kernel<S, COLL, CUMF, ODD, GENERAL, TILE_X, TILE_STAGES>;
		constexpr int smem = tile_smem_bytes<T, TILE_X, ODD, TILE_STAGES>();
		constexpr int threads = TILE_X;
		// per-device launch facts of this instantiation, computed once
		static int per_sm_cache[64] = {0};
		static int sms_cache[64] = {0};
		int dev = 0;
		cudaGetDevice(&dev);
		if (dev < 0 || dev >= 64)
			return cudaErrorInvalidDevice;
		if (per_sm_cache[dev] == 0) {
			cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
			if (e != cudaSuccess)
				return e;
			int per_sm = 0, sms = 0;
			e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
			if (e != cudaSuccess)
				return e;
			e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
			if (e != cudaSuccess)
				return e;
			if (per_sm < 1)
				return cudaErrorInvalidConfiguration;
			sms_cache[dev] = sms;
			per_sm_cache[dev] = per_sm < TILE_MAX_BLOCKS_PER_SM ? per_sm : TILE_MAX_BLOCKS_PER_SM;
		}
		const int tiles_x = (a.X + TILE_X - 1) / TILE_X;
		const long long ntiles = (long long) tiles_x * a.Y * a.Z;
		long long grid = (long long) per_sm_cache[dev] * sms_cache[dev];
		if (grid > ntiles)
			grid = ntiles;
		if (L.blocks_out)
			*L.blocks_out = grid;
		if (L.dry_run)
			return cudaSuccess;
		kern<<<(unsigned) grid, threads, smem, L.stream>>>(a, L.status, ntiles, tiles_x,
														   L.wait_limit >= 0 ? L.wait_limit : WAIT_LIMIT);
		return cudaGetLastError();
	}

	template <int COLL, int CUMF, bool ODD>
	static cudaError_t launch_split(const StepLaunch& L, const StepArgs<T, R>& a)
	{
		constexpr int minb_in = split_minb<R, COLL, ODD>();
		constexpr int minb_bd = direct_minb<R, COLL, CUMF, ODD, true, false>();
		if (L.blocks_out)
			*L.blocks_out = L.split_n[0] + L.split_n[1];
		if (L.dry_run)
			return cudaSuccess;
		if (L.split_n[0] > 0)
			aa_split_kernel<S, COLL, CUMF, ODD, true, minb_in>
				<<<(unsigned) L.split_n[0], 128, 0, L.stream>>>(a, L.split_tiles, L.split_tiles_x);
		if (L.split_n[1] > 0)
			aa_split_kernel<S, COLL, CUMF, ODD, false, minb_bd>
				<<<(unsigned) L.split_n[1], 128, 0, L.stream>>>(a, L.split_tiles + L.split_n[0], L.split_tiles_x);
		return cudaGetLastError();
	}

	template <int COLL, int CUMF, bool ODD, bool GENERAL>
	static cudaError_t launch_one(const StepLaunch& L, const StepArgs<T, R>& a)
	{
		// the tile kernel's windows wrap z on periodic lattices: slabs run the direct kernel
		if (L.kernel == KERNEL_TILE && !L.distributed_z)
			return launch_tile<COLL, CUMF, ODD, GENERAL>(L, a);
		// plain steps of a lattice with a map (observation steps run the direct kernel)
		if constexpr (GENERAL)
			if (L.kernel == KERNEL_SPLIT && L.split_tiles && !L.macro && !L.partials)
				return launch_split<COLL, CUMF, ODD>(L, a);
		if (L.blocks_out)  // one partial-sum slot per warp
			*L.blocks_out = (long long) L.grid.x * L.grid.y * L.grid.z * ((L.block.x * L.block.y) / 32);
		if (L.dry_run)
			return cudaSuccess;
		if (L.macro || L.partials)
			aa_step_kernel<S, COLL, CUMF, ODD, GENERAL, true, direct_minb<R, COLL, CUMF, ODD, GENERAL, true>()>
				<<<L.grid, L.block, 0, L.stream>>>(a);
		else
			aa_step_kernel<S, COLL, CUMF, ODD, GENERAL, false, direct_minb<R, COLL, CUMF, ODD, GENERAL, false>()>
				<<<L.grid, L.block, 0, L.stream>>>(a);
		return cudaGetLastError();
	}

	template <int COLL, int CUMF>
	static cudaError_t launch_parity(const StepLaunch& L, const StepArgs<T, R>& a)
	{
		const bool general = L.map != nullptr;
		if (L.odd)
			return general ? launch_one<COLL, CUMF, true, true>(L, a) : launch_one<COLL, CUMF, true, false>(L, a);
		return general ? launch_one<COLL, CUMF, false, true>(L, a) : launch_one<COLL, CUMF, false, false>(L, a);
	}

	// ---- coupled flow + D3Q7 scalar step (ade.cuh)
	template <int COLL, int CUMF, bool ODD, bool GENERAL>
	static cudaError_t ade_one(const StepLaunch& L, const StepArgs<T, R>& a, const AdeArgs<R>& d)
	{
		if (L.blocks_out)  // one partial-sum slot per warp
			*L.blocks_out = (long long) L.grid.x * L.grid.y * L.grid.z * ((L.block.x * L.block.y) / 32);
		if (L.dry_run)
			return cudaSuccess;
		if (L.macro || L.partials || d.phi)
			ade_step_kernel<S, COLL, CUMF, ODD, GENERAL, true, ade_minb<R, COLL, CUMF, ODD, GENERAL, true>()>
				<<<L.grid, L.block, 0, L.stream>>>(a, d);
		else
			ade_step_kernel<S, COLL, CUMF, ODD, GENERAL, false, ade_minb<R, COLL, CUMF, ODD, GENERAL, false>()>
				<<<L.grid, L.block, 0, L.stream>>>(a, d);
		return cudaGetLastError();
	}

	template <int COLL, int CUMF>
	static cudaError_t ade_parity(const StepLaunch& L, const StepArgs<T, R>& a, const AdeArgs<R>& d)
	{
		const bool general = L.map != nullptr;
		if (L.odd)
			return general ? ade_one<COLL, CUMF, true, true>(L, a, d) : ade_one<COLL, CUMF, true, false>(L, a, d);
		return general ? ade_one<COLL, CUMF, false, true>(L, a, d) : ade_one<COLL, CUMF, false, false>(L, a, d);
	}

	static cudaError_t ade_step(const StepLaunch& L)
	{
		if constexpr (sizeof(T) != sizeof(R)) {
			(void) L;
			return cudaErrorNotSupported;
		}
		else {
			if (!L.ade)
				return cudaErrorInvalidValue;
			const StepArgs<T, R> a = step_args(L);
			AdeArgs<R> d;
			d.g = (R*) L.ade->g;
			d.sq = L.ade->sq;
			d.sy = L.ade->sy;
			d.sz = L.ade->sz;
			d.map = L.ade->map;
			d.dcoef = (const R*) L.ade->dcoef;
			d.D = (R) L.ade->D;
			d.inflow_phi = (R) L.ade->inflow_phi;
			d.phi = (R*) L.ade->phi;
			d.coll = L.ade->coll;
			switch (L.coll) {
				case COLL_CUM:
					switch (L.cum_flags) {
						case 0:
							return ade_parity<COLL_CUM, 0>(L, a, d);
						case CUM_ANTIALIAS:
							return ade_parity<COLL_CUM, CUM_ANTIALIAS>(L, a, d);
						case CUM_2017 | CUM_ANTIALIAS:
							return ade_parity<COLL_CUM, CUM_2017 | CUM_ANTIALIAS>(L, a, d);
						default:
							return cudaErrorInvalidValue;
					}
				case COLL_SRT:
					return ade_parity<COLL_SRT, 0>(L, a, d);
				case COLL_BGK:
					return ade_parity<COLL_BGK, 0>(L, a, d);
				case COLL_MRT:
					return ade_parity<COLL_MRT, 0>(L, a, d);
				default:
					return cudaErrorInvalidValue;
			}
		}
	}

	static StepArgs<T, R> step_args(const StepLaunch& L)
	{
		return make_step_args<S>(L);
	}

	static cudaError_t step(const StepLaunch& L)
	{
		const StepArgs<T, R> a = step_args(L);
		switch (L.coll) {
			case COLL_CUM:
				switch (L.cum_flags) {
					case 0:
						return launch_parity<COLL_CUM, 0>(L, a);
					case CUM_ANTIALIAS:
						return launch_parity<COLL_CUM, CUM_ANTIALIAS>(L, a);
					case CUM_2017 | CUM_ANTIALIAS:
						return launch_parity<COLL_CUM, CUM_2017 | CUM_ANTIALIAS>(L, a);
					default:
						return cudaErrorInvalidValue;
				}
			case COLL_SRT:
				return launch_parity<COLL_SRT, 0>(L, a);
			case COLL_BGK:
				return launch_parity<COLL_BGK, 0>(L, a);
			case COLL_MRT:
				return launch_parity<COLL_MRT, 0>(L, a);
			default:
				return cudaErrorInvalidValue;
		}
	}

	// ---- A-B pull step
	template <int COLL, int CUMF>
	static cudaError_t ab_launch(const StepLaunch& L, const StepArgs<T, R>& a)
	{
		if (L.blocks_out)  // one partial-sum slot per warp
			*L.blocks_out = (long long) L.grid.x * L.grid.y * L.grid.z * ((L.block.x * L.block.y) / 32);
		if (L.dry_run)
			return cudaSuccess;
		if (L.macro || L.partials)
			ab_step_kernel<S, COLL, CUMF, true, ab_minb<R, COLL, CUMF, true>()>
				<<<L.grid, L.block, 0, L.stream>>>(a, (T*) L.f_out);
		else
			ab_step_kernel<S, COLL, CUMF, false, ab_minb<R, COLL, CUMF, false>()>
				<<<L.grid, L.block, 0, L.stream>>>(a, (T*) L.f_out);
		return cudaGetLastError();
	}

	static cudaError_t ab_step(const StepLaunch& L)
	{
		const StepArgs<T, R> a = step_args(L);
		switch (L.coll) {
			case COLL_CUM:
				switch (L.cum_flags) {
					case 0:
						return ab_launch<COLL_CUM, 0>(L, a);
					case CUM_ANTIALIAS:
						return ab_launch<COLL_CUM, CUM_ANTIALIAS>(L, a);
					case CUM_2017 | CUM_ANTIALIAS:
						return ab_launch<COLL_CUM, CUM_2017 | CUM_ANTIALIAS>(L, a);
					default:
						return cudaErrorInvalidValue;
				}
			case COLL_SRT:
				return ab_launch<COLL_SRT, 0>(L, a);
			case COLL_BGK:
				return ab_launch<COLL_BGK, 0>(L, a);
			case COLL_MRT:
				return ab_launch<COLL_MRT, 0>(L, a);
			default:
				return cudaErrorInvalidValue;
		}
	}

	// ---- ensemble of periodic lattices
	static void ens_entry(void* dst, const Geometry& g, const CollParamsD& pd, long long tile0)
	{
		EnsMember<T, R> e{};
		e.f = (T*) g.f;
		e.sq = g.sq;
		e.sy = g.sy;
		e.sz = g.sz;
		e.x0 = g.x0;
		e.X = g.X;
		e.Y = g.Y;
		e.Z = g.Z;
		e.n = g.X * g.Y * g.Z;
		e.tile0 = tile0;
		e.dx = make_fast_div(g.X);
		e.dy = make_fast_div(g.Y);
		e.p = make_coll_params<R>(pd);
		e.p2 = make_coll_params<F2>(pd);
		memcpy(dst, &e, sizeof(e));
	}

	template <int COLL, int CUMF, bool ODD, bool OUT, int TPB>
	static cudaError_t ens_launch(const EnsLaunch& L)
	{
		// the member's collision constants are read from the member table (kernel
		// parameters in the single-lattice kernel); the caps are the largest
		// that compile without spills (-Xptxas -v)
		constexpr int minb = sizeof(R) == 8 ? (TPB == 128 ? 2 : 1) : (TPB == 128 ? ENS_MINB128 : ENS_MINB128 / 2);
		auto kern = ens_step_kernel<S, COLL, CUMF, ODD, OUT, TPB, minb>;
		static int per_sm_cache[64] = {0};
		static int sms_cache[64] = {0};
		int dev = 0;
		cudaGetDevice(&dev);
		if (dev < 0 || dev >= 64)
			return cudaErrorInvalidDevice;
		if (per_sm_cache[dev] == 0) {
			int per_sm = 0, sms = 0;
			cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TPB, 0);
			if (e != cudaSuccess)
				return e;
			e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
			if (e != cudaSuccess)
				return e;
			if (per_sm < 1)
				return cudaErrorInvalidConfiguration;
			per_sm_cache[dev] = per_sm;
			sms_cache[dev] = sms;
		}
		long long grid = L.grid > 0 ? L.grid : (long long) per_sm_cache[dev] * sms_cache[dev];
		if (grid > L.ntiles)
			grid = L.ntiles;
		if (grid > 0x7fffffffLL)
			grid = 0x7fffffffLL;
		if (L.blocks_out)
			*L.blocks_out = grid;
		if (L.dry_run || grid < 1)
			return cudaSuccess;
		kern<<<(unsigned) grid, TPB, 0, L.stream>>>((const EnsMember<T, R>*) L.members, L.tile_member, L.ntiles, L.partials);
		return cudaGetLastError();
	}

	// grid policy 3: the persistent two-site kernel over tiles of 256 sites
	template <int COLL, int CUMF, bool ODD, bool OUT>
	static cudaError_t ens_pair_launch(const EnsLaunch& L)
	{
		if constexpr (sizeof(R) != 4) {
			(void) L;
			return cudaErrorNotSupported;
		}
		else {
			auto kern = ens_pair_kernel<S, COLL, CUMF, ODD, OUT, ENS_PAIR_MINB>;
			static int per_sm_cache[64] = {0};
			static int sms_cache[64] = {0};
			int dev = 0;
			cudaGetDevice(&dev);
			if (dev < 0 || dev >= 64)
				return cudaErrorInvalidDevice;
			if (per_sm_cache[dev] == 0) {
				int per_sm = 0, sms = 0;
				cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0);
				if (e != cudaSuccess)
					return e;
				e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
				if (e != cudaSuccess)
					return e;
				if (per_sm < 1)
					return cudaErrorInvalidConfiguration;
				per_sm_cache[dev] = per_sm;
				sms_cache[dev] = sms;
			}
			long long grid = (long long) per_sm_cache[dev] * sms_cache[dev];
			if (grid > L.ntiles)
				grid = L.ntiles;
			if (L.blocks_out)
				*L.blocks_out = grid;
			if (L.dry_run || grid < 1)
				return cudaSuccess;
			kern<<<(unsigned) grid, 128, 0, L.stream>>>((const EnsMember<T, float>*) L.members, L.tile_member, L.ntiles,
														L.partials);
			return cudaGetLastError();
		}
	}

	template <int COLL, int CUMF>
	static cudaError_t ens_dispatch(const EnsLaunch& L)
	{
		const bool out = L.partials != nullptr;
		if (L.pair) {
			if (L.tpb != 256)
				return cudaErrorNotSupported;
			if (L.odd)
				return out ? ens_pair_launch<COLL, CUMF, true, true>(L) : ens_pair_launch<COLL, CUMF, true, false>(L);
			return out ? ens_pair_launch<COLL, CUMF, false, true>(L) : ens_pair_launch<COLL, CUMF, false, false>(L);
		}
		if (L.tpb == 256) {
			if (L.odd)
				return out ? ens_launch<COLL, CUMF, true, true, 256>(L) : ens_launch<COLL, CUMF, true, false, 256>(L);
			return out ? ens_launch<COLL, CUMF, false, true, 256>(L) : ens_launch<COLL, CUMF, false, false, 256>(L);
		}
		if (L.tpb != 128)
			return cudaErrorInvalidValue;
		if (L.odd)
			return out ? ens_launch<COLL, CUMF, true, true, 128>(L) : ens_launch<COLL, CUMF, true, false, 128>(L);
		return out ? ens_launch<COLL, CUMF, false, true, 128>(L) : ens_launch<COLL, CUMF, false, false, 128>(L);
	}

	static cudaError_t ens_step(const EnsLaunch& L)
	{
		switch (L.coll) {
			case COLL_CUM:
				switch (L.cum_flags) {
					case 0:
						return ens_dispatch<COLL_CUM, 0>(L);
					case CUM_ANTIALIAS:
						return ens_dispatch<COLL_CUM, CUM_ANTIALIAS>(L);
					case CUM_2017 | CUM_ANTIALIAS:
						return ens_dispatch<COLL_CUM, CUM_2017 | CUM_ANTIALIAS>(L);
					default:
						return cudaErrorInvalidValue;
				}
			case COLL_SRT:
				return ens_dispatch<COLL_SRT, 0>(L);
			case COLL_BGK:
				return ens_dispatch<COLL_BGK, 0>(L);
			case COLL_MRT:
				return ens_dispatch<COLL_MRT, 0>(L);
			default:
				return cudaErrorInvalidValue;
		}
	}

	static cudaError_t init_eq(const Geometry& g, const InitSpec& spec, cudaStream_t st);
	static cudaError_t pack(const Geometry& g, void* dense, int dtype, int ghost, cudaStream_t st);
	static cudaError_t unpack(const Geometry& g, const void* dense, int dtype, int ghost, cudaStream_t st);
};

// equilibrium everywhere incl. the ghost layer (lbm_block.hpp:248-278); one
// thread per site of the (X+2)(Y+2)(Z+2) box.  The Taylor-Green field follows
// sim_NSE/sim_4.cu:145-163 at cell centres (i + 1/2 - N/2) with k = 2 pi / N.
template <typename S>
__global__ void init_eq_kernel(Geometry g, InitSpec spec)
{
	using R = typename S::R;
	using T = typename S::T;
	const long long nx = g.X + 2, ny = g.Y + 2, nz = g.Z + 2;
	const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
	if (i >= nx * ny * nz)
		return;
	const int x = (int) (i % nx) - 1;
	const int y = (int) ((i / nx) % ny) - 1;
	const int z = (int) (i / (nx * ny)) - 1;
	const bool interior = x >= 0 && x < g.X && y >= 0 && y < g.Y && z >= 0 && z < g.Z;
	double r = spec.rho0, u = spec.vx0, v = spec.vy0, w = spec.vz0;
	if (interior && spec.mode == 1) {
		const long long s = ((long long) z * g.Y + y) * g.X + x;
		r = spec.rho[s];
		u = spec.vx[s];
		v = spec.vy[s];
		w = spec.vz[s];
	}
	else if (interior && spec.mode == 2) {
		const double pi = 3.14159265358979323846;
		const double kx = 2 * pi / g.X, ky = 2 * pi / g.Y, kz = 2 * pi / g.Z;
		const double px = kx * (x + 0.5 - 0.5 * g.X), py = ky * (y + 0.5 - 0.5 * g.Y), pz = kz * (z + 0.5 - 0.5 * g.Z);
		const double u0 = spec.u0;
		u = u0 * sin(px) * cos(py) * cos(pz);
		v = -u0 * (kx / ky) * cos(px) * sin(py) * cos(pz);
		w = 0;
		r = spec.rho0 + 3 * (u0 * u0 / 16) * (cos(2 * px) + cos(2 * py)) * (cos(2 * pz) + 2);
	}
	else if (spec.mode == 2) {
		u = v = w = 0;
	}
	R f[27];
	set_equilibrium<R>(f, spec.eq, (R) r, (R) u, (R) v, (R) w);
	T* base = (T*) g.f + (long long) (z + 1) * g.sz + (long long) (y + 1) * g.sy + g.x0 + x;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			S::template store<q>(base + q * g.sq, f[q]);
		}
	);
}

// dense [27][nz][ny][nx] <-> storage
template <typename S, typename D, bool TO_DENSE>
__global__ void convert_kernel(Geometry g, D* dense, int ghost)
{
	using T = typename S::T;
	const int gh = ghost ? 1 : 0;
	const long long nx = g.X + 2 * gh, ny = g.Y + 2 * gh, nz = g.Z + 2 * gh;
	const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
	if (i >= nx * ny * nz)
		return;
	const int x = (int) (i % nx) - gh;
	const int y = (int) ((i / nx) % ny) - gh;
	const int z = (int) (i / (nx * ny)) - gh;
	T* base = (T*) g.f + (long long) (z + 1) * g.sz + (long long) (y + 1) * g.sy + g.x0 + x;
	const long long n = nx * ny * nz;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (TO_DENSE)
				dense[q * n + i] = (D) S::template load<q>(base + q * g.sq);
			else
				S::template store<q>(base + q * g.sq, (typename S::R) dense[q * n + i]);
		}
	);
}

template <typename S>
cudaError_t StorageUnit<S>::init_eq(const Geometry& g, const InitSpec& spec, cudaStream_t st)
{
	const long long n = (long long) (g.X + 2) * (g.Y + 2) * (g.Z + 2);
	const int bs = 128;
	init_eq_kernel<S><<<(unsigned) ((n + bs - 1) / bs), bs, 0, st>>>(g, spec);
	return cudaGetLastError();
}

template <typename S>
cudaError_t StorageUnit<S>::pack(const Geometry& g, void* dense, int dtype, int ghost, cudaStream_t st)
{
	const int gh = ghost ? 1 : 0;
	const long long n = (long long) (g.X + 2 * gh) * (g.Y + 2 * gh) * (g.Z + 2 * gh);
	const int bs = 128;
	const unsigned nb = (unsigned) ((n + bs - 1) / bs);
	if (dtype == 0)
		convert_kernel<S, double, true><<<nb, bs, 0, st>>>(g, (double*) dense, ghost);
	else
		convert_kernel<S, float, true><<<nb, bs, 0, st>>>(g, (float*) dense, ghost);
	return cudaGetLastError();
}

template <typename S>
cudaError_t StorageUnit<S>::unpack(const Geometry& g, const void* dense, int dtype, int ghost, cudaStream_t st)
{
	const int gh = ghost ? 1 : 0;
	const long long n = (long long) (g.X + 2 * gh) * (g.Y + 2 * gh) * (g.Z + 2 * gh);
	const int bs = 128;
	const unsigned nb = (unsigned) ((n + bs - 1) / bs);
	if (dtype == 0)
		convert_kernel<S, double, false><<<nb, bs, 0, st>>>(g, (double*) dense, ghost);
	else
		convert_kernel<S, float, false><<<nb, bs, 0, st>>>(g, (float*) dense, ghost);
	return cudaGetLastError();
}

}  // namespace lbm

#define LBM_DEFINE_STORAGE_OPS(FN, S, NAME)                                                                          \
	namespace lbm {                                                                                                  \
	const StorageOps& FN()                                                                                           \
	{                                                                                                                \
		static const StorageOps ops = {&StorageUnit<S>::step,                                                        \
									   &StorageUnit<S>::init_eq,                                                     \
									   &StorageUnit<S>::pack,                                                        \
									   &StorageUnit<S>::unpack,                                                      \
									   &StorageUnit<S>::ab_step,                                                     \
									   sizeof(EnsMember<typename S::T, typename S::R>),                              \
									   &StorageUnit<S>::ens_entry,                                                   \
									   &StorageUnit<S>::ens_step,                                                    \
									   &StorageUnit<S>::ade_step,                                                    \
									   (int) sizeof(typename S::R),                                                  \
									   (int) sizeof(typename S::T),                                                  \
									   NAME};                                                                        \
		return ops;                                                                                                  \
	}                                                                                                                \
	}
