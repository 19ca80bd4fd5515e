// Collision plugins: a user's collision operator in the COLL slot of the
// fused A-A step.
//
// The reference composes the step kernel from compile-time plugins,
// LBM_CONFIG<TRAITS, KernelStruct, DATA, COLL, EQ, STREAMING, BC, MACRO>
// (include/lbm3d/defs.h:288-310); cudaLBMKernel (kernels.h:59-112) calls
// COLL::collision(KS) on the site's D3Q27_KernelStruct (defs.h:256-262:
// f[27], rho, vx, vy, vz, fx, fy, fz, lbmViscosity), e.g.
// D3Q27_SRT::collision (d3q27/col_srt.h:7-15).  A user adds a collision by
// writing such a struct.  Here the struct is
//
//     struct MyCollision
//     {
//         template <typename R>
//         __device__ static void collision(lbm::Site<R>& s, const lbm::CollParams<R>& p);
//     };
//
// where s.f[27] are the site's post-streaming populations in the reference's
// slot order, s.rho, s.vx, s.vy, s.vz its density and half-force-shifted
// velocity (common.h:31-49), s.ir = 1 / rho, and p the lattice's collision
// constants (p.nu the viscosity, p.fx..fz the body force, p.tau the SRT
// relaxation time, p.eq the equilibrium of lbm_desc.equilibrium).  The
// collision overwrites s.f with the post-collision populations.  R is the
// arithmetic type of the storage (double for LBM_STORE_F64, float else).
//
//     LBM_COLLISION_PLUGIN(my_collision_launcher, MyCollision, LBM_PLUGIN_ALL_STORAGES)
//
// compiled with nvcc for sm_100a into a shared library then defines the
// extern "C" launcher that lbm_register_collision takes.  The launcher runs
// the library's own per-site step (aa_step_site: A-A streaming, every
// boundary type of the map, macro and sums outputs) with the collision
// inlined, one thread per site, as the built-in collisions' direct kernel;
// with LBM_KERNEL_PAIR on a storage with FP32 arithmetic it runs the
// two-site kernels (pair.cuh) instead, with R = F2: two x-adjacent sites per
// thread on the packed FP32 instructions.  A collision written with the
// arithmetic operators and the library's helpers (set_equilibrium, opp,
// rcp, sqrt, fabs; no comparisons of R values) compiles for F2 as it does
// for float and double.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/tnl_lbm_b200.h"
#include "aa_kernels.cuh"
#include "coll_params.cuh"
#include "d3q27.cuh"
#include "launch.h"
#include "pair.cuh"

// storage sets of a plugin: bit LBM_STORE_* per storage it is compiled for
#define LBM_PLUGIN_STORAGE(st) (1u << (st))
#define LBM_PLUGIN_ALL_STORAGES 0xffu

namespace lbm {

// resident 128-thread blocks per SM: 128 registers per thread for FP32
// arithmetic, 256 for FP64 (the direct kernels' budgets for SRT and BGK)
template <typename R>
constexpr int plugin_minb()
{
	return sizeof(R) == 8 ? 2 : 4;
}

template <typename S, typename C, bool ODD, bool GENERAL, bool OUT>
__global__ void __launch_bounds__(128, plugin_minb<typename S::R>())
	aa_step_plugin_kernel(const StepArgs<typename S::T, typename S::R> a)
{
	using R = typename S::R;
	if constexpr (OUT)
		launch_dependents();
	aa_step_site<S, ODD, GENERAL, OUT>(a, [&](Site<R>& s) { C::template collision<R>(s, a.p); });
}

// a plugin's collision struct on the two-site kernels: 4 resident blocks per
// SM (128 registers), the budget of the built-in SRT and BGK
template <typename C>
struct PluginPairCollision
{
	template <typename R>
	__device__ static __forceinline__ void collision(Site<R>& s, const CollParams<R>& p)
	{
		C::template collision<R>(s, p);
	}
	template <typename T, bool ODD>
	static constexpr int pair_minb()
	{
		return 4;
	}
};

template <typename S, typename C, bool ODD, bool GENERAL>
cudaError_t plugin_launch(const StepLaunch& L)
{
	const StepArgs<typename S::T, typename S::R> a = make_step_args<S>(L);
	if (L.macro || L.partials)
		aa_step_plugin_kernel<S, C, ODD, GENERAL, true><<<L.grid, L.block, 0, L.stream>>>(a);
	else
		aa_step_plugin_kernel<S, C, ODD, GENERAL, false><<<L.grid, L.block, 0, L.stream>>>(a);
	return cudaGetLastError();
}

// one step of storage S: the launch shape and the partial-sum slots of the
// direct kernel (one per warp), then the even or odd, periodic or mapped kernel
template <typename S, typename C>
cudaError_t plugin_step(const StepLaunch& L)
{
	if constexpr (sizeof(typename S::R) == 4)
		if (L.kernel == KERNEL_PAIR) {
			const cudaError_t e = pair_step_with<S, PluginPairCollision<C>>(L);
			if (e != cudaErrorNotSupported)
				return e;
		}
	if (L.nothing_skipped)
		*L.nothing_skipped = false;
	if (L.blocks_out)
		*L.blocks_out = (long long) L.grid.x * L.grid.y * L.grid.z * ((L.block.x * L.block.y) / 32);
	if (L.dry_run)
		return cudaSuccess;
	const bool general = L.map != nullptr;
	if (L.odd)
		return general ? plugin_launch<S, C, true, true>(L) : plugin_launch<S, C, true, false>(L);
	return general ? plugin_launch<S, C, false, true>(L) : plugin_launch<S, C, false, false>(L);
}

template <typename C, unsigned STORAGES>
int32_t plugin_dispatch(const void* step, int32_t storage)
{
	if (storage < LBM_STORE_F64 || storage > LBM_STORE_I16S || !((STORAGES >> storage) & 1u))
		return (int32_t) cudaErrorNotSupported;
	if (!step)
		return 0;
	const StepLaunch& L = *static_cast<const StepLaunch*>(step);
	cudaError_t e = cudaErrorNotSupported;
	switch (storage) {
		case LBM_STORE_F64:
			if constexpr ((STORAGES & LBM_PLUGIN_STORAGE(LBM_STORE_F64)) != 0)
				e = plugin_step<StoreF64, C>(L);
			break;
		case LBM_STORE_F32:
			if constexpr ((STORAGES & LBM_PLUGIN_STORAGE(LBM_STORE_F32)) != 0)
				e = plugin_step<StoreF32, C>(L);
			break;
		case LBM_STORE_F32S:
			if constexpr ((STORAGES & LBM_PLUGIN_STORAGE(LBM_STORE_F32S)) != 0)
				e = plugin_step<StoreF32S, C>(L);
			break;
		case LBM_STORE_F16S:
			if constexpr ((STORAGES & LBM_PLUGIN_STORAGE(LBM_STORE_F16S)) != 0)
				e = plugin_step<StoreF16S, C>(L);
			break;
		case LBM_STORE_BF16S:
			if constexpr ((STORAGES & LBM_PLUGIN_STORAGE(LBM_STORE_BF16S)) != 0)
				e = plugin_step<StoreBF16S, C>(L);
			break;
		case LBM_STORE_F16SR:
			if constexpr ((STORAGES & LBM_PLUGIN_STORAGE(LBM_STORE_F16SR)) != 0)
				e = plugin_step<StoreF16SR, C>(L);
			break;
		case LBM_STORE_BF16SR:
			if constexpr ((STORAGES & LBM_PLUGIN_STORAGE(LBM_STORE_BF16SR)) != 0)
				e = plugin_step<StoreBF16SR, C>(L);
			break;
		case LBM_STORE_I16S:
			if constexpr ((STORAGES & LBM_PLUGIN_STORAGE(LBM_STORE_I16S)) != 0)
				e = plugin_step<StoreI16S, C>(L);
			break;
		default:
			break;
	}
	return (int32_t) e;
}

}  // namespace lbm

// Defines the extern "C" launcher SYMBOL of collision struct COLLISION for
// the storages of STORAGES (LBM_PLUGIN_STORAGE bits or LBM_PLUGIN_ALL_STORAGES).
#define LBM_COLLISION_PLUGIN(SYMBOL, COLLISION, STORAGES)                                \
	extern "C" __attribute__((visibility("default"))) int32_t SYMBOL(const void* step, \
																	 int32_t storage)   \
	{                                                                                    \
		return lbm::plugin_dispatch<COLLISION, (STORAGES)>(step, storage);               \
	}
