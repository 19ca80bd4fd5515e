// Example collision plugins for the open COLL slot (csrc/plugin.cuh).
//
// Built by tnl-lbm_b200/build.py into lib/libtnl_lbm_b200_examples.so and
// registered at run time with lbm_register_collision (pytnl_lbm:
// register_collision).  Each struct plays the part of a reference collision
// struct such as D3Q27_SRT (include/lbm3d/d3q27/col_srt.h:7-15): a static
// collision() on one site's populations, inlined into the library's fused
// A-A step.
#include "../csrc/plugin.cuh"

namespace {

// The library's SRT collision through the plugin slot: the same update as
// LBM_COLL_SRT, bit for bit (one kernel body, aa_step_site).
struct SrtThroughPlugin
{
	template <typename R>
	__device__ static void collision(lbm::Site<R>& s, const lbm::CollParams<R>& p)
	{
		lbm::collide_srt(s, p);
	}
};

// No collision: the step only streams the populations and applies the
// boundary types of the map.
struct StreamingOnly
{
	template <typename R>
	__device__ static void collision(lbm::Site<R>&, const lbm::CollParams<R>&)
	{
	}
};

// Two-relaxation-time collision (I. Ginzburg, F. Verhaeghe, D. d'Humieres,
// Commun. Comput. Phys. 3 (2008) 427-478), a collision the reference does not
// ship: the parts of f_q symmetric and antisymmetric under q -> opp(q) relax
// towards those of the second-order equilibrium (eq.h:13-130) at
// omega+ = 1/tau, tau = 3 nu + 1/2, and at omega- fixed by the "magic"
// parameter Lambda = (1/omega+ - 1/2)(1/omega- - 1/2) = 3/16.  No force term.
struct TwoRelaxationTime
{
	template <typename R>
	__device__ static void collision(lbm::Site<R>& s, const lbm::CollParams<R>& p)
	{
		R feq[27];
		lbm::set_equilibrium(feq, lbm::EQ_SECOND_ORDER, s.rho, s.vx, s.vy, s.vz);
		const R wp = p.inv_tau;
		const R wm = R(1) / (R(3.0 / 16.0) / (p.tau - R(0.5)) + R(0.5));
		R out[27];
#pragma unroll
		for (int q = 0; q < 27; q++) {
			const int b = lbm::opp(q);
			const R sym = R(0.5) * ((s.f[q] + s.f[b]) - (feq[q] + feq[b]));
			const R anti = R(0.5) * ((s.f[q] - s.f[b]) - (feq[q] - feq[b]));
			out[q] = s.f[q] - wp * sym - wm * anti;
		}
#pragma unroll
		for (int q = 0; q < 27; q++)
			s.f[q] = out[q];
	}
};

}  // namespace

LBM_COLLISION_PLUGIN(lbm_example_srt, SrtThroughPlugin, LBM_PLUGIN_ALL_STORAGES)
LBM_COLLISION_PLUGIN(lbm_example_streaming, StreamingOnly,
					 LBM_PLUGIN_STORAGE(LBM_STORE_F64) | LBM_PLUGIN_STORAGE(LBM_STORE_F32))
LBM_COLLISION_PLUGIN(lbm_example_trt, TwoRelaxationTime,
					 LBM_PLUGIN_STORAGE(LBM_STORE_F64) | LBM_PLUGIN_STORAGE(LBM_STORE_F32))
