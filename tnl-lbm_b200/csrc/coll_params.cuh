// Collision-slot constants of one viscosity and force in the compute type,
// from the double-precision values the host computes once (launch.h).
#pragma once

#include "aa_kernels.cuh"
#include "collision.cuh"
#include "launch.h"

namespace lbm {

template <typename R>
inline CollParams<R> make_coll_params(const CollParamsD& d)
{
	CollParams<R> p{};
	const double w1 = d.w1;
	const double g = 1.0 / w1 - 0.5;
	p.nu = (R) d.nu;
	p.fx = (R) d.fx;
	p.fy = (R) d.fy;
	p.fz = (R) d.fz;
	p.hfx = (R) (0.5 * d.fx);
	p.hfy = (R) (0.5 * d.fy);
	p.hfz = (R) (0.5 * d.fz);
	p.w1 = (R) w1;
	p.one_m_w1 = (R) (1.0 - w1);
	p.k33 = (R) (3.0 * (1.0 - 0.5 * w1));
	p.hw1 = (R) (0.5 * w1);
	p.w1_3h = (R) (1.5 * w1);
	p.w1_3 = (R) (3.0 * w1);
	p.w3 = (R) d.w3;
	p.w4 = (R) d.w4;
	p.w5 = (R) d.w5;
	p.c43 = (R) (2.0 / 3.0 * g * d.A);
	p.c45 = (R) (-4.0 / 3.0 * g * d.A);
	p.cB = (R) (-1.0 / 3.0 * g * d.B);
	p.inv_tau = (R) (1.0 / d.tau);
	p.srt_force = (R) (1.0 - 0.5 / d.tau);
	p.bgk_force = (R) (1.0 - 0.5 * w1);
	p.tau = (R) d.tau;
	p.tau2 = (R) (d.tau * d.tau);
	p.eq = d.eq;
	return p;
}

// kernel arguments of one A-A step of storage S from the host's launch record
template <typename S>
inline StepArgs<typename S::T, typename S::R> make_step_args(const StepLaunch& L)
{
	using T = typename S::T;
	using R = typename S::R;
	StepArgs<T, R> a;
	a.f = (T*) L.g.f;
	a.sq = L.g.sq;
	a.sy = L.g.sy;
	a.sz = L.g.sz;
	a.x0 = L.g.x0;
	a.X = L.g.X;
	a.Y = L.g.Y;
	a.Z = L.g.Z;
	a.map = L.map;
	a.in_vx = (const R*) L.inflow[0];
	a.in_vy = (const R*) L.inflow[1];
	a.in_vz = (const R*) L.inflow[2];
	a.macro = (R*) L.macro;
	a.partials = L.partials;
	a.zwrap = L.distributed_z ? 0 : 1;
	a.p = make_coll_params<R>(L.p);
	return a;
}

}  // namespace lbm
