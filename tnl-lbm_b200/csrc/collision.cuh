// Per-site operators of the D3Q27 hot path for the sm_100a kernels: moments,
// equilibria and the collision operators that share TNL-LBM's COLL slot
// (cumulant, SRT, BGK, MRT-LES).  All routines work on a register-resident
// site (27 populations plus rho and u) and are fully unrolled, so every array
// index below is a compile-time constant.
//
// Per-viscosity quantities (omega1, the Geier 2017 rates omega3..5, A, B and
// their products) are computed once per lattice on the host
// (lbm_abi.cu: make_coll_params) instead of per site as the reference does in
// col_cum.h:195-228.
#pragma once

#include "d3q27.cuh"

namespace lbm {

template <typename R>
struct Site
{
	R f[27];
	R rho, ir, vx, vy, vz;	// ir = 1 / rho
};

// collision-slot identifiers (runtime values of lbm_desc.collision)
enum Coll : int
{
	COLL_CUM = 0,
	COLL_SRT = 1,
	COLL_BGK = 2,
	COLL_MRT = 3
};
// cumulant variant bits (USE_GEIER_CUM_2017 / USE_GEIER_CUM_ANTIALIAS, defs.h:312-315)
enum : int
{
	CUM_2017 = 1,
	CUM_ANTIALIAS = 2
};
// equilibrium identifiers: D3Q27_EQ (eq.h) and D3Q27_EQ_INV_CUM (eq_inv_cum.h)
enum : int
{
	EQ_SECOND_ORDER = 0,
	EQ_INV_CUM = 1
};

// per-lattice constants of the collision slot, in the compute type
template <typename R>
struct CollParams
{
	R nu;
	R fx, fy, fz;
	R hfx, hfy, hfz;  // half force for the velocity shift (common.h:40-48)
	// cumulant
	R w1, one_m_w1;
	R k33;			  // 3 (1 - omega1/2)
	R hw1, w1_3h, w1_3;	 // omega1/2, 3 omega1/2, 3 omega1
	R w3, w4, w5;	  // Geier 2017 third/fourth-order rates
	R c43, c45, cB;	  // (2/3) g A, -(4/3) g A, -(1/3) g B with g = 1/omega1 - 1/2
	// SRT / BGK / MRT
	R inv_tau, srt_force;  // 1/tau, 1 - 1/(2 tau)
	R bgk_force;		   // 1 - omega1/2
	R tau, tau2;		   // MRT-LES: tau and tau^2
	int eq;				   // equilibrium used by SRT and by equilibrium BCs
};

template <typename R>
__device__ __forceinline__ R rcp(R x)
{
	return R(1) / x;
}
template <>
__device__ __forceinline__ float rcp<float>(float x)
{
	return __frcp_rn(x);
}
// division where a few ulp do not matter (limiter weights)
template <typename R>
__device__ __forceinline__ R div_approx(R a, R b)
{
	return a / b;
}
template <>
__device__ __forceinline__ float div_approx<float>(float a, float b)
{
	return __fdividef(a, b);
}

// density and velocity with the half-force shift; pairwise summation order of
// common.h:31-49 (Geier 2015 Appendix J)
template <typename R>
__device__ __forceinline__ void density_velocity(Site<R>& s, const CollParams<R>& p)
{
	const R* f = s.f;
	s.rho = ((((f[PPP] + f[MMM]) + (f[PMP] + f[MPM])) + ((f[PPM] + f[MMP]) + (f[MPP] + f[PMM])))
			 + (((f[ZPP] + f[ZMM]) + (f[ZPM] + f[ZMP])) + ((f[PZP] + f[MZM]) + (f[PZM] + f[MZP]))
				+ ((f[PPZ] + f[MMZ]) + (f[PMZ] + f[MPZ])))
			 + ((f[PZZ] + f[MZZ]) + (f[ZPZ] + f[ZMZ]) + (f[ZZP] + f[ZZM])))
		  + f[ZZZ];
	s.ir = rcp(s.rho);
	s.vz = ((((f[PPP] - f[MMM]) + (f[MPP] - f[PMM])) + ((f[PMP] - f[MPM]) + (f[MMP] - f[PPM])))
			+ (((f[ZPP] - f[ZMM]) + (f[ZMP] - f[ZPM])) + ((f[PZP] - f[MZM]) + (f[MZP] - f[PZM]))) + (f[ZZP] - f[ZZM]) + p.hfz)
		 * s.ir;
	s.vx = ((((f[PPP] - f[MMM]) + (f[PMP] - f[MPM])) + ((f[PPM] - f[MMP]) + (f[PMM] - f[MPP])))
			+ (((f[PZP] - f[MZM]) + (f[PZM] - f[MZP])) + ((f[PPZ] - f[MMZ]) + (f[PMZ] - f[MPZ]))) + (f[PZZ] - f[MZZ]) + p.hfx)
		 * s.ir;
	s.vy = ((((f[PPP] - f[MMM]) + (f[PPM] - f[MMP])) + ((f[MPP] - f[PMM]) + (f[MPM] - f[PMP])))
			+ (((f[PPZ] - f[MMZ]) + (f[MPZ] - f[PMZ])) + ((f[ZPP] - f[ZMM]) + (f[ZPM] - f[ZMP]))) + (f[ZPZ] - f[ZMZ]) + p.hfy)
		 * s.ir;
}

// ---------------------------------------------------------------------------
// equilibria, direction by direction
// ---------------------------------------------------------------------------

// second-order equilibrium w_q rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u^2) (eq.h:13-130)
template <int Q, typename R>
__device__ __forceinline__ R eq_second(R rho, R vx, R vy, R vz, R usq)
{
	const R cu = R(cx(Q)) * vx + R(cy(Q)) * vy + R(cz(Q)) * vz;
	return R(weight(Q)) * rho * ((R(1) - R(1.5) * usq + R(3) * cu) + R(4.5) * cu * cu);
}

// per-axis factor of the factorised equilibrium (eq_inv_cum.h:24-136)
template <int C, typename R>
__device__ __forceinline__ R inv_cum_axis(R v, R v3v)	// v3v = 3 v^2
{
	return C == 0 ? v3v - R(2) : (C > 0 ? v3v + R(3) * v + R(1) : v3v - R(3) * v + R(1));
}
template <int Q>
__host__ __device__ constexpr double inv_cum_coef()
{
	return nnz(Q) == 0 ? -1.0 / 27.0 : nnz(Q) == 1 ? 1.0 / 54.0 : nnz(Q) == 2 ? -1.0 / 108.0 : 1.0 / 216.0;
}
template <int Q, typename R>
__device__ __forceinline__ R eq_inv_cum(R rho, R vx, R vy, R vz, R vx3, R vy3, R vz3)
{
	return R(inv_cum_coef<Q>()) * rho
		 * (inv_cum_axis<cx(Q)>(vx, vx3) * inv_cum_axis<cy(Q)>(vy, vy3) * inv_cum_axis<cz(Q)>(vz, vz3));
}

template <typename R>
__device__ __forceinline__ void set_equilibrium(R* f, int eq, R rho, R vx, R vy, R vz)
{
	if (eq == EQ_INV_CUM) {
		const R vx3 = R(3) * vx * vx, vy3 = R(3) * vy * vy, vz3 = R(3) * vz * vz;
#pragma unroll
		for (int q = 0; q < 27; q++) {
			// explicit instantiation per direction
			switch (q) {
#define LBM_EQ_CASE(Q) \
	case Q: f[Q] = eq_inv_cum<Q>(rho, vx, vy, vz, vx3, vy3, vz3); break;
				LBM_EQ_CASE(0) LBM_EQ_CASE(1) LBM_EQ_CASE(2) LBM_EQ_CASE(3) LBM_EQ_CASE(4) LBM_EQ_CASE(5)
				LBM_EQ_CASE(6) LBM_EQ_CASE(7) LBM_EQ_CASE(8) LBM_EQ_CASE(9) LBM_EQ_CASE(10) LBM_EQ_CASE(11)
				LBM_EQ_CASE(12) LBM_EQ_CASE(13) LBM_EQ_CASE(14) LBM_EQ_CASE(15) LBM_EQ_CASE(16) LBM_EQ_CASE(17)
				LBM_EQ_CASE(18) LBM_EQ_CASE(19) LBM_EQ_CASE(20) LBM_EQ_CASE(21) LBM_EQ_CASE(22) LBM_EQ_CASE(23)
				LBM_EQ_CASE(24) LBM_EQ_CASE(25) LBM_EQ_CASE(26)
#undef LBM_EQ_CASE
			}
		}
	}
	else {
		const R usq = vx * vx + vy * vy + vz * vz;
#pragma unroll
		for (int q = 0; q < 27; q++) {
			switch (q) {
#define LBM_EQ_CASE(Q) \
	case Q: f[Q] = eq_second<Q>(rho, vx, vy, vz, usq); break;
				LBM_EQ_CASE(0) LBM_EQ_CASE(1) LBM_EQ_CASE(2) LBM_EQ_CASE(3) LBM_EQ_CASE(4) LBM_EQ_CASE(5)
				LBM_EQ_CASE(6) LBM_EQ_CASE(7) LBM_EQ_CASE(8) LBM_EQ_CASE(9) LBM_EQ_CASE(10) LBM_EQ_CASE(11)
				LBM_EQ_CASE(12) LBM_EQ_CASE(13) LBM_EQ_CASE(14) LBM_EQ_CASE(15) LBM_EQ_CASE(16) LBM_EQ_CASE(17)
				LBM_EQ_CASE(18) LBM_EQ_CASE(19) LBM_EQ_CASE(20) LBM_EQ_CASE(21) LBM_EQ_CASE(22) LBM_EQ_CASE(23)
				LBM_EQ_CASE(24) LBM_EQ_CASE(25) LBM_EQ_CASE(26)
#undef LBM_EQ_CASE
			}
		}
	}
}

// ---------------------------------------------------------------------------
// cumulant collision (col_cum.h:13-511; Geier 2015 / Geier 2017)
// ---------------------------------------------------------------------------

// cube index of a direction or of a moment triple (orders or positions 0..2)
__host__ __device__ constexpr int ci(int i, int j, int k)
{
	return i * 9 + j * 3 + k;
}

// forward chimera transform of a line (m, z, p) about velocity u (Eqs 6-14)
template <typename R>
__device__ __forceinline__ void chim_fwd(R& m, R& z, R& p, R u, R u2)
{
	const R s = p + m, d = p - m;
	const R k0 = s + z;
	const R k1 = d - u * k0;
	const R k2 = s - R(2) * u * d + u2 * k0;
	m = k0;
	z = k1;
	p = k2;
}

// backward chimera transform (Eqs 88-96 of Geier 2015), written through the
// sum s = v+ + v- = k0 u^2 + 2 u k1 + k2 and the difference d = v+ - v- =
// u k0 + k1 of the outer values: v0 = k0 - s, v+- = (s +- d) / 2.  The three
// values then add up to k0 and their first moment is d up to one rounding
// each, the mass and momentum the line carries, where the term-by-term form
// of the paper rounds every term separately.
template <typename R>
__device__ __forceinline__ void chim_bwd(R& a, R& b, R& c, R u, R u2)
{
	const R k0 = a, k1 = b, k2 = c;
	const R s = k0 * u2 + (R(2) * u * k1 + k2);
	const R hd = R(0.5) * (u * k0 + k1);
	a = s * R(0.5) - hd;
	b = k0 - s;
	c = s * R(0.5) + hd;
}

template <typename R, int FLAGS>
__device__ __forceinline__ void collide_cumulant(Site<R>& s, const CollParams<R>& p)
{
	constexpr bool v2017 = (FLAGS & CUM_2017) != 0;
	constexpr bool antialias = (FLAGS & CUM_ANTIALIAS) != 0;
	const R rho = s.rho, ir = s.ir, vx = s.vx, vy = s.vy, vz = s.vz;
	const R vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;

	R M[27];
#pragma unroll
	for (int q = 0; q < 27; q++)
		M[ci(cx(q) + 1, cy(q) + 1, cz(q) + 1)] = s.f[q];
#pragma unroll
	for (int i = 0; i < 3; i++)
#pragma unroll
		for (int j = 0; j < 3; j++)
			chim_fwd(M[ci(i, j, 0)], M[ci(i, j, 1)], M[ci(i, j, 2)], vz, vz2);
#pragma unroll
	for (int i = 0; i < 3; i++)
#pragma unroll
		for (int k = 0; k < 3; k++)
			chim_fwd(M[ci(i, 0, k)], M[ci(i, 1, k)], M[ci(i, 2, k)], vy, vy2);
#pragma unroll
	for (int j = 0; j < 3; j++)
#pragma unroll
		for (int k = 0; k < 3; k++)
			chim_fwd(M[ci(0, j, k)], M[ci(1, j, k)], M[ci(2, j, k)], vx, vx2);

	// central moments M[ci(a,b,c)] = k_abc; cumulants of order <= 3 equal them
	const R k000 = M[ci(0, 0, 0)];
	const R C110 = M[ci(1, 1, 0)], C101 = M[ci(1, 0, 1)], C011 = M[ci(0, 1, 1)];
	const R C200 = M[ci(2, 0, 0)], C020 = M[ci(0, 2, 0)], C002 = M[ci(0, 0, 2)];

	// velocity derivatives for the anti-aliasing terms (col_cum.h:234-250)
	R Dxu = 0, Dyv = 0, Dzw = 0, DxvDyu = 0, DxwDzu = 0, DywDzv = 0;
	if (antialias) {
		// omega2 = 1
		Dxu = -p.hw1 * ir * (R(2) * C200 - C020 - C002) - R(0.5) * ir * (C200 + C020 + C002 - (rho - R(1)));
		Dyv = Dxu + p.w1_3h * ir * (C200 - C020);
		Dzw = Dxu + p.w1_3h * ir * (C200 - C002);
		DxvDyu = -p.w1_3 * ir * C110;
		DxwDzu = -p.w1_3 * ir * C101;
		DywDzv = -p.w1_3 * ir * C011;
	}

	// second order (col_cum.h:231-259), omega2 = 1
	const R Cs110 = p.one_m_w1 * C110;
	const R Cs101 = p.one_m_w1 * C101;
	const R Cs011 = p.one_m_w1 * C011;
	const R e33 = p.one_m_w1 * (C200 - C020) - p.k33 * rho * (vx2 * Dxu - vy2 * Dyv);
	const R e34 = p.one_m_w1 * (C200 - C002) - p.k33 * rho * (vx2 * Dxu - vz2 * Dzw);
	const R e35 = k000 - R(1.5) * rho * (vx2 * Dxu + vy2 * Dyv + vz2 * Dzw);
	const R third = R(1.0 / 3.0);
	const R Cs200 = third * (e33 + e34 + e35);
	const R Cs020 = third * (e34 + e35 - R(2) * e33);
	const R Cs002 = third * (e33 + e35 - R(2) * e34);

	R Cs120 = 0, Cs102 = 0, Cs210 = 0, Cs012 = 0, Cs021 = 0, Cs201 = 0, Cs111 = 0;
	R ks211, ks121, ks112, ks220, ks022, ks202, ks122 = 0, ks212 = 0, ks221 = 0, ks222;
	if (v2017) {
		const R C120 = M[ci(1, 2, 0)], C102 = M[ci(1, 0, 2)], C210 = M[ci(2, 1, 0)];
		const R C012 = M[ci(0, 1, 2)], C201 = M[ci(2, 0, 1)], C021 = M[ci(0, 2, 1)];
		const R C111 = M[ci(1, 1, 1)];
		// fourth-order cumulants (Eqs 51-54 of Geier 2015)
		const R C211 = M[ci(2, 1, 1)] - (C200 * C011 + R(2) * C101 * C110) * ir;
		const R C121 = M[ci(1, 2, 1)] - (C020 * C101 + R(2) * C110 * C011) * ir;
		const R C112 = M[ci(1, 1, 2)] - (C002 * C110 + R(2) * C011 * C101) * ir;
		const R C220 = M[ci(2, 2, 0)] - (C020 * C200 + R(2) * C110 * C110) * ir;
		const R C022 = M[ci(0, 2, 2)] - (C002 * C020 + R(2) * C011 * C011) * ir;
		const R C202 = M[ci(2, 0, 2)] - (C200 * C002 + R(2) * C101 * C101) * ir;
		// fifth- and sixth-order cumulants relax fully (omega9 = omega10 = 1), so
		// only the fourth-order ones and below are needed (col_cum.h:294-297)

		// limited third-order rates (col_cum.h:203-216), lambda = 0.01
		const R lam_rho = R(0.01) * rho;
		const R a1 = C120 + C102, a2 = C210 + C012, a3 = C201 + C021;
		const R b1 = C120 - C102, b2 = C210 - C012, b3 = C201 - C021;
		const R A1 = fabs(a1), A2 = fabs(a2), A3 = fabs(a3), B1 = fabs(b1), B2 = fabs(b2), B3 = fabs(b3), D = fabs(C111);
		const R w120p102 = p.w3 + (R(1) - p.w3) * div_approx(A1, lam_rho + A1);
		const R w210p012 = p.w3 + (R(1) - p.w3) * div_approx(A2, lam_rho + A2);
		const R w201p021 = p.w3 + (R(1) - p.w3) * div_approx(A3, lam_rho + A3);
		const R w120m102 = p.w4 + (R(1) - p.w4) * div_approx(B1, lam_rho + B1);
		const R w210m012 = p.w4 + (R(1) - p.w4) * div_approx(B2, lam_rho + B2);
		const R w201m021 = p.w4 + (R(1) - p.w4) * div_approx(B3, lam_rho + B3);
		const R w111 = p.w5 + (R(1) - p.w5) * div_approx(D, lam_rho + D);
		// third order (Eqs 117-122, 42)
		const R e117 = (R(1) - w120p102) * a1;
		const R e118 = (R(1) - w210p012) * a2;
		const R e119 = (R(1) - w201p021) * a3;
		const R e120 = (R(1) - w120m102) * b1;
		const R e121 = (R(1) - w210m012) * b2;
		const R e122 = (R(1) - w201m021) * b3;
		Cs120 = R(0.5) * (e120 + e117);
		Cs102 = R(0.5) * (e117 - e120);
		Cs210 = R(0.5) * (e121 + e118);
		Cs012 = R(0.5) * (e118 - e121);
		Cs021 = R(0.5) * (e119 - e122);
		Cs201 = R(0.5) * (e122 + e119);
		Cs111 = (R(1) - w111) * C111;
		// fourth order (Eqs 43-48), omega6 = omega7 = omega8 = 1
		(void) C220;
		(void) C022;
		(void) C202;
		(void) C211;
		(void) C121;
		(void) C112;
		const R aA = p.c43 * rho, aB = p.cB * rho;
		const R e43 = aA * (Dxu - R(2) * Dyv + Dzw);
		const R e44 = aA * (Dxu + Dyv - R(2) * Dzw);
		const R e45 = p.c45 * rho * (Dxu + Dyv + Dzw);
		const R Cs220 = third * (e43 + e44 + e45);
		const R Cs202 = third * (e45 - e43);
		const R Cs022 = third * (e45 - e44);
		const R Cs211 = aB * DywDzv;
		const R Cs121 = aB * DxwDzu;
		const R Cs112 = aB * DxvDyu;
		// back to central moments (Eqs 81-84); Cs221, Cs212, Cs122, Cs222 = 0
		ks211 = Cs211 + (Cs200 * Cs011 + R(2) * Cs101 * Cs110) * ir;
		ks121 = Cs121 + (Cs020 * Cs101 + R(2) * Cs110 * Cs011) * ir;
		ks112 = Cs112 + (Cs002 * Cs110 + R(2) * Cs011 * Cs101) * ir;
		ks220 = Cs220 + (Cs020 * Cs200 + R(2) * Cs110 * Cs110) * ir;
		ks022 = Cs022 + (Cs002 * Cs020 + R(2) * Cs011 * Cs011) * ir;
		ks202 = Cs202 + (Cs200 * Cs002 + R(2) * Cs101 * Cs101) * ir;
		ks122 = (Cs020 * Cs102 + Cs002 * Cs120 + R(4) * Cs011 * Cs111 + R(2) * (Cs110 * Cs012 + Cs101 * Cs021)) * ir;
		ks212 = (Cs002 * Cs210 + Cs200 * Cs012 + R(4) * Cs101 * Cs111 + R(2) * (Cs011 * Cs201 + Cs110 * Cs102)) * ir;
		ks221 = (Cs200 * Cs021 + Cs020 * Cs201 + R(4) * Cs110 * Cs111 + R(2) * (Cs101 * Cs120 + Cs011 * Cs210)) * ir;
		ks222 = (R(4) * Cs111 * Cs111 + Cs200 * ks022 + Cs020 * ks202 + Cs002 * ks220
				 + R(4) * (Cs011 * ks211 + Cs101 * ks121 + Cs110 * ks112) + R(2) * (Cs120 * Cs102 + Cs210 * Cs012 + Cs201 * Cs021))
				  * ir
			  - (R(16) * Cs110 * Cs101 * Cs011 + R(4) * (Cs101 * Cs101 * Cs020 + Cs011 * Cs011 * Cs200 + Cs110 * Cs110 * Cs002)
				 + R(2) * Cs200 * Cs020 * Cs002)
					* ir * ir;
	}
	else {
		// default variant (col_cum.h:330-366)
		ks211 = (Cs200 * Cs011 + R(2) * Cs101 * Cs110) * ir;
		ks121 = (Cs020 * Cs101 + R(2) * Cs110 * Cs011) * ir;
		ks112 = (Cs002 * Cs110 + R(2) * Cs011 * Cs101) * ir;
		ks220 = (Cs020 * Cs200 + R(2) * Cs110 * Cs110) * ir;
		ks022 = (Cs002 * Cs020 + R(2) * Cs011 * Cs011) * ir;
		ks202 = (Cs200 * Cs002 + R(2) * Cs101 * Cs101) * ir;
		ks222 = (Cs200 * ks022 + Cs020 * ks202 + Cs002 * ks220 + R(4) * (Cs011 * ks211 + Cs101 * ks121 + Cs110 * ks112)) * ir
			  - (R(16) * Cs110 * Cs101 * Cs011 + R(4) * (Cs101 * Cs101 * Cs020 + Cs011 * Cs011 * Cs200 + Cs110 * Cs110 * Cs002)
				 + R(2) * Cs200 * Cs020 * Cs002)
					* ir * ir;
	}

	// post-collision central moments; first moments flipped (col_cum.h:369-373)
	M[ci(1, 0, 0)] = -M[ci(1, 0, 0)];
	M[ci(0, 1, 0)] = -M[ci(0, 1, 0)];
	M[ci(0, 0, 1)] = -M[ci(0, 0, 1)];
	M[ci(1, 1, 0)] = Cs110;
	M[ci(1, 0, 1)] = Cs101;
	M[ci(0, 1, 1)] = Cs011;
	M[ci(2, 0, 0)] = Cs200;
	M[ci(0, 2, 0)] = Cs020;
	M[ci(0, 0, 2)] = Cs002;
	M[ci(1, 2, 0)] = Cs120;
	M[ci(1, 0, 2)] = Cs102;
	M[ci(2, 1, 0)] = Cs210;
	M[ci(0, 1, 2)] = Cs012;
	M[ci(2, 0, 1)] = Cs201;
	M[ci(0, 2, 1)] = Cs021;
	M[ci(1, 1, 1)] = Cs111;
	M[ci(2, 1, 1)] = ks211;
	M[ci(1, 2, 1)] = ks121;
	M[ci(1, 1, 2)] = ks112;
	M[ci(2, 2, 0)] = ks220;
	M[ci(0, 2, 2)] = ks022;
	M[ci(2, 0, 2)] = ks202;
	M[ci(1, 2, 2)] = ks122;
	M[ci(2, 1, 2)] = ks212;
	M[ci(2, 2, 1)] = ks221;
	M[ci(2, 2, 2)] = ks222;

#pragma unroll
	for (int j = 0; j < 3; j++)
#pragma unroll
		for (int k = 0; k < 3; k++)
			chim_bwd(M[ci(0, j, k)], M[ci(1, j, k)], M[ci(2, j, k)], vx, vx2);
#pragma unroll
	for (int i = 0; i < 3; i++)
#pragma unroll
		for (int k = 0; k < 3; k++)
			chim_bwd(M[ci(i, 0, k)], M[ci(i, 1, k)], M[ci(i, 2, k)], vy, vy2);
#pragma unroll
	for (int i = 0; i < 3; i++)
#pragma unroll
		for (int j = 0; j < 3; j++)
			chim_bwd(M[ci(i, j, 0)], M[ci(i, j, 1)], M[ci(i, j, 2)], vz, vz2);
#pragma unroll
	for (int q = 0; q < 27; q++)
		s.f[q] = M[ci(cx(q) + 1, cy(q) + 1, cz(q) + 1)];
}

// ---------------------------------------------------------------------------
// SRT, BGK, MRT-LES through the same slot
// ---------------------------------------------------------------------------

// Guo-like forcing term S_q = 3 (c_q - u).F / rho (col_srt.h:22-48)
template <int Q, typename R>
__device__ __forceinline__ R force_term(const Site<R>& s, const CollParams<R>& p, R irho)
{
	return R(3) * ((R(cx(Q)) - s.vx) * p.fx + (R(cy(Q)) - s.vy) * p.fy + (R(cz(Q)) - s.vz) * p.fz) * irho;
}

// 1 / rho for the SRT forcing, 1 where rho = 0 (col_srt.h:19, the ADE case)
template <typename R>
__device__ __forceinline__ R inv_rho_or_one(const Site<R>& s)
{
	return s.rho == R(0) ? R(1) : s.ir;
}

// textbook BGK (col_srt.h:14-105)
template <typename R>
__device__ __forceinline__ void collide_srt(Site<R>& s, const CollParams<R>& p)
{
	R feq[27];
	set_equilibrium(feq, p.eq, s.rho, s.vx, s.vy, s.vz);
	const R irho = inv_rho_or_one(s);
#pragma unroll
	for (int q = 0; q < 27; q++) {
		R S;
		switch (q) {
#define LBM_S(Q) \
	case Q: S = force_term<Q>(s, p, irho); break;
			LBM_S(0) LBM_S(1) LBM_S(2) LBM_S(3) LBM_S(4) LBM_S(5) LBM_S(6) LBM_S(7) LBM_S(8) LBM_S(9) LBM_S(10) LBM_S(11)
			LBM_S(12) LBM_S(13) LBM_S(14) LBM_S(15) LBM_S(16) LBM_S(17) LBM_S(18) LBM_S(19) LBM_S(20) LBM_S(21) LBM_S(22)
			LBM_S(23) LBM_S(24) LBM_S(25) LBM_S(26)
#undef LBM_S
		}
		s.f[q] += (feq[q] - s.f[q]) * p.inv_tau + p.srt_force * S * feq[q];
	}
}

// Geier's improved BGK with factorised equilibrium (col_bgk.h:18-144)
template <typename R>
__device__ __forceinline__ void collide_bgk(Site<R>& s, const CollParams<R>& p)
{
	const R third = R(1.0 / 3.0);
	const R Xz = third - R(1) + s.vx * s.vx, Xp = R(-0.5) * (Xz + R(1) + s.vx), Xm = Xp + s.vx;
	const R Yz = third - R(1) + s.vy * s.vy, Yp = R(-0.5) * (Yz + R(1) + s.vy), Ym = Yp + s.vy;
	const R Zz = third - R(1) + s.vz * s.vz, Zp = R(-0.5) * (Zz + R(1) + s.vz), Zm = Zp + s.vz;
#pragma unroll
	for (int q = 0; q < 27; q++) {
		const R X = cx(q) == 0 ? Xz : (cx(q) > 0 ? Xp : Xm);
		const R Y = cy(q) == 0 ? Yz : (cy(q) > 0 ? Yp : Ym);
		const R Z = cz(q) == 0 ? Zz : (cz(q) > 0 ? Zp : Zm);
		R S;
		switch (q) {
#define LBM_S(Q) \
	case Q: S = force_term<Q>(s, p, s.ir); break;
			LBM_S(0) LBM_S(1) LBM_S(2) LBM_S(3) LBM_S(4) LBM_S(5) LBM_S(6) LBM_S(7) LBM_S(8) LBM_S(9) LBM_S(10) LBM_S(11)
			LBM_S(12) LBM_S(13) LBM_S(14) LBM_S(15) LBM_S(16) LBM_S(17) LBM_S(18) LBM_S(19) LBM_S(20) LBM_S(21) LBM_S(22)
			LBM_S(23) LBM_S(24) LBM_S(25) LBM_S(26)
#undef LBM_S
		}
		const R feq = -s.rho * X * Y * Z;
		s.f[q] += (feq - s.f[q]) * p.w1 + p.bgk_force * S * feq;
	}
}

// MRT-LES: Smagorinsky-relaxed second moments, populations rebuilt from
// rho, u and the relaxed tensor (col_mrt.h:14-141)
template <typename R>
__device__ __forceinline__ void collide_mrt(Site<R>& s, const CollParams<R>& p)
{
	R Pxx = 0, Pyy = 0, Pzz = 0, Pxy = 0, Pxz = 0, Pyz = 0;
#pragma unroll
	for (int q = 0; q < 27; q++) {
		const R v = s.f[q];
		if (cx(q) != 0)
			Pxx += v;
		if (cy(q) != 0)
			Pyy += v;
		if (cz(q) != 0)
			Pzz += v;
		if (cx(q) * cy(q) != 0)
			Pxy += R(cx(q) * cy(q)) * v;
		if (cx(q) * cz(q) != 0)
			Pxz += R(cx(q) * cz(q)) * v;
		if (cy(q) * cz(q) != 0)
			Pyz += R(cy(q) * cz(q)) * v;
	}
	const R rho = s.rho, vx = s.vx, vy = s.vy, vz = s.vz;
	const R third = R(1.0 / 3.0);
	const R Pnxx = Pxx - rho * (third + vx * vx);
	const R Pnyy = Pyy - rho * (third + vy * vy);
	const R Pnzz = Pzz - rho * (third + vz * vz);
	const R Pnxz = Pxz - rho * vx * vz;
	const R Pnxy = Pxy - rho * vx * vy;
	const R Pnyz = Pyz - rho * vy * vz;
	const R Q = R(2) * (Pnxx * Pnxx + Pnyy * Pnyy + Pnzz * Pnzz + R(2) * (Pnxy * Pnxy + Pnxz * Pnxz + Pnyz * Pnyz));
	const R omega = R(2) / (sqrt(p.tau2 + R(2 * 0.0342 * 9.0) * sqrt(Q) * s.ir) + p.tau);
	Pxx -= omega * Pnxx;
	Pyy -= omega * Pnyy;
	Pzz -= omega * Pnzz;
	Pxy -= omega * Pnxy;
	Pxz -= omega * Pnxz;
	Pyz -= omega * Pnyz;
	const R P2 = Pxx + Pyy + Pzz;
#pragma unroll
	for (int q = 0; q < 27; q++) {
		const R cu = vx * R(cx(q)) + vy * R(cy(q)) + vz * R(cz(q));
		const R cc = Pxx * R(cx(q) * cx(q)) + Pyy * R(cy(q) * cy(q)) + Pzz * R(cz(q) * cz(q))
				   + R(2) * (Pxy * R(cx(q) * cy(q)) + Pxz * R(cx(q) * cz(q)) + Pyz * R(cy(q) * cz(q)));
		s.f[q] = R(weight(q)) * (rho * ((R(2.5) - R(1.5) * R(nnz(q))) + R(3) * cu) + R(4.5) * cc - R(1.5) * P2);
	}
}

template <typename R, int COLL, int CUMF>
__device__ __forceinline__ void collide(Site<R>& s, const CollParams<R>& p)
{
	if constexpr (COLL == COLL_CUM)
		collide_cumulant<R, CUMF>(s, p);
	else if constexpr (COLL == COLL_SRT)
		collide_srt(s, p);
	else if constexpr (COLL == COLL_BGK)
		collide_bgk(s, p);
	else
		collide_mrt(s, p);
}

}  // namespace lbm
