/*
 * CPU restatement of TNL-LBM's D3Q27 A-A hot path (the oracle port).
 *
 * TEST INFRASTRUCTURE ONLY: the test-suite, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py use this library as a checker.  The product
 * library never links it and no product code path calls it.
 *
 * The file is compiled twice (REAL=double, suffix _f64; REAL=float, suffix
 * _f32) into oracle/_build/liboracle.so by oracle/Makefile.  Every routine
 * cites the reference file:line it restates (paths inside TNL-LBM).  Where the
 * reference's evaluation order determines the rounded result (pairwise density
 * sums, factor order of the equilibria, chimera transforms), the same order is
 * kept so that the FP64 build agrees with the reference's own code to the last
 * bit or nearly so; the structure (table-driven directions, generic chimera
 * passes over a 3x3x3 moment cube) is this project's own.
 *
 * Population storage: canonical order [27][Z+2][Y+2][X+2], x fastest, with one
 * ghost layer in every direction, which the reference's A-A kernel assumes
 * (include/lbm3d/kernels.h:30-37, lbm_block.hpp:256-257).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL double
#endif
#ifndef SFX
#define SFX _f64
#endif
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define API(name) CAT(name, SFX)

typedef REAL real_t;

/* single-precision builds use the float math functions, as the reference's
 * C++ overloads do for dreal = float */
#define IS_FLOAT (sizeof(REAL) == sizeof(float))
#define FABS(v) (IS_FLOAT ? (real_t) fabsf((float) (v)) : (real_t) fabs((double) (v)))
#define SQRT(v) (IS_FLOAT ? (real_t) sqrtf((float) (v)) : (real_t) sqrt((double) (v)))

/* ------------------------------------------------------------------ */
/* direction table: slot order of include/lbm3d/defs.h:318-350         */
/* ------------------------------------------------------------------ */
enum {
	ZZZ, PZZ, MZZ, ZPZ, ZMZ, ZZP, ZZM, PPZ, MMZ, PMZ, MPZ, PZP, MZM, PZM, MZP,
	ZPP, ZMM, ZPM, ZMP, PPP, MMM, PPM, MMP, PMP, MPM, PMM, MPP
};
static const int CX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
static const int CY[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
static const int CZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1};

static inline int opposite(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }

/* slot index of direction with components (cx, cy, cz) */
static int dir_of(int cx, int cy, int cz)
{
	for (int q = 0; q < 27; q++)
		if (CX[q] == cx && CY[q] == cy && CZ[q] == cz)
			return q;
	return -1;
}

/* GEO site types of D3Q27_BC_All (include/lbm3d/d3q27/bc.h:17-43) */
enum {
	GEO_FLUID, GEO_WALL, GEO_INFLOW, GEO_INFLOW_LEFT, GEO_INFLOW_BB_LEFT, GEO_INFLOW_EQ_LEFT, GEO_OUTFLOW_EQ,
	GEO_OUTFLOW_RIGHT, GEO_OUTFLOW_RIGHT_INTERP, GEO_PERIODIC, GEO_NOTHING, GEO_SYM_TOP, GEO_SYM_BOTTOM,
	GEO_SYM_LEFT, GEO_SYM_RIGHT, GEO_SYM_BACK, GEO_SYM_FRONT
};

/* collision operator ids and equilibrium ids used across the oracle API */
enum { COLL_CUM = 0, COLL_SRT = 1, COLL_BGK = 2, COLL_MRT = 3 };
enum { EQ_SECOND_ORDER = 0, EQ_INV_CUM = 1 };
enum { CUM_GEIER2017 = 1, CUM_ANTIALIAS = 2 };

typedef struct {
	real_t f[27];
	real_t fx, fy, fz;
	real_t vx, vy, vz;
	real_t rho, nu;
} site_t;

/* ------------------------------------------------------------------ */
/* equilibria                                                          */
/* ------------------------------------------------------------------ */

/* second-order Maxwell-Boltzmann equilibrium, w_q * rho * feq
 * (include/lbm3d/d3q27/eq.h:13-130) */
static real_t weight_of(int q)
{
	const int n = (CX[q] != 0) + (CY[q] != 0) + (CZ[q] != 0);
	switch (n) {
		case 0: return (real_t) (8.0 / 27.0);
		case 1: return (real_t) (2.0 / 27.0);
		case 2: return (real_t) (1.0 / 54.0);
		default: return (real_t) (1.0 / 216.0);
	}
}

static void eq_second_order(real_t rho, real_t vx, real_t vy, real_t vz, real_t* out)
{
	const real_t three = 3, half3 = (real_t) 1.5, nine_half = (real_t) 4.5, one = 1;
	for (int q = 0; q < 27; q++) {
		const real_t cu = ((real_t) CX[q] * vx + (real_t) CY[q] * vy) + (real_t) CZ[q] * vz;
		const real_t feq = ((one - half3 * ((vx * vx + vy * vy) + vz * vz)) + three * cu) + nine_half * cu * cu;
		out[q] = weight_of(q) * rho * feq;
	}
}

/* factorised equilibrium of the equilibrium cumulants
 * (include/lbm3d/d3q27/eq_inv_cum.h:24-136): a signed weight times a
 * product of one factor per axis */
static real_t axis_factor(int c, real_t v)
{
	const real_t three = 3;
	if (c == 0)
		return three * v * v - (real_t) 2;
	if (c > 0)
		return three * v * v + three * v + (real_t) 1;
	return three * v * v - three * v + (real_t) 1;
}

static real_t inv_cum_coef(int q)
{
	const int n = (CX[q] != 0) + (CY[q] != 0) + (CZ[q] != 0);
	switch (n) {
		case 0: return -(real_t) (1.0 / 27.0);
		case 1: return (real_t) (1.0 / 54.0);
		case 2: return -(real_t) (1.0 / 108.0);
		default: return (real_t) (1.0 / 216.0);
	}
}

static void eq_inv_cum(real_t rho, real_t vx, real_t vy, real_t vz, real_t* out)
{
	for (int q = 0; q < 27; q++) {
		const real_t prod = (axis_factor(CX[q], vx) * axis_factor(CY[q], vy)) * axis_factor(CZ[q], vz);
		out[q] = inv_cum_coef(q) * rho * prod;
	}
}

static void equilibrium(int eq, real_t rho, real_t vx, real_t vy, real_t vz, real_t* out)
{
	if (eq == EQ_INV_CUM)
		eq_inv_cum(rho, vx, vy, vz, out);
	else
		eq_second_order(rho, vx, vy, vz, out);
}

/* ------------------------------------------------------------------ */
/* density and velocity (include/lbm3d/d3q27/common.h:17-50)            */
/* The pairwise grouping follows Geier 2015 Appendix J as the reference */
/* ------------------------------------------------------------------ */
static void density_velocity(site_t* s)
{
	const real_t* f = s->f;
	s->rho = ((((f[PPP] + f[MMM]) + (f[PMP] + f[MPM])) + ((f[PPM] + f[MMP]) + (f[MPP] + f[PMM])))
			  + (((f[ZPP] + f[ZMM]) + (f[ZPM] + f[ZMP])) + ((f[PZP] + f[MZM]) + (f[PZM] + f[MZP]))
				 + ((f[PPZ] + f[MMZ]) + (f[PMZ] + f[MPZ])))
			  + ((f[PZZ] + f[MZZ]) + (f[ZPZ] + f[ZMZ]) + (f[ZZP] + f[ZZM])))
		   + f[ZZZ];
	const real_t half = (real_t) 0.5;
	s->vz = ((((f[PPP] - f[MMM]) + (f[MPP] - f[PMM])) + ((f[PMP] - f[MPM]) + (f[MMP] - f[PPM])))
			 + (((f[ZPP] - f[ZMM]) + (f[ZMP] - f[ZPM])) + ((f[PZP] - f[MZM]) + (f[MZP] - f[PZM])))
			 + (f[ZZP] - f[ZZM]) + s->fz * half)
		  / s->rho;
	s->vx = ((((f[PPP] - f[MMM]) + (f[PMP] - f[MPM])) + ((f[PPM] - f[MMP]) + (f[PMM] - f[MPP])))
			 + (((f[PZP] - f[MZM]) + (f[PZM] - f[MZP])) + ((f[PPZ] - f[MMZ]) + (f[PMZ] - f[MPZ])))
			 + (f[PZZ] - f[MZZ]) + s->fx * half)
		  / s->rho;
	s->vy = ((((f[PPP] - f[MMM]) + (f[PPM] - f[MMP])) + ((f[MPP] - f[PMM]) + (f[MPM] - f[PMP])))
			 + (((f[PPZ] - f[MMZ]) + (f[MPZ] - f[PMZ])) + ((f[ZPP] - f[ZMM]) + (f[ZPM] - f[ZMP])))
			 + (f[ZPZ] - f[ZMZ]) + s->fy * half)
		  / s->rho;
}

/* ------------------------------------------------------------------ */
/* cumulant collision (include/lbm3d/d3q27/col_cum.h:13-511)            */
/* ------------------------------------------------------------------ */

/* 3x3x3 cube M[i][j][k]: axis positions m,z,p = 0,1,2 before a pass,
 * moment orders 0,1,2 after it */
typedef real_t cube_t[3][3][3];

/* forward chimera transform of one line (col_cum.h:62-167, Eqs 6-14 of
 * Geier 2017): (m, z, p) -> (k0, k1, k2) about velocity u */
static inline void chimera_fwd(real_t* m, real_t* z, real_t* p, real_t u, real_t u2)
{
	const real_t two = 2;
	const real_t k0 = (*p + *m) + *z;
	const real_t k1 = (*p - *m) - u * k0;
	const real_t k2 = (*p + *m) - two * u * (*p - *m) + u2 * k0;
	*m = k0;
	*z = k1;
	*p = k2;
}

/* backward chimera transform of one line (col_cum.h:375-472, Eqs 88-96 of
 * Geier 2015): (k0, k1, k2) -> (m, z, p) */
static inline void chimera_bwd(real_t* a, real_t* b, real_t* c, real_t u, real_t u2)
{
	const real_t one = 1, two = 2, half = (real_t) 0.5;
	const real_t k0 = *a, k1 = *b, k2 = *c;
	const real_t vz = k0 * (one - u2) - two * u * k1 - k2;
	const real_t vm = (k0 * (u2 - u) + k1 * (two * u - one) + k2) * half;
	const real_t vp = (k0 * (u2 + u) + k1 * (two * u + one) + k2) * half;
	*a = vm;
	*b = vz;
	*c = vp;
}

static void cube_from_f(const real_t* f, cube_t M)
{
	for (int q = 0; q < 27; q++)
		M[CX[q] + 1][CY[q] + 1][CZ[q] + 1] = f[q];
}

static void f_from_cube(cube_t M, real_t* f)
{
	for (int q = 0; q < 27; q++)
		f[q] = M[CX[q] + 1][CY[q] + 1][CZ[q] + 1];
}

/* relaxation rates that depend on the viscosity only (col_cum.h:195-228) */
typedef struct {
	real_t omega1, omega2, omega3, omega4, omega5, A, B;
} cum_rates_t;

static cum_rates_t cum_rates(real_t nu)
{
	const real_t one = 1, two = 2, three = 3, half = (real_t) 0.5;
	cum_rates_t r;
	const real_t w1 = one / (three * nu + half);
	const real_t w2 = one;
	r.omega1 = w1;
	r.omega2 = w2;
	r.omega3 = (real_t) 8 * (w1 - two) * (w2 * (three * w1 - one) - (real_t) 5 * w1)
			 / ((real_t) 8 * ((real_t) 5 - two * w1) * w1 + w2 * ((real_t) 8 + w1 * ((real_t) 9 * w1 - (real_t) 26)));
	r.omega4 = (real_t) 8 * (w1 - two) * (w1 + w2 * (three * w1 - (real_t) 7))
			 / (w2 * ((real_t) 56 - (real_t) 42 * w1 + (real_t) 9 * w1 * w1) - (real_t) 8 * w1);
	r.omega5 = (real_t) 24 * (w1 - two)
			 * ((real_t) 4 * w1 * w1 + w1 * w2 * ((real_t) 18 - (real_t) 13 * w1)
				+ w2 * w2 * (two + w1 * ((real_t) 6 * w1 - (real_t) 11)))
			 / ((real_t) 16 * w1 * w1 * (w1 - (real_t) 6) - two * w1 * w2 * ((real_t) 216 + (real_t) 5 * w1 * ((real_t) 9 * w1 - (real_t) 46))
				+ w2 * w2 * (w1 * (three * w1 - (real_t) 10) * ((real_t) 15 * w1 - (real_t) 28) - (real_t) 48));
	r.A = ((real_t) 4 * w1 * w1 + two * w1 * w2 * (w1 - (real_t) 6) + w2 * w2 * (w1 * ((real_t) 10 - three * w1) - (real_t) 4))
		/ (w1 - w2) / (w2 * (two + three * w1) - (real_t) 8 * w1);
	r.B = ((real_t) 4 * w1 * w2 * ((real_t) 9 * w1 - (real_t) 16) - (real_t) 4 * w1 * w1
		   - two * w2 * w2 * (two + (real_t) 9 * w1 * (w1 - two)))
		* (real_t) (1.0 / 3.0) / (w1 - w2) / (w2 * (two + three * w1) - (real_t) 8 * w1);
	return r;
}

/* limiter omega + (1 - omega)|C| / (rho*lambda + |C|)  (col_cum.h:203-216) */
static inline real_t limited(real_t omega, real_t c, real_t rho, real_t lambda)
{
	return omega + ((real_t) 1 - omega) * FABS(c) / (rho * lambda + FABS(c));
}

static void collide_cumulant(site_t* s, int flags)
{
	const int v2017 = (flags & CUM_GEIER2017) != 0;
	const int antialias = (flags & CUM_ANTIALIAS) != 0;
	const real_t one = 1, two = 2, three = 3, four = 4, half = (real_t) 0.5;
	const real_t third = (real_t) (1.0 / 3.0);
	const real_t rho = s->rho, vx = s->vx, vy = s->vy, vz = s->vz;
	const real_t ir = one / rho;
	const real_t vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;

	cube_t M;
	cube_from_f(s->f, M);
	/* z pass (Eqs 6-8), y pass (Eqs 9-11), x pass (Eqs 12-14) */
	for (int i = 0; i < 3; i++)
		for (int j = 0; j < 3; j++)
			chimera_fwd(&M[i][j][0], &M[i][j][1], &M[i][j][2], vz, vz2);
	for (int i = 0; i < 3; i++)
		for (int k = 0; k < 3; k++)
			chimera_fwd(&M[i][0][k], &M[i][1][k], &M[i][2][k], vy, vy2);
	for (int j = 0; j < 3; j++)
		for (int k = 0; k < 3; k++)
			chimera_fwd(&M[0][j][k], &M[1][j][k], &M[2][j][k], vx, vx2);

	/* central moments k_abc = M[a][b][c]; cumulants of order <= 3 equal them */
#define K(a, b, c) M[a][b][c]
	const real_t k000 = K(0, 0, 0);
	const real_t C110 = K(1, 1, 0), C101 = K(1, 0, 1), C011 = K(0, 1, 1);
	const real_t C200 = K(2, 0, 0), C020 = K(0, 2, 0), C002 = K(0, 0, 2);
	const real_t C120 = K(1, 2, 0), C102 = K(1, 0, 2), C210 = K(2, 1, 0);
	const real_t C012 = K(0, 1, 2), C201 = K(2, 0, 1), C021 = K(0, 2, 1);
	const real_t C111 = K(1, 1, 1);

	const real_t w1 = one / (three * s->nu + half);
	const real_t w2 = one;

	/* Eqs 27-32 of Geier 2017, part I (col_cum.h:234-250) */
	real_t Dxu = 0, Dyv = 0, Dzw = 0, DxvDyu = 0, DxwDzu = 0, DywDzv = 0;
	if (antialias) {
		Dxu = -w1 * half * ir * (two * C200 - C020 - C002) - w2 * half * ir * (C200 + C020 + C002 - (-one + rho));
		Dyv = Dxu + (real_t) 1.5 * w1 * ir * (C200 - C020);
		Dzw = Dxu + (real_t) 1.5 * w1 * ir * (C200 - C002);
		DxvDyu = -three * w1 * ir * C110;
		DxwDzu = -three * w1 * ir * C101;
		DywDzv = -three * w1 * ir * C011;
	}

	/* second order (col_cum.h:231-259) */
	const real_t Cs110 = (one - w1) * C110;
	const real_t Cs101 = (one - w1) * C101;
	const real_t Cs011 = (one - w1) * C011;
	const real_t e33 = (one - w1) * (C200 - C020) - three * rho * (one - w1 * half) * (vx2 * Dxu - vy2 * Dyv);
	const real_t e34 = (one - w1) * (C200 - C002) - three * rho * (one - w1 * half) * (vx2 * Dxu - vz2 * Dzw);
	const real_t e35 = k000 * w2 + (one - w2) * (C200 + C020 + C002)
					 - three * rho * (one - w2 * half) * (vx2 * Dxu + vy2 * Dyv + vz2 * Dzw);
	const real_t Cs200 = third * (e33 + e34 + e35);
	const real_t Cs020 = third * (-two * e33 + e34 + e35);
	const real_t Cs002 = third * (e33 - two * e34 + e35);

	real_t Cs120 = 0, Cs102 = 0, Cs210 = 0, Cs012 = 0, Cs021 = 0, Cs201 = 0, Cs111 = 0;
	real_t ks211, ks121, ks112, ks220, ks022, ks202, ks122, ks212, ks221, ks222;
	if (v2017) {
		/* fourth-order cumulants (Eqs 51-54 of Geier 2015; col_cum.h:169-191) */
		const real_t k211 = K(2, 1, 1), k121 = K(1, 2, 1), k112 = K(1, 1, 2);
		const real_t k220 = K(2, 2, 0), k022 = K(0, 2, 2), k202 = K(2, 0, 2);
		const real_t k122 = K(1, 2, 2), k212 = K(2, 1, 2), k221 = K(2, 2, 1), k222 = K(2, 2, 2);
		const real_t k110 = C110, k101 = C101, k011 = C011, k200 = C200, k020 = C020, k002 = C002;
		const real_t k120 = C120, k102 = C102, k210 = C210, k012 = C012, k201 = C201, k021 = C021, k111 = C111;
		const real_t C211 = k211 - (k200 * k011 + two * k101 * k110) * ir;
		const real_t C121 = k121 - (k020 * k101 + two * k110 * k011) * ir;
		const real_t C112 = k112 - (k002 * k110 + two * k011 * k101) * ir;
		const real_t C220 = k220 - (k020 * k200 + two * k110 * k110) * ir;
		const real_t C022 = k022 - (k002 * k020 + two * k011 * k011) * ir;
		const real_t C202 = k202 - (k200 * k002 + two * k101 * k101) * ir;
		const real_t C122 = k122 - (k020 * k102 + k002 * k120 + four * k011 * k111 + two * (k110 * k012 + k101 * k021)) * ir;
		const real_t C212 = k212 - (k002 * k210 + k200 * k012 + four * k101 * k111 + two * (k011 * k201 + k110 * k102)) * ir;
		const real_t C221 = k221 - (k200 * k021 + k020 * k201 + four * k110 * k111 + two * (k101 * k120 + k011 * k210)) * ir;
		const real_t C222 = k222
						  - (four * k111 * k111 + k200 * k022 + k020 * k202 + k002 * k220
							 + four * (k011 * k211 + k101 * k121 + k110 * k112) + two * (k120 * k102 + k210 * k012 + k201 * k021))
								* ir
						  + ((real_t) 16 * k110 * k101 * k011 + four * (k101 * k101 * k020 + k011 * k011 * k200 + k110 * k110 * k002)
							 + two * k200 * k020 * k002)
								* ir * ir;

		const cum_rates_t r = cum_rates(s->nu);
		const real_t lam = (real_t) 0.01;
		const real_t w120p102 = limited(r.omega3, C120 + C102, rho, lam);
		const real_t w210p012 = limited(r.omega3, C210 + C012, rho, lam);
		const real_t w201p021 = limited(r.omega3, C201 + C021, rho, lam);
		const real_t w120m102 = limited(r.omega4, C120 - C102, rho, lam);
		const real_t w210m012 = limited(r.omega4, C210 - C012, rho, lam);
		const real_t w201m021 = limited(r.omega4, C201 - C021, rho, lam);
		const real_t w111 = limited(r.omega5, C111, rho, lam);

		/* third order (Eqs 117-122 and 42; col_cum.h:262-277) */
		const real_t e117 = (one - w120p102) * (C120 + C102);
		const real_t e118 = (one - w210p012) * (C210 + C012);
		const real_t e119 = (one - w201p021) * (C201 + C021);
		const real_t e120 = (one - w120m102) * (C120 - C102);
		const real_t e121 = (one - w210m012) * (C210 - C012);
		const real_t e122 = (one - w201m021) * (C201 - C021);
		Cs120 = half * (e120 + e117);
		Cs102 = half * (-e120 + e117);
		Cs210 = half * (e121 + e118);
		Cs012 = half * (-e121 + e118);
		Cs021 = half * (-e122 + e119);
		Cs201 = half * (e122 + e119);
		Cs111 = (one - w111) * C111;

		/* fourth order (Eqs 43-52; col_cum.h:279-297), omega6..10 = 1 */
		const real_t w6 = one, w7 = one, w8 = one, w9 = one, w10 = one;
		const real_t g = (one / w1 - half);
		const real_t e43 = (real_t) (2.0 / 3.0) * g * w6 * r.A * rho * (Dxu - two * Dyv + Dzw) + (one - w6) * (C220 - two * C202 + C022);
		const real_t e44 = (real_t) (2.0 / 3.0) * g * w6 * r.A * rho * (Dxu + Dyv - two * Dzw) + (one - w6) * (C220 + C202 - two * C022);
		const real_t e45 = -(real_t) (4.0 / 3.0) * g * w7 * r.A * rho * (Dxu + Dyv + Dzw) + (one - w7) * (C220 + C202 + C022);
		const real_t Cs220 = third * (e43 + e44 + e45);
		const real_t Cs202 = third * (-e43 + e45);
		const real_t Cs022 = third * (-e44 + e45);
		const real_t Cs211 = -third * g * w8 * r.B * rho * DywDzv + (one - w8) * C211;
		const real_t Cs121 = -third * g * w8 * r.B * rho * DxwDzu + (one - w8) * C121;
		const real_t Cs112 = -third * g * w8 * r.B * rho * DxvDyu + (one - w8) * C112;
		const real_t Cs221 = (one - w9) * C221;
		const real_t Cs212 = (one - w9) * C212;
		const real_t Cs122 = (one - w9) * C122;
		const real_t Cs222 = (one - w10) * C222;

		/* back to central moments (Eqs 81-84 of Geier 2015; col_cum.h:303-328) */
		ks211 = Cs211 + (Cs200 * Cs011 + two * Cs101 * Cs110) * ir;
		ks121 = Cs121 + (Cs020 * Cs101 + two * Cs110 * Cs011) * ir;
		ks112 = Cs112 + (Cs002 * Cs110 + two * Cs011 * Cs101) * ir;
		ks220 = Cs220 + (Cs020 * Cs200 + two * Cs110 * Cs110) * ir;
		ks022 = Cs022 + (Cs002 * Cs020 + two * Cs011 * Cs011) * ir;
		ks202 = Cs202 + (Cs200 * Cs002 + two * Cs101 * Cs101) * ir;
		ks122 = Cs122 + (Cs020 * Cs102 + Cs002 * Cs120 + four * Cs011 * Cs111 + two * (Cs110 * Cs012 + Cs101 * Cs021)) * ir;
		ks212 = Cs212 + (Cs002 * Cs210 + Cs200 * Cs012 + four * Cs101 * Cs111 + two * (Cs011 * Cs201 + Cs110 * Cs102)) * ir;
		ks221 = Cs221 + (Cs200 * Cs021 + Cs020 * Cs201 + four * Cs110 * Cs111 + two * (Cs101 * Cs120 + Cs011 * Cs210)) * ir;
		ks222 = Cs222
			  + (four * Cs111 * Cs111 + Cs200 * ks022 + Cs020 * ks202 + Cs002 * ks220
				 + four * (Cs011 * ks211 + Cs101 * ks121 + Cs110 * ks112) + two * (Cs120 * Cs102 + Cs210 * Cs012 + Cs201 * Cs021))
					* ir
			  - ((real_t) 16 * Cs110 * Cs101 * Cs011 + four * (Cs101 * Cs101 * Cs020 + Cs011 * Cs011 * Cs200 + Cs110 * Cs110 * Cs002)
				 + two * Cs200 * Cs020 * Cs002)
					* ir * ir;
	}
	else {
		/* default variant: third- and higher-order cumulants relax to zero
		 * (col_cum.h:330-366) */
		ks211 = (Cs200 * Cs011 + two * Cs101 * Cs110) * ir;
		ks121 = (Cs020 * Cs101 + two * Cs110 * Cs011) * ir;
		ks112 = (Cs002 * Cs110 + two * Cs011 * Cs101) * ir;
		ks220 = (Cs020 * Cs200 + two * Cs110 * Cs110) * ir;
		ks022 = (Cs002 * Cs020 + two * Cs011 * Cs011) * ir;
		ks202 = (Cs200 * Cs002 + two * Cs101 * Cs101) * ir;
		ks122 = 0;
		ks212 = 0;
		ks221 = 0;
		ks222 = (Cs200 * ks022 + Cs020 * ks202 + Cs002 * ks220 + four * (Cs011 * ks211 + Cs101 * ks121 + Cs110 * ks112)) * ir
			  - ((real_t) 16 * Cs110 * Cs101 * Cs011 + four * (Cs101 * Cs101 * Cs020 + Cs011 * Cs011 * Cs200 + Cs110 * Cs110 * Cs002)
				 + two * Cs200 * Cs020 * Cs002)
					* ir * ir;
	}

	/* post-collision central moments; first moments flipped by the forcing
	 * scheme of Geier 2017 (col_cum.h:369-373) */
	K(0, 0, 0) = k000;
	K(1, 0, 0) = -K(1, 0, 0);
	K(0, 1, 0) = -K(0, 1, 0);
	K(0, 0, 1) = -K(0, 0, 1);
	K(1, 1, 0) = Cs110;
	K(1, 0, 1) = Cs101;
	K(0, 1, 1) = Cs011;
	K(2, 0, 0) = Cs200;
	K(0, 2, 0) = Cs020;
	K(0, 0, 2) = Cs002;
	K(1, 2, 0) = Cs120;
	K(1, 0, 2) = Cs102;
	K(2, 1, 0) = Cs210;
	K(0, 1, 2) = Cs012;
	K(2, 0, 1) = Cs201;
	K(0, 2, 1) = Cs021;
	K(1, 1, 1) = Cs111;
	K(2, 1, 1) = ks211;
	K(1, 2, 1) = ks121;
	K(1, 1, 2) = ks112;
	K(2, 2, 0) = ks220;
	K(0, 2, 2) = ks022;
	K(2, 0, 2) = ks202;
	K(1, 2, 2) = ks122;
	K(2, 1, 2) = ks212;
	K(2, 2, 1) = ks221;
	K(2, 2, 2) = ks222;
#undef K

	/* backward: x pass (Eqs 88-90), y pass (91-93), z pass (94-96) */
	for (int j = 0; j < 3; j++)
		for (int k = 0; k < 3; k++)
			chimera_bwd(&M[0][j][k], &M[1][j][k], &M[2][j][k], vx, vx2);
	for (int i = 0; i < 3; i++)
		for (int k = 0; k < 3; k++)
			chimera_bwd(&M[i][0][k], &M[i][1][k], &M[i][2][k], vy, vy2);
	for (int i = 0; i < 3; i++)
		for (int j = 0; j < 3; j++)
			chimera_bwd(&M[i][j][0], &M[i][j][1], &M[i][j][2], vz, vz2);
	f_from_cube(M, s->f);
}

/* ------------------------------------------------------------------ */
/* SRT / BGK / MRT through the same slot                               */
/* ------------------------------------------------------------------ */

/* forcing term S_q = 3 (c_q - u).F / rho, written per axis as (-u + c) F */
static inline real_t force_term(int q, const site_t* s, real_t irho)
{
	const real_t tx = (-s->vx + (real_t) CX[q]) * s->fx;
	const real_t ty = (-s->vy + (real_t) CY[q]) * s->fy;
	const real_t tz = (-s->vz + (real_t) CZ[q]) * s->fz;
	return ((real_t) 3 * ((tx + ty) + tz)) * irho;
}

/* textbook BGK with Guo-like forcing (include/lbm3d/d3q27/col_srt.h:14-105) */
static void collide_srt(site_t* s, int eq)
{
	const real_t tau = (real_t) 3 * s->nu + (real_t) 0.5;
	const real_t irho = (real_t) 1 / (s->rho == 0 ? (real_t) 1 : s->rho);
	real_t feq[27];
	equilibrium(eq, s->rho, s->vx, s->vy, s->vz, feq);
	for (int q = 0; q < 27; q++) {
		const real_t S = force_term(q, s, irho);
		s->f[q] += (feq[q] - s->f[q]) / tau + ((real_t) 1 - (real_t) 0.5 / tau) * S * feq[q];
	}
}

/* Geier's improved BGK with factorised equilibrium, no Galilean correction
 * (include/lbm3d/d3q27/col_bgk.h:18-144) */
static void collide_bgk(site_t* s)
{
	const real_t one = 1, half = (real_t) 0.5, third = (real_t) (1.0 / 3.0);
	const real_t w1 = one / ((real_t) 3 * s->nu + half);
	const real_t Xz = third - one + s->vx * s->vx, Xp = -half * (Xz + one + s->vx), Xm = Xp + s->vx;
	const real_t Yz = third - one + s->vy * s->vy, Yp = -half * (Yz + one + s->vy), Ym = Yp + s->vy;
	const real_t Zz = third - one + s->vz * s->vz, Zp = -half * (Zz + one + s->vz), Zm = Zp + s->vz;
	for (int q = 0; q < 27; q++) {
		const real_t X = CX[q] == 0 ? Xz : (CX[q] > 0 ? Xp : Xm);
		const real_t Y = CY[q] == 0 ? Yz : (CY[q] > 0 ? Yp : Ym);
		const real_t Z = CZ[q] == 0 ? Zz : (CZ[q] > 0 ? Zp : Zm);
		const real_t tx = (-s->vx + (real_t) CX[q]) * s->fx;
		const real_t ty = (-s->vy + (real_t) CY[q]) * s->fy;
		const real_t tz = (-s->vz + (real_t) CZ[q]) * s->fz;
		const real_t S = ((real_t) 3 * ((tx + ty) + tz)) / s->rho;
		const real_t feq = -s->rho * X * Y * Z;
		s->f[q] += (feq - s->f[q]) * w1 + (one - half * w1) * S * feq;
	}
}

/* MRT-LES: relax only the second-moment tensor with a Smagorinsky rate and
 * rebuild the populations (include/lbm3d/d3q27/col_mrt.h:14-141) */
static void collide_mrt(site_t* s)
{
	const real_t* f = s->f;
	real_t Pxx = 0, Pyy = 0, Pzz = 0, Pxy = 0, Pxz = 0, Pyz = 0;
	/* summation order of the reference: directions with the component in the
	 * enumeration order mmm, mmz, mmp, mzm, ..., ppp */
	static const int order[27] = {MMM, MMZ, MMP, MZM, MZZ, MZP, MPM, MPZ, MPP, ZMM, ZMZ, ZMP, ZZM, ZZZ,
								  ZZP, ZPM, ZPZ, ZPP, PMM, PMZ, PMP, PZM, PZZ, PZP, PPM, PPZ, PPP};
	int first_xx = 1, first_yy = 1, first_zz = 1, first_xy = 1, first_xz = 1, first_yz = 1;
	for (int n = 0; n < 27; n++) {
		const int q = order[n];
		if (CX[q] != 0) {
			Pxx = first_xx ? f[q] : Pxx + f[q];
			first_xx = 0;
		}
		if (CY[q] != 0) {
			Pyy = first_yy ? f[q] : Pyy + f[q];
			first_yy = 0;
		}
		if (CZ[q] != 0) {
			Pzz = first_zz ? f[q] : Pzz + f[q];
			first_zz = 0;
		}
		if (CX[q] * CY[q] != 0) {
			const real_t t = CX[q] * CY[q] > 0 ? f[q] : -f[q];
			Pxy = first_xy ? t : (CX[q] * CY[q] > 0 ? Pxy + f[q] : Pxy - f[q]);
			first_xy = 0;
		}
		if (CX[q] * CZ[q] != 0) {
			const real_t t = CX[q] * CZ[q] > 0 ? f[q] : -f[q];
			Pxz = first_xz ? t : (CX[q] * CZ[q] > 0 ? Pxz + f[q] : Pxz - f[q]);
			first_xz = 0;
		}
		if (CY[q] * CZ[q] != 0) {
			const real_t t = CY[q] * CZ[q] > 0 ? f[q] : -f[q];
			Pyz = first_yz ? t : (CY[q] * CZ[q] > 0 ? Pyz + f[q] : Pyz - f[q]);
			first_yz = 0;
		}
	}
	const real_t rho = s->rho, vx = s->vx, vy = s->vy, vz = s->vz;
	const real_t third = (real_t) (1.0 / 3.0), two = 2, three = 3;
	const real_t Pnxx = Pxx - rho * (third + vx * vx);
	const real_t Pnyy = Pyy - rho * (third + vy * vy);
	const real_t Pnzz = Pzz - rho * (third + vz * vz);
	const real_t Pnxz = Pxz - rho * vx * vz;
	const real_t Pnxy = Pxy - rho * vx * vy;
	const real_t Pnyz = Pyz - rho * vy * vz;
	const real_t Q = two * (Pnxx * Pnxx + Pnyy * Pnyy + Pnzz * Pnzz + two * (Pnxy * Pnxy + Pnxz * Pnxz + Pnyz * Pnyz));
	const real_t tau = three * s->nu + (real_t) 0.5;
	const real_t C = (real_t) 0.0342;
	const real_t omega = two / (SQRT(tau * tau + two * C * three * three * SQRT(Q) / rho) + tau);
	Pxx -= omega * Pnxx;
	Pyy -= omega * Pnyy;
	Pzz -= omega * Pnzz;
	Pxy -= omega * Pnxy;
	Pxz -= omega * Pnxz;
	Pyz -= omega * Pnyz;
	const real_t P2 = (Pxx + Pyy) + Pzz;
	for (int q = 0; q < 27; q++) {
		const int n = (CX[q] != 0) + (CY[q] != 0) + (CZ[q] != 0);
		const real_t cu = ((vx * (real_t) CX[q] + vy * (real_t) CY[q]) + vz * (real_t) CZ[q]);
		const real_t cc = ((Pxx * (real_t) (CX[q] * CX[q]) + Pyy * (real_t) (CY[q] * CY[q])) + Pzz * (real_t) (CZ[q] * CZ[q]))
						+ two * ((Pxy * (real_t) (CX[q] * CY[q]) + Pxz * (real_t) (CX[q] * CZ[q])) + Pyz * (real_t) (CY[q] * CZ[q]));
		s->f[q] = weight_of(q) * (rho * (((real_t) 2.5 - (real_t) 1.5 * (real_t) n) + three * cu) + (real_t) 4.5 * cc - (real_t) 1.5 * P2);
	}
}

static void collide(site_t* s, int coll, int eq, int cum_flags)
{
	switch (coll) {
		case COLL_CUM: collide_cumulant(s, cum_flags); break;
		case COLL_SRT: collide_srt(s, eq); break;
		case COLL_BGK: collide_bgk(s); break;
		default: collide_mrt(s); break;
	}
}

/* ------------------------------------------------------------------ */
/* lattice, A-A streaming and boundary conditions                      */
/* ------------------------------------------------------------------ */
typedef struct {
	long X, Y, Z;
	long sy, sz, sq; /* strides of the canonical ghost-layer storage */
	real_t* f;
	const int16_t* map;
	real_t nu, fx, fy, fz;
	const double *in_vx, *in_vy, *in_vz;
	real_t* macro;
	int coll, eq, cum_flags;
	int even;
} lattice_t;

static inline long slot(const lattice_t* L, int q, long x, long y, long z)
{
	return q * L->sq + (z + 1) * L->sz + (y + 1) * L->sy + (x + 1);
}

static void inflow_velocity(const lattice_t* L, site_t* s, long y, long z)
{
	const long i = L->Y * z + y; /* NSE_Data_InflowProfile (lbm_data.h:105-132) */
	s->vx = L->in_vx ? (real_t) L->in_vx[i] : 0;
	s->vy = L->in_vy ? (real_t) L->in_vy[i] : 0;
	s->vz = L->in_vz ? (real_t) L->in_vz[i] : 0;
}

/* A-A read (include/lbm3d/d3q27/streaming_AA.h:79-116): even step reads the
 * site's own slots; odd step reads, for direction q, the opposite slot of the
 * upwind neighbour x - c_q */
static void aa_read(const lattice_t* L, site_t* s, const long* nx, const long* ny, const long* nz)
{
	for (int q = 0; q < 27; q++) {
		if (L->even)
			s->f[q] = L->f[slot(L, q, nx[1], ny[1], nz[1])];
		else
			s->f[q] = L->f[slot(L, opposite(q), nx[1 - CX[q]], ny[1 - CY[q]], nz[1 - CZ[q]])];
	}
}

/* A-A write (streaming_AA.h:12-76): even step stores direction q into the
 * opposite slot of the site; odd step pushes it into slot q of x + c_q */
static void aa_write(const lattice_t* L, const site_t* s, const long* nx, const long* ny, const long* nz)
{
	for (int q = 0; q < 27; q++) {
		if (L->even)
			L->f[slot(L, opposite(q), nx[1], ny[1], nz[1])] = s->f[q];
		else
			L->f[slot(L, q, nx[1 + CX[q]], ny[1 + CY[q]], nz[1 + CZ[q]])] = s->f[q];
	}
}

static void set_equilibrium(const lattice_t* L, site_t* s)
{
	equilibrium(L->eq, s->rho, s->vx, s->vy, s->vz, s->f);
}

/* density of a left inlet from the known populations
 * (include/lbm3d/d3q27/bc.h:97-110 and 169-182) */
static real_t inlet_density(const site_t* s)
{
	const real_t* f = s->f;
	return (real_t) 1.0 / (1 - s->vx)
		 * ((f[ZZZ] + (+((f[ZPP] + f[ZMM]) + (f[ZPM] + f[ZMP])) + ((f[ZPZ] + f[ZMZ]) + (f[ZZP] + f[ZZM]))))
			+ 2 * (f[MZZ] + (+((f[MPP] + f[MMM]) + (f[MPM] + f[MMP])) + ((f[MPZ] + f[MMZ]) + (f[MZP] + f[MZM])))));
}

/* moment-based inlet of Eichler (bc.h:91-142) */
static void inlet_moments(site_t* s)
{
	real_t* f = s->f;
	s->rho = inlet_density(s);
	const real_t rho = s->rho, vx = s->vx, vy = s->vy, vz = s->vz;
	const real_t third = (real_t) (1.0 / 3.0), ninth = (real_t) (1.0 / 9.0);
	const real_t m100 = rho * vx, m010 = rho * vy, m001 = rho * vz;
	const real_t m011 = rho * (vy * vz);
	const real_t m020 = third * rho + rho * (vy * vy);
	const real_t m002 = third * rho + rho * (vz * vz);
	const real_t m021 = third * rho * vz + rho * ((vy * vy) * vz);
	const real_t m012 = third * rho * vy + rho * (vy * (vz * vz));
	const real_t m022 = ninth * rho + third * rho * (vy * vy + vz * vz) + rho * (vy * vy) * (vz * vz);
	f[PZZ] = m100 + (m022 - (m020 + m002)) + f[MZZ] + (+((f[ZPP] + f[ZMM]) + (f[ZPM] + f[ZMP])) + ((f[ZZP] + f[ZZM]) + (f[ZPZ] + f[ZMZ])))
		   + 2 * (+((f[MPP] + f[MMM]) + (f[MPM] + f[MMP])) + ((f[MPZ] + f[MMZ]) + (f[MZP] + f[MZM])));
	const real_t h = (real_t) 0.5, qt = (real_t) 0.25;
	f[PPZ] = h * ((m020 - m022) + (-m012 + m010)) - (f[MPZ] + f[ZPZ]);
	f[PMZ] = h * ((m020 - m022) + (m012 - m010)) - (f[MMZ] + f[ZMZ]);
	f[PZP] = h * ((m002 - m022) + (-m021 + m001)) - (f[MZP] + f[ZZP]);
	f[PZM] = h * ((m002 - m022) + (m021 - m001)) - (f[MZM] + f[ZZM]);
	f[PPP] = qt * ((m022 + m011) + (m021 + m012)) - (f[MPP] + f[ZPP]);
	f[PPM] = qt * ((m022 - m011) + (-m021 + m012)) - (f[MPM] + f[ZPM]);
	f[PMP] = qt * ((m022 - m011) + (m021 - m012)) - (f[MMP] + f[ZMP]);
	f[PMM] = qt * ((m022 + m011) + (-m021 - m012)) - (f[MMM] + f[ZMM]);
}

/* symmetry planes copy the mirrored populations across one axis
 * (bc.h:222-293): axis 0/1/2 = x/y/z, side = direction that is overwritten */
static void symmetry(site_t* s, int axis, int side)
{
	for (int q = 0; q < 27; q++) {
		const int c[3] = {CX[q], CY[q], CZ[q]};
		if (c[axis] != side)
			continue;
		int m[3] = {c[0], c[1], c[2]};
		m[axis] = -side;
		s->f[q] = s->f[dir_of(m[0], m[1], m[2])];
	}
}

static int does_collide(int geo)
{
	/* bc.h:406-412 */
	return geo == GEO_FLUID || geo == GEO_PERIODIC || geo == GEO_OUTFLOW_RIGHT || geo == GEO_OUTFLOW_RIGHT_INTERP
		|| geo == GEO_INFLOW_LEFT || geo == GEO_INFLOW_BB_LEFT;
}

/* one lattice-site update: kernels.h:92-111 with D3Q27_BC_All (bc.h:60-422) */
static void site_update(const lattice_t* L, long x, long y, long z)
{
	const int geo = L->map[(z * L->Y + y) * L->X + x];
	long nx[3], ny[3], nz[3];
	/* neighbour indices (kernels.h:21-37): wrap on periodic sites, otherwise
	 * plain +-1 into the ghost layer */
	if (geo == GEO_PERIODIC) {
		nx[0] = x == 0 ? L->X - 1 : x - 1;
		nx[2] = x == L->X - 1 ? 0 : x + 1;
		ny[0] = y == 0 ? L->Y - 1 : y - 1;
		ny[2] = y == L->Y - 1 ? 0 : y + 1;
		nz[0] = z == 0 ? L->Z - 1 : z - 1;
		nz[2] = z == L->Z - 1 ? 0 : z + 1;
	}
	else {
		nx[0] = x - 1;
		nx[2] = x + 1;
		ny[0] = y - 1;
		ny[2] = y + 1;
		nz[0] = z - 1;
		nz[2] = z + 1;
	}
	nx[1] = x;
	ny[1] = y;
	nz[1] = z;

	site_t s;
	s.fx = L->fx;
	s.fy = L->fy;
	s.fz = L->fz;
	s.nu = L->nu;
	s.vx = s.vy = s.vz = 0;
	s.rho = 1;

	if (geo == GEO_NOTHING) {
		/* bc.h:63-70: no streaming, no collision, no store */
		s.rho = 1;
		s.vx = s.vy = s.vz = 0;
	}
	else {
		long rx[3] = {nx[0], nx[1], nx[2]};
		if (geo == GEO_OUTFLOW_RIGHT) {
			/* pull location shifted one site upstream (bc.h:73-74) */
			rx[1] = rx[2] = rx[0];
		}
		aa_read(L, &s, rx, ny, nz);
		switch (geo) {
			case GEO_INFLOW:
				inflow_velocity(L, &s, y, z);
				s.rho = 1;
				set_equilibrium(L, &s);
				break;
			case GEO_INFLOW_LEFT:
				inflow_velocity(L, &s, y, z);
				inlet_moments(&s);
				break;
			case GEO_INFLOW_BB_LEFT: {
				/* bc.h:143-165: incoming populations from the site's own slots */
				inflow_velocity(L, &s, y, z);
				const real_t two = 2, three = 3;
				const real_t w2 = (real_t) (2.0 / 27.0), w1 = (real_t) (1.0 / 54.0), w3 = (real_t) (1.0 / 216.0);
				const real_t r = s.rho;
#define OWN(q) L->f[slot(L, (q), x, y, z)]
				s.f[PZZ] = OWN(MZZ) - two * w2 * r * three * (-s.vx);
				s.f[PPZ] = OWN(MMZ) - two * w1 * r * three * (-s.vx - s.vy);
				s.f[PMZ] = OWN(MPZ) - two * w1 * r * three * (-s.vx + s.vy);
				s.f[PZP] = OWN(MZM) - two * w1 * r * three * (-s.vx - s.vz);
				s.f[PZM] = OWN(MZP) - two * w1 * r * three * (-s.vx + s.vz);
				s.f[PPP] = OWN(MMM) - two * w3 * r * three * (-s.vx - s.vy - s.vz);
				s.f[PPM] = OWN(MMP) - two * w3 * r * three * (-s.vx - s.vy + s.vz);
				s.f[PMP] = OWN(MPM) - two * w3 * r * three * (-s.vx + s.vy - s.vz);
				s.f[PMM] = OWN(MPP) - two * w3 * r * three * (-s.vx + s.vy + s.vz);
#undef OWN
				density_velocity(&s);
				break;
			}
			case GEO_INFLOW_EQ_LEFT:
				inflow_velocity(L, &s, y, z);
				s.rho = inlet_density(&s);
				set_equilibrium(L, &s);
				break;
			case GEO_OUTFLOW_EQ:
				density_velocity(&s);
				s.rho = 1;
				set_equilibrium(L, &s);
				break;
			case GEO_OUTFLOW_RIGHT:
				density_velocity(&s);
				s.rho = 1;
				break;
			case GEO_WALL:
				/* full-way bounce-back: swap each direction with its opposite
				 * (bc.h:201-221) */
				s.rho = 1;
				s.vx = s.vy = s.vz = 0;
				for (int q = 1; q < 27; q += 2) {
					const real_t t = s.f[q];
					s.f[q] = s.f[q + 1];
					s.f[q + 1] = t;
				}
				break;
			case GEO_SYM_TOP: symmetry(&s, 2, -1); density_velocity(&s); break;
			case GEO_SYM_BOTTOM: symmetry(&s, 2, 1); density_velocity(&s); break;
			case GEO_SYM_LEFT: symmetry(&s, 0, 1); density_velocity(&s); break;
			case GEO_SYM_RIGHT: symmetry(&s, 0, -1); density_velocity(&s); break;
			case GEO_SYM_BACK: symmetry(&s, 1, 1); density_velocity(&s); break;
			case GEO_SYM_FRONT: symmetry(&s, 1, -1); density_velocity(&s); break;
			default: density_velocity(&s); break;
		}
		if (does_collide(geo))
			collide(&s, L->coll, L->eq, L->cum_flags);
		aa_write(L, &s, nx, ny, nz);
	}
	if (L->macro) {
		/* D3Q27_MACRO_Default::outputMacro (macro.h:70-76) */
		const long n = L->X * L->Y * L->Z, i = (z * L->Y + y) * L->X + x;
		L->macro[i] = s.rho;
		L->macro[n + i] = s.vx;
		L->macro[2 * n + i] = s.vy;
		L->macro[3 * n + i] = s.vz;
	}
}

/* ------------------------------------------------------------------ */
/* exported API (same argument meaning as oracle/ref_harness.cpp)       */
/* ------------------------------------------------------------------ */

int API(orc_aa_run)(int coll, int eq, int cum_flags, long X, long Y, long Z, real_t* f, const int16_t* map, double nu,
					double fx, double fy, double fz, const double* in_vx, const double* in_vy, const double* in_vz,
					real_t* macro, long start_iter, int nsteps, int nthreads)
{
	const long n = X * Y * Z;
	int ordered = 0;
	for (long i = 0; i < n; i++) {
		if (map[i] < 0 || map[i] == GEO_OUTFLOW_RIGHT_INTERP || map[i] > GEO_SYM_FRONT)
			return -2;
		if (map[i] == GEO_INFLOW_BB_LEFT || map[i] == GEO_OUTFLOW_RIGHT)
			ordered = 1;
	}
	lattice_t L;
	L.X = X;
	L.Y = Y;
	L.Z = Z;
	L.sy = X + 2;
	L.sz = (X + 2) * (Y + 2);
	L.sq = (X + 2) * (Y + 2) * (Z + 2);
	L.f = f;
	L.map = map;
	L.nu = (real_t) nu;
	L.fx = (real_t) fx;
	L.fy = (real_t) fy;
	L.fz = (real_t) fz;
	L.in_vx = in_vx;
	L.in_vy = in_vy;
	L.in_vz = in_vz;
	L.macro = macro;
	L.coll = coll;
	L.eq = eq;
	L.cum_flags = cum_flags;
#ifdef _OPENMP
	const int threads = nthreads > 0 ? nthreads : omp_get_max_threads();
#else
	(void) nthreads;
#endif
	for (int step = 0; step < nsteps; step++) {
		L.even = ((start_iter + step) % 2) == 0;
		if (ordered) {
			/* order-dependent site types: the reference's loop order
			 * (state.hpp:1388-1397), single thread */
			for (long x = 0; x < X; x++)
				for (long z = 0; z < Z; z++)
					for (long y = 0; y < Y; y++)
						site_update(&L, x, y, z);
		}
		else {
#pragma omp parallel for schedule(static) collapse(2) num_threads(threads)
			for (long z = 0; z < Z; z++)
				for (long y = 0; y < Y; y++)
					for (long x = 0; x < X; x++)
						site_update(&L, x, y, z);
		}
	}
	return 0;
}

/* equilibrium everywhere incl. ghosts (lbm_block.hpp:248-278); interior from
 * fields when given (sim_4.cu:145-163 passes per-site rho, u) */
int API(orc_init_equilibrium)(int eq, long X, long Y, long Z, real_t* f, const double* rho, const double* vx, const double* vy,
							  const double* vz, double rho0, double vx0, double vy0, double vz0)
{
	const long sq = (X + 2) * (Y + 2) * (Z + 2);
	real_t site[27];
	for (long z = -1; z <= Z; z++)
		for (long y = -1; y <= Y; y++)
			for (long x = -1; x <= X; x++) {
				const int interior = x >= 0 && x < X && y >= 0 && y < Y && z >= 0 && z < Z;
				const long i = (z * Y + y) * X + x;
				if (interior && rho)
					equilibrium(eq, (real_t) rho[i], (real_t) vx[i], (real_t) vy[i], (real_t) vz[i], site);
				else
					equilibrium(eq, (real_t) rho0, (real_t) vx0, (real_t) vy0, (real_t) vz0, site);
				const long s = ((z + 1) * (Y + 2) + (y + 1)) * (X + 2) + (x + 1);
				for (int q = 0; q < 27; q++)
					f[q * sq + s] = site[q];
			}
	return 0;
}

int API(orc_collide)(int coll, int eq, int cum_flags, long n, real_t* f, real_t* macro_out, double nu, double fx, double fy,
					 double fz)
{
	for (long i = 0; i < n; i++) {
		site_t s;
		memcpy(s.f, f + 27 * i, sizeof(s.f));
		s.nu = (real_t) nu;
		s.fx = (real_t) fx;
		s.fy = (real_t) fy;
		s.fz = (real_t) fz;
		density_velocity(&s);
		if (macro_out) {
			macro_out[4 * i] = s.rho;
			macro_out[4 * i + 1] = s.vx;
			macro_out[4 * i + 2] = s.vy;
			macro_out[4 * i + 3] = s.vz;
		}
		collide(&s, coll, eq, cum_flags);
		memcpy(f + 27 * i, s.f, sizeof(s.f));
	}
	return 0;
}

int API(orc_equilibrium)(int eq, long n, const double* rho, const double* vx, const double* vy, const double* vz, real_t* out)
{
	for (long i = 0; i < n; i++)
		equilibrium(eq, (real_t) rho[i], (real_t) vx[i], (real_t) vy[i], (real_t) vz[i], out + 27 * i);
	return 0;
}
