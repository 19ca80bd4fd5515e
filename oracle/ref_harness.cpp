// Reference harness: TNL-LBM's own per-site operator headers, compiled
// unmodified from the reference tree (include/lbm3d/d3q27/*.h) against the
// small shim in oracle/shim, driven by the per-site loop of the reference's
// kernel (include/lbm3d/kernels.h:5-112) and its host OpenMP loop
// (include/lbm3d/state.hpp:1388-1397).
//
// TEST INFRASTRUCTURE ONLY.  The resulting oracle/_ref/*.so is used by the
// test-suite as a checker, by tests/golden/make_golden.py to produce fixtures,
// and by bench.py's CPU-baseline leg.  The product library never links it.
//
// Streaming pattern: A-A (streaming_AA.h) by default; compiled with
// -DAB_PATTERN the same file runs the reference's A-B pull scheme
// (streaming_AB.h) with its two buffers swapped after every step
// (lbm.hpp:314-322) and the clamped neighbour indices of a single block
// (kernels.h:48-55), and exports ref_ab_run instead of ref_aa_run.  The two
// headers define the same template name, so each pattern is its own library.
// The reference's A-A kernel assumes
// one ghost layer of lattice sites in every direction (kernels.h:30-37) that
// is initialised together with the interior (lbm_block.hpp:248-278), so the
// harness allocates that layer.  Storage order is the reference's own
// (q, x, z, y) with y fastest (defs.h:90-91, lbm_data.h:50-54); the exported
// functions exchange populations in the canonical order
// [27][Z+2][Y+2][X+2] (x fastest, ghost layer included) and transpose at the
// boundary of each call.
//
// Variant selection: the cumulant flags USE_GEIER_CUM_2017 and
// USE_GEIER_CUM_ANTIALIAS are preprocessor switches in the reference
// (defs.h:312-315), so this file is compiled once per flag set (see Makefile).

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#ifdef _OPENMP
	#include <omp.h>
#endif

#include "lbm3d/defs.h"	 // resolves to oracle/shim/lbm3d/defs.h

#include "lbm3d/d3q27/bc.h"
#include "lbm3d/d3q27/col_bgk.h"
#include "lbm3d/d3q27/col_cum.h"
#include "lbm3d/d3q27/col_mrt.h"
#include "lbm3d/d3q27/col_srt.h"
#include "lbm3d/d3q27/col_srt_adjoint.h"
#include "lbm3d/d3q27/eq.h"
#include "lbm3d/d3q27/eq_inv_cum.h"
#include "lbm3d/d3q27/macro.h"
#ifdef AB_PATTERN
	#include "lbm3d/d3q27/streaming_AB.h"
#else
	#include "lbm3d/d3q27/streaming_AA.h"
	// the D3Q7 advection-diffusion operators (coupled to the flow in the A-A build)
	#include "lbm3d/d3q7/bc.h"
	#include "lbm3d/d3q7/col_clbm.h"
	#include "lbm3d/d3q7/col_mrt.h"
	#include "lbm3d/d3q7/col_srt.h"
	#include "lbm3d/d3q7/eq.h"
	#include "lbm3d/d3q7/macro.h"
	#include "lbm3d/d3q7/streaming_AA.h"
#endif

namespace {

template <typename DREAL>
struct HarnessTraits
{
	using real = double;
	using dreal = DREAL;
	using idx = long int;
	using map_t = short int;
};

int g_unsupported_hit = 0;

#ifndef AB_PATTERN
// The reference's A-A streaming lacks the two members that D3Q27_BC_All calls
// for adjoint and interpolated-outflow sites (bc.h:79, bc.h:196).  The harness
// rejects maps containing those site types before stepping, so these bodies
// are unreachable; they only let bc.h instantiate.
template <typename TRAITS>
struct HarnessStreamingAA : D3Q27_STREAMING<TRAITS>
{
	using idx = typename TRAITS::idx;

	template <typename D, typename K>
	static void streamingAdjoint(D&, K&, idx, idx, idx, idx, idx, idx, idx, idx, idx)
	{
		g_unsupported_hit = 1;
	}

	template <typename D, typename K>
	static void streamingInterpRight(D&, K&, idx, idx, idx, idx, idx, idx, idx, idx, idx)
	{
		g_unsupported_hit = 1;
	}
};
template <typename TRAITS>
using HarnessStreaming = HarnessStreamingAA<TRAITS>;
#else
template <typename TRAITS>
using HarnessStreaming = D3Q27_STREAMING<TRAITS>;
#endif

// Kernel data: the members D3Q27_BC_All, D3Q27_STREAMING and
// D3Q27_MACRO_Default touch (lbm_data.h:8-61 LBM_Data, :65-73 NSE_Data,
// :95-133 NSE_Data_InflowProfile), with the ghost-layer indexer.
template <typename TRAITS>
struct HarnessData
{
	using idx = typename TRAITS::idx;
	using dreal = typename TRAITS::dreal;
	using map_t = typename TRAITS::map_t;

	bool even_iter = true;
	idx nx = 0, ny = 0, nz = 0;	 // interior sizes
	idx XYZ = 0;				 // per-direction stride incl. ghosts
	dreal lbmViscosity = 0;
	dreal fx = 0, fy = 0, fz = 0;
	dreal* dfs[DFMAX] = {nullptr};
	dreal* dmacro = nullptr;
	const map_t* dmap = nullptr;
	const dreal* inflow_vx = nullptr;
	const dreal* inflow_vy = nullptr;
	const dreal* inflow_vz = nullptr;

	idx X() const { return nx; }
	idx Y() const { return ny; }
	idx Z() const { return nz; }

	// reference storage order (q, x, z, y), y fastest; coordinates may be -1..N
	idx storage(idx x, idx y, idx z) const
	{
		return ((x + 1) * (nz + 2) + (z + 1)) * (ny + 2) + (y + 1);
	}

	map_t map(idx x, idx y, idx z) const
	{
		return dmap[(z * ny + y) * nx + x];
	}

	dreal& df(uint8_t type, int q, idx x, idx y, idx z)
	{
		return dfs[type][q * XYZ + storage(x, y, z)];
	}

	dreal& macro(int id, idx x, idx y, idx z)
	{
		return dmacro[((id * nz + z) * ny + y) * nx + x];
	}

	template <typename LBM_KS>
	void inflow(LBM_KS& KS, idx x, idx y, idx z)
	{
		(void) x;
		KS.vx = inflow_vx ? inflow_vx[ny * z + y] : 0;
		KS.vy = inflow_vy ? inflow_vy[ny * z + y] : 0;
		KS.vz = inflow_vz ? inflow_vz[ny * z + y] : 0;
	}
};

template <typename DREAL, typename COLL, typename EQ>
using HarnessConfig = LBM_CONFIG<
	HarnessTraits<DREAL>,
	D3Q27_KernelStruct,
	HarnessData<HarnessTraits<DREAL>>,
	COLL,
	EQ,
	HarnessStreaming<HarnessTraits<DREAL>>,
	D3Q27_BC_All,
	D3Q27_MACRO_Default<HarnessTraits<DREAL>>>;

// neighbour indices as kernelInitIndices (kernels.h:5-57), A-A branch, single
// block (no distribution)
template <typename NSE>
inline void init_indices(
	typename NSE::DATA& SD,
	typename NSE::TRAITS::map_t map,
	long x,
	long y,
	long z,
	long& xp,
	long& xm,
	long& yp,
	long& ym,
	long& zp,
	long& zm
)
{
	if (NSE::BC::isPeriodic(map)) {
		xp = (x == SD.X() - 1) ? 0 : (x + 1);
		xm = (x == 0) ? (SD.X() - 1) : (x - 1);
		yp = (y == SD.Y() - 1) ? 0 : (y + 1);
		ym = (y == 0) ? (SD.Y() - 1) : (y - 1);
		zp = (z == SD.Z() - 1) ? 0 : (z + 1);
		zm = (z == 0) ? (SD.Z() - 1) : (z - 1);
	}
	else {
#ifdef AB_PATTERN
		xp = std::min(x + 1, (long) SD.X() - 1);
		xm = std::max(x - 1, 0L);
		yp = std::min(y + 1, (long) SD.Y() - 1);
		ym = std::max(y - 1, 0L);
		zp = std::min(z + 1, (long) SD.Z() - 1);
		zm = std::max(z - 1, 0L);
#else
		xp = x + 1;
		xm = x - 1;
		yp = y + 1;
		ym = y - 1;
		zp = z + 1;
		zm = z - 1;
#endif
	}
}

// one lattice-site update, the body of cudaLBMKernel / LBMKernel (kernels.h:92-111)
template <typename NSE>
inline void site_update(typename NSE::DATA& SD, long x, long y, long z, bool output_macro)
{
	using dreal = typename NSE::TRAITS::dreal;
	const auto gi_map = SD.map(x, y, z);
	long xp, xm, yp, ym, zp, zm;
	init_indices<NSE>(SD, gi_map, x, y, z, xp, xm, yp, ym, zp, zm);

	typename NSE::template KernelStruct<dreal> KS;
	NSE::MACRO::copyQuantities(SD, KS, x, y, z);
	NSE::MACRO::template computeForcing<typename NSE::BC>(SD, KS, xm, x, xp, ym, y, yp, zm, z, zp);
	NSE::BC::preCollision(SD, KS, gi_map, xm, x, xp, ym, y, yp, zm, z, zp);
	if (NSE::BC::doCollision(gi_map))
		NSE::COLL::collision(KS);
	NSE::BC::postCollision(SD, KS, gi_map, xm, x, xp, ym, y, yp, zm, z, zp);
	if (output_macro)
		NSE::MACRO::outputMacro(SD, KS, x, y, z);
}

// site types whose A-A update reads a slot that another site writes in the same
// pass (GEO_INFLOW_BB_LEFT bc.h:155-163, GEO_OUTFLOW_RIGHT bc.h:73-74); with
// these present the harness runs single-threaded in the reference loop order
bool map_is_order_dependent(const short* map, long n)
{
#ifdef AB_PATTERN
	(void) map;
	(void) n;
	return false;  // A-B reads only the previous step's buffer
#else
	for (long i = 0; i < n; i++)
		if (map[i] == 4 || map[i] == 7)
			return true;
	return false;
#endif
}

bool map_is_supported(const short* map, long n)
{
	for (long i = 0; i < n; i++) {
#ifdef AB_PATTERN
		if (map[i] < 0 || map[i] > 16)
			return false;
#else
		if (map[i] < 0 || map[i] == 8 || map[i] > 16)
			return false;
#endif
	}
	return true;
}

template <typename DREAL, int Q = 27>
void canonical_to_ref(const DREAL* src, DREAL* dst, long X, long Y, long Z)
{
	const long XYZ = (X + 2) * (Y + 2) * (Z + 2);
	for (int q = 0; q < Q; q++)
		for (long z = 0; z < Z + 2; z++)
			for (long y = 0; y < Y + 2; y++)
				for (long x = 0; x < X + 2; x++)
					dst[q * XYZ + (x * (Z + 2) + z) * (Y + 2) + y] = src[q * XYZ + (z * (Y + 2) + y) * (X + 2) + x];
}

// The same conversion into a freshly allocated, untouched buffer, with the
// (x, z) rows split over the threads as the time loop splits them (static
// schedule), so that each thread's pages are first touched, and therefore
// placed, on its own NUMA node as in the reference's OpenMP host path.
template <typename DREAL, int Q = 27>
void canonical_to_ref_first_touch(const DREAL* src, DREAL* dst, long X, long Y, long Z, int threads)
{
	const long XYZ = (X + 2) * (Y + 2) * (Z + 2);
#pragma omp parallel for schedule(static) collapse(2) num_threads(threads)
	for (long x = 0; x < X + 2; x++)
		for (long z = 0; z < Z + 2; z++)
			for (int q = 0; q < Q; q++)
				for (long y = 0; y < Y + 2; y++)
					dst[q * XYZ + (x * (Z + 2) + z) * (Y + 2) + y] = src[q * XYZ + (z * (Y + 2) + y) * (X + 2) + x];
}

template <typename DREAL, int Q = 27>
void ref_to_canonical(const DREAL* src, DREAL* dst, long X, long Y, long Z)
{
	const long XYZ = (X + 2) * (Y + 2) * (Z + 2);
	for (int q = 0; q < Q; q++)
		for (long z = 0; z < Z + 2; z++)
			for (long y = 0; y < Y + 2; y++)
				for (long x = 0; x < X + 2; x++)
					dst[q * XYZ + (z * (Y + 2) + y) * (X + 2) + x] = src[q * XYZ + (x * (Z + 2) + z) * (Y + 2) + y];
}

template <typename NSE>
int run_aa(
	long X,
	long Y,
	long Z,
	typename NSE::TRAITS::dreal* f_canonical,
	const short* map,
	double nu,
	double fx,
	double fy,
	double fz,
	const double* in_vx,
	const double* in_vy,
	const double* in_vz,
	typename NSE::TRAITS::dreal* macro,
	long start_iter,
	int nsteps,
	int nthreads,
	double* elapsed_s
)
{
	using dreal = typename NSE::TRAITS::dreal;
	const long n = X * Y * Z;
	if (! map_is_supported(map, n))
		return -2;
	const long XYZ = (X + 2) * (Y + 2) * (Z + 2);
	const bool sequential = map_is_order_dependent(map, n);
#ifdef _OPENMP
	const int threads = sequential ? 1 : (nthreads > 0 ? nthreads : omp_get_max_threads());
#else
	const int threads = 1;
	(void) nthreads;
	(void) sequential;
#endif
	// populations in the reference's order, first touched by the threads that
	// update them (new[] leaves the buffer untouched)
	std::unique_ptr<dreal[]> df_owner(new dreal[27 * XYZ]);
	dreal* const df = df_owner.get();
	canonical_to_ref_first_touch(f_canonical, df, X, Y, Z, threads);

	std::vector<dreal> pvx, pvy, pvz;
	auto convert_profile = [&](const double* src, std::vector<dreal>& dst) -> const dreal*
	{
		if (! src)
			return nullptr;
		dst.resize(Y * Z);
		for (long i = 0; i < Y * Z; i++)
			dst[i] = (dreal) src[i];
		return dst.data();
	};

	typename NSE::DATA SD;
	SD.nx = X;
	SD.ny = Y;
	SD.nz = Z;
	SD.XYZ = XYZ;
	SD.lbmViscosity = (dreal) nu;
	SD.fx = (dreal) fx;
	SD.fy = (dreal) fy;
	SD.fz = (dreal) fz;
	SD.dfs[df_cur] = df;
#ifdef AB_PATTERN
	// the write buffer starts as a copy: ghost and GEO_NOTHING entries are
	// never written and must hold the same values in both buffers
	std::vector<dreal> df2(df, df + 27 * XYZ);
	SD.dfs[df_out] = df2.data();
#endif
	SD.dmacro = macro;
	SD.dmap = map;
	SD.inflow_vx = convert_profile(in_vx, pvx);
	SD.inflow_vy = convert_profile(in_vy, pvy);
	SD.inflow_vz = convert_profile(in_vz, pvz);

	g_unsupported_hit = 0;
	const auto t0 = std::chrono::steady_clock::now();
	for (int s = 0; s < nsteps; s++) {
		// LBM::updateKernelData (lbm.hpp:311)
		SD.even_iter = ((start_iter + s) % 2) == 0;
		const bool output_macro = macro != nullptr;
		// host loop of State::SimUpdate (state.hpp:1388-1397): x, z outer, y inner
#pragma omp parallel for schedule(static) collapse(2) num_threads(threads)
		for (long x = 0; x < X; x++)
			for (long z = 0; z < Z; z++)
				for (long y = 0; y < Y; y++)
					site_update<NSE>(SD, x, y, z, output_macro);
#ifdef AB_PATTERN
		std::swap(SD.dfs[df_cur], SD.dfs[df_out]);	// pointer rotation of lbm.hpp:314-322
#endif
	}
	const auto t1 = std::chrono::steady_clock::now();
	if (elapsed_s)
		*elapsed_s = std::chrono::duration<double>(t1 - t0).count();
	ref_to_canonical(SD.dfs[df_cur], f_canonical, X, Y, Z);
	return g_unsupported_hit ? -3 : 0;
}

template <typename DREAL, typename COLL, typename EQ>
int run_aa_typed(
	long X,
	long Y,
	long Z,
	void* f,
	const short* map,
	double nu,
	double fx,
	double fy,
	double fz,
	const double* vx,
	const double* vy,
	const double* vz,
	void* macro,
	long start_iter,
	int nsteps,
	int nthreads,
	double* elapsed
)
{
	using NSE = HarnessConfig<DREAL, COLL, EQ>;
	return run_aa<NSE>(
		X, Y, Z, (DREAL*) f, map, nu, fx, fy, fz, vx, vy, vz, (DREAL*) macro, start_iter, nsteps, nthreads, elapsed
	);
}

template <typename DREAL, typename EQ>
int dispatch_coll(int coll, long X, long Y, long Z, void* f, const short* map, double nu, double fx, double fy, double fz,
				  const double* vx, const double* vy, const double* vz, void* macro, long it, int ns, int nt, double* el)
{
	using T = HarnessTraits<DREAL>;
	switch (coll) {
		case 0:
			return run_aa_typed<DREAL, D3Q27_CUM<T, EQ>, EQ>(X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro, it, ns, nt, el);
		case 1:
			return run_aa_typed<DREAL, D3Q27_SRT<T, EQ>, EQ>(X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro, it, ns, nt, el);
		case 2:
			return run_aa_typed<DREAL, D3Q27_BGK<T, EQ>, EQ>(X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro, it, ns, nt, el);
		case 3:
			return run_aa_typed<DREAL, D3Q27_MRT<T, EQ>, EQ>(X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro, it, ns, nt, el);
		default:
			return -1;
	}
}

#ifndef AB_PATTERN
// ---- coupled D3Q7 advection-diffusion (State_NSE_ADE) ------------------------
// Kernel data of the scalar: ADE_Data + ADE_Data_ConstInflow (lbm_data.h:211-262)
// over the harness indexer.  The phase-transfer arrays are not provided; the
// harness rejects maps that would read them.
template <typename TRAITS>
struct HarnessAdeData : HarnessData<TRAITS>
{
	using idx = typename TRAITS::idx;
	using dreal = typename TRAITS::dreal;

	const dreal* dcoef = nullptr;  // per-site diffusion [Z][Y][X] or null
	dreal inflow_phi = 1;
	dreal phiTransferCoefficient = 0;

	dreal diffusionCoefficient(idx x, idx y, idx z) const
	{
		return dcoef ? dcoef[(z * this->ny + y) * this->nx + x] : this->lbmViscosity;
	}

	bool& phiTransferDirection(int, idx, idx, idx)
	{
		static bool none = false;
		g_unsupported_hit = 1;
		return none;
	}

	template <typename LBM_KS>
	void inflow(LBM_KS& KS, idx, idx, idx)
	{
		KS.phi = inflow_phi;
	}
};

template <typename DREAL, typename COLL>
using HarnessAdeConfig = LBM_CONFIG<
	HarnessTraits<DREAL>,
	D3Q7_KernelStruct,
	HarnessAdeData<HarnessTraits<DREAL>>,
	COLL,
	D3Q7_EQ<HarnessTraits<DREAL>>,
	D3Q7_STREAMING<HarnessTraits<DREAL>>,
	D3Q7_BC_All,
	D3Q7_MACRO_Default<HarnessTraits<DREAL>>>;

// one site of the coupled kernel cudaLBMKernel<NSE, ADE> (kernels.h:138-195)
template <typename NSE, typename ADE>
inline void coupled_update(typename NSE::DATA& SD, typename ADE::DATA& AD, long x, long y, long z, bool output_macro)
{
	using dreal = typename NSE::TRAITS::dreal;
	const auto nse_map = SD.map(x, y, z);
	const auto ade_map = AD.map(x, y, z);
	long xp, xm, yp, ym, zp, zm;
	init_indices<NSE>(SD, nse_map, x, y, z, xp, xm, yp, ym, zp, zm);

	typename NSE::template KernelStruct<dreal> KS;
	NSE::MACRO::copyQuantities(SD, KS, x, y, z);
	NSE::MACRO::template computeForcing<typename NSE::BC>(SD, KS, xm, x, xp, ym, y, yp, zm, z, zp);
	NSE::BC::preCollision(SD, KS, nse_map, xm, x, xp, ym, y, yp, zm, z, zp);
	if (NSE::BC::doCollision(nse_map))
		NSE::COLL::collision(KS);
	NSE::BC::postCollision(SD, KS, nse_map, xm, x, xp, ym, y, yp, zm, z, zp);
	if (output_macro)
		NSE::MACRO::outputMacro(SD, KS, x, y, z);

	typename ADE::template KernelStruct<dreal> AKS;
	AKS.vx = KS.vx;
	AKS.vy = KS.vy;
	AKS.vz = KS.vz;
	ADE::MACRO::copyQuantities(AD, AKS, x, y, z);
	ADE::BC::preCollision(AD, AKS, ade_map, xm, x, xp, ym, y, yp, zm, z, zp);
	if (ADE::BC::doCollision(ade_map))
		ADE::COLL::collision(AKS);
	ADE::BC::postCollision(AD, AKS, ade_map, xm, x, xp, ym, y, yp, zm, z, zp);
	if (output_macro)
		ADE::MACRO::outputMacro(AD, AKS, x, y, z);
}

// scalar site types whose update depends on nothing but the site's own slots
// (the outflow and phase-transfer types read slots other sites write)
bool ade_map_is_supported(const short* map, long n)
{
	for (long i = 0; i < n; i++) {
		const short g = map[i];
		if (!(g == 0 || g == 1 || g == 2 || g == 3 || g == 7 || g == 9 || g == 10 || (g >= 12 && g <= 17)))
			return false;
	}
	return true;
}

template <typename NSE, typename ADE>
int run_aa_ade(long X, long Y, long Z, typename NSE::TRAITS::dreal* f_canonical, const short* map, double nu, double fx,
			   double fy, double fz, const double* in_vx, const double* in_vy, const double* in_vz,
			   typename NSE::TRAITS::dreal* macro, typename NSE::TRAITS::dreal* g_canonical, const short* ade_map, double D,
			   const double* dfield, double inflow_phi, typename NSE::TRAITS::dreal* phi, long start_iter, int nsteps)
{
	using dreal = typename NSE::TRAITS::dreal;
	const long n = X * Y * Z;
	if (!map_is_supported(map, n) || map_is_order_dependent(map, n) || !ade_map_is_supported(ade_map, n))
		return -2;
	if ((macro == nullptr) != (phi == nullptr))
		return -1;
	const long XYZ = (X + 2) * (Y + 2) * (Z + 2);
	std::vector<dreal> df(27 * XYZ), dg(7 * XYZ);
	canonical_to_ref<dreal, 27>(f_canonical, df.data(), X, Y, Z);
	canonical_to_ref<dreal, 7>(g_canonical, dg.data(), X, Y, Z);
	std::vector<dreal> pvx, pvy, pvz, pd;
	auto convert = [](const double* src, long m, std::vector<dreal>& dst) -> const dreal*
	{
		if (!src)
			return nullptr;
		dst.resize(m);
		for (long i = 0; i < m; i++)
			dst[i] = (dreal) src[i];
		return dst.data();
	};

	typename NSE::DATA SD;
	SD.nx = X;
	SD.ny = Y;
	SD.nz = Z;
	SD.XYZ = XYZ;
	SD.lbmViscosity = (dreal) nu;
	SD.fx = (dreal) fx;
	SD.fy = (dreal) fy;
	SD.fz = (dreal) fz;
	SD.dfs[df_cur] = df.data();
	SD.dmacro = macro;
	SD.dmap = map;
	SD.inflow_vx = convert(in_vx, Y * Z, pvx);
	SD.inflow_vy = convert(in_vy, Y * Z, pvy);
	SD.inflow_vz = convert(in_vz, Y * Z, pvz);

	typename ADE::DATA AD;
	AD.nx = X;
	AD.ny = Y;
	AD.nz = Z;
	AD.XYZ = XYZ;
	AD.lbmViscosity = (dreal) D;
	AD.dfs[df_cur] = dg.data();
	AD.dmacro = phi;
	AD.dmap = ade_map;
	AD.dcoef = convert(dfield, n, pd);
	AD.inflow_phi = (dreal) inflow_phi;

	g_unsupported_hit = 0;
	for (int s = 0; s < nsteps; s++) {
		SD.even_iter = AD.even_iter = ((start_iter + s) % 2) == 0;
		const bool output_macro = macro != nullptr;
		for (long x = 0; x < X; x++)
			for (long z = 0; z < Z; z++)
				for (long y = 0; y < Y; y++)
					coupled_update<NSE, ADE>(SD, AD, x, y, z, output_macro);
	}
	ref_to_canonical<dreal, 27>(SD.dfs[df_cur], f_canonical, X, Y, Z);
	ref_to_canonical<dreal, 7>(AD.dfs[df_cur], g_canonical, X, Y, Z);
	return g_unsupported_hit ? -3 : 0;
}

template <typename T>
struct TypeTag
{
	using type = T;
};

template <typename DREAL, typename NSE_COLL, typename EQ>
int ade_dispatch(int ade_coll, long X, long Y, long Z, void* f, const short* map, double nu, double fx, double fy, double fz,
				 const double* vx, const double* vy, const double* vz, void* macro, void* g, const short* ade_map, double D,
				 const double* dfield, double inflow_phi, void* phi, long it, int ns)
{
	using T = HarnessTraits<DREAL>;
	using NSE = HarnessConfig<DREAL, NSE_COLL, EQ>;
	auto run = [&](auto ade_tag) -> int
	{
		using ADE = HarnessAdeConfig<DREAL, typename decltype(ade_tag)::type>;
		return run_aa_ade<NSE, ADE>(X, Y, Z, (DREAL*) f, map, nu, fx, fy, fz, vx, vy, vz, (DREAL*) macro, (DREAL*) g, ade_map, D,
									dfield, inflow_phi, (DREAL*) phi, it, ns);
	};
	switch (ade_coll) {
		case 0:
			return run(TypeTag<D3Q7_SRT<T>>{});
		case 1:
			return run(TypeTag<D3Q7_MRT<T>>{});
		case 2:
			return run(TypeTag<D3Q7_CLBM<T>>{});
		default:
			return -1;
	}
}

template <typename DREAL, typename EQ>
int ade_dispatch_nse(int coll, int ade_coll, long X, long Y, long Z, void* f, const short* map, double nu, double fx, double fy,
					 double fz, const double* vx, const double* vy, const double* vz, void* macro, void* g, const short* ade_map,
					 double D, const double* dfield, double inflow_phi, void* phi, long it, int ns)
{
	using T = HarnessTraits<DREAL>;
	switch (coll) {
		case 0:
			return ade_dispatch<DREAL, D3Q27_CUM<T, EQ>, EQ>(ade_coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro, g, ade_map, D,
															 dfield, inflow_phi, phi, it, ns);
		case 1:
			return ade_dispatch<DREAL, D3Q27_SRT<T, EQ>, EQ>(ade_coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro, g, ade_map, D,
															 dfield, inflow_phi, phi, it, ns);
		case 2:
			return ade_dispatch<DREAL, D3Q27_BGK<T, EQ>, EQ>(ade_coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro, g, ade_map, D,
															 dfield, inflow_phi, phi, it, ns);
		case 3:
			return ade_dispatch<DREAL, D3Q27_MRT<T, EQ>, EQ>(ade_coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro, g, ade_map, D,
															 dfield, inflow_phi, phi, it, ns);
		default:
			return -1;
	}
}

// per-site scalar collision: computeDensityAndVelocity then COLL::collision
// (d3q7/common.h:15-26, col_*.h) on n sites g[n][7] with velocities v[n][3]
template <typename DREAL, typename COLL>
int ade_collide_typed(long n, DREAL* g, const double* v, DREAL* phi_out, double D)
{
	for (long s = 0; s < n; s++) {
		D3Q7_KernelStruct<DREAL> KS;
		for (int q = 0; q < 7; q++)
			KS.f[q] = g[s * 7 + q];
		KS.vx = (DREAL) v[3 * s];
		KS.vy = (DREAL) v[3 * s + 1];
		KS.vz = (DREAL) v[3 * s + 2];
		KS.lbmViscosity = (DREAL) D;
		COLL::computeDensityAndVelocity(KS);
		if (phi_out)
			phi_out[s] = KS.phi;
		COLL::collision(KS);
		for (int q = 0; q < 7; q++)
			g[s * 7 + q] = KS.f[q];
	}
	return 0;
}
#endif	// !AB_PATTERN

// equilibrium of one site through the collision's inherited setEquilibriumLat
// (common.h:127-158), which takes rho and u in `real` (double)
template <typename DREAL, typename EQ>
void eq_into(DREAL* out27, double rho, double vx, double vy, double vz)
{
	struct View
	{
		DREAL* p;
		DREAL& operator()(int q, long, long, long)
		{
			return p[q];
		}
	} v{out27};
	D3Q27_COMMON<HarnessTraits<DREAL>, EQ>::setEquilibriumLat(v, 0, 0, 0, rho, vx, vy, vz);
}

template <typename DREAL, typename EQ>
int init_eq_typed(long X, long Y, long Z, DREAL* f, const double* rho, const double* vx, const double* vy, const double* vz,
				  double rho0, double vx0, double vy0, double vz0)
{
	const long XYZ = (X + 2) * (Y + 2) * (Z + 2);
	DREAL site[27];
	for (long z = -1; z <= Z; z++)
		for (long y = -1; y <= Y; y++)
			for (long x = -1; x <= X; x++) {
				const bool interior = x >= 0 && x < X && y >= 0 && y < Y && z >= 0 && z < Z;
				const long i = (z * Y + y) * X + x;
				if (interior && rho)
					eq_into<DREAL, EQ>(site, rho[i], vx[i], vy[i], vz[i]);
				else
					eq_into<DREAL, EQ>(site, rho0, vx0, vy0, vz0);
				const long s = ((z + 1) * (Y + 2) + (y + 1)) * (X + 2) + (x + 1);
				for (int q = 0; q < 27; q++)
					f[q * XYZ + s] = site[q];
			}
	return 0;
}

template <typename DREAL, typename COLL>
int collide_typed(long n, DREAL* f, DREAL* macro_out, double nu, double fx, double fy, double fz)
{
	for (long s = 0; s < n; s++) {
		D3Q27_KernelStruct<DREAL> KS;
		for (int q = 0; q < 27; q++)
			KS.f[q] = f[s * 27 + q];
		KS.lbmViscosity = (DREAL) nu;
		KS.fx = (DREAL) fx;
		KS.fy = (DREAL) fy;
		KS.fz = (DREAL) fz;
		COLL::computeDensityAndVelocity(KS);
		if (macro_out) {
			macro_out[s * 4 + 0] = KS.rho;
			macro_out[s * 4 + 1] = KS.vx;
			macro_out[s * 4 + 2] = KS.vy;
			macro_out[s * 4 + 3] = KS.vz;
		}
		COLL::collision(KS);
		for (int q = 0; q < 27; q++)
			f[s * 27 + q] = KS.f[q];
	}
	return 0;
}

template <typename DREAL, typename EQ>
int collide_dispatch(int coll, long n, void* f, void* m, double nu, double fx, double fy, double fz)
{
	using T = HarnessTraits<DREAL>;
	switch (coll) {
		case 0:
			return collide_typed<DREAL, D3Q27_CUM<T, EQ>>(n, (DREAL*) f, (DREAL*) m, nu, fx, fy, fz);
		case 1:
			return collide_typed<DREAL, D3Q27_SRT<T, EQ>>(n, (DREAL*) f, (DREAL*) m, nu, fx, fy, fz);
		case 2:
			return collide_typed<DREAL, D3Q27_BGK<T, EQ>>(n, (DREAL*) f, (DREAL*) m, nu, fx, fy, fz);
		case 3:
			return collide_typed<DREAL, D3Q27_MRT<T, EQ>>(n, (DREAL*) f, (DREAL*) m, nu, fx, fy, fz);
		default:
			return -1;
	}
}

// kernel struct of the adjoint configuration: the primary and the measured
// macro quantities that D3Q27_COMMON_ADJOINT::setEquilibrium reads
template <typename REAL>
struct HarnessAdjointKS : D3Q27_KernelStruct<REAL>
{
	REAL rho_m = 1.0, vx_m = 0, vy_m = 0, vz_m = 0;
};

// direction vectors in slot order (the enum of lbm3d/defs.h)
const int HCX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
const int HCY[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
const int HCZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1};

// data view for D3Q27_MACRO_Mean::outputMacro: 13 macro fields of n sites,
// field-major, and the statistics counter (lbm_data.h:24)
template <typename DREAL>
struct MeanData
{
	DREAL* m;
	long n;
	int stat_counter;
	DREAL& macro(int id, long x, long, long)
	{
		return m[id * n + x];
	}
};

template <typename DREAL>
int mean_update_typed(long n, const DREAL* macro4, DREAL* stats9, int counter)
{
	std::vector<DREAL> all((size_t) 13 * n);
	std::memcpy(all.data() + 4 * n, stats9, sizeof(DREAL) * 9 * n);
	MeanData<DREAL> SD{all.data(), n, counter};
	for (long i = 0; i < n; i++) {
		D3Q27_KernelStruct<DREAL> KS;
		KS.rho = macro4[i];
		KS.vx = macro4[n + i];
		KS.vy = macro4[2 * n + i];
		KS.vz = macro4[3 * n + i];
		D3Q27_MACRO_Mean<HarnessTraits<DREAL>>::outputMacro(SD, KS, i, 0, 0);
	}
	std::memcpy(stats9, all.data() + 4 * n, sizeof(DREAL) * 9 * n);
	return 0;
}

}  // namespace

extern "C" {

#ifndef AB_PATTERN
// Coupled flow + D3Q7 scalar steps (cudaLBMKernel<NSE, ADE>, kernels.h:114-196),
// single-threaded in the reference loop order.  prec, coll, eq, f, map,
// inflow, macro as ref_aa_run; ade_coll: 0 D3Q7_SRT, 1 D3Q7_MRT, 2 D3Q7_CLBM;
// g: [7][Z+2][Y+2][X+2] scalar populations, updated in place; ade_map:
// [Z][Y][X] scalar GEO types; D: diffusion coefficient, dfield: per-site
// [Z][Y][X] or NULL; inflow_phi: phi of GEO_INFLOW sites; phi: [Z][Y][X] output
// (together with macro) or NULL.  Returns -2 for maps with order-dependent or
// unprovided site types.
int ref_aa_ade_run(int prec, int coll, int eq, int ade_coll, long X, long Y, long Z, void* f, const short* map, double nu,
				   double fx, double fy, double fz, const double* vx, const double* vy, const double* vz, void* macro, void* g,
				   const short* ade_map, double D, const double* dfield, double inflow_phi, void* phi, long start_iter,
				   int nsteps)
{
	if (prec == 0) {
		if (eq == 0)
			return ade_dispatch_nse<double, D3Q27_EQ<HarnessTraits<double>>>(coll, ade_coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy,
																			 vz, macro, g, ade_map, D, dfield, inflow_phi, phi,
																			 start_iter, nsteps);
		return ade_dispatch_nse<double, D3Q27_EQ_INV_CUM<HarnessTraits<double>>>(coll, ade_coll, X, Y, Z, f, map, nu, fx, fy, fz,
																				 vx, vy, vz, macro, g, ade_map, D, dfield,
																				 inflow_phi, phi, start_iter, nsteps);
	}
	if (eq == 0)
		return ade_dispatch_nse<float, D3Q27_EQ<HarnessTraits<float>>>(coll, ade_coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz,
																	   macro, g, ade_map, D, dfield, inflow_phi, phi, start_iter,
																	   nsteps);
	return ade_dispatch_nse<float, D3Q27_EQ_INV_CUM<HarnessTraits<float>>>(coll, ade_coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy,
																		   vz, macro, g, ade_map, D, dfield, inflow_phi, phi,
																		   start_iter, nsteps);
}

// Per-site scalar collision on n sites (FP64): g[n][7] in place, v[n][3]
// velocities, phi_out[n] the pre-collision phi or NULL.
int ref_ade_collide(int ade_coll, long n, double* g, const double* v, double* phi_out, double D)
{
	using T = HarnessTraits<double>;
	switch (ade_coll) {
		case 0:
			return ade_collide_typed<double, D3Q7_SRT<T>>(n, g, v, phi_out, D);
		case 1:
			return ade_collide_typed<double, D3Q7_MRT<T>>(n, g, v, phi_out, D);
		case 2:
			return ade_collide_typed<double, D3Q7_CLBM<T>>(n, g, v, phi_out, D);
		default:
			return -1;
	}
}
#endif

// One statistics update of D3Q27_MACRO_Mean::outputMacro (macro.h:117-171) on
// n sites: macro4 [4][n] (rho, vx, vy, vz) of the step, stats9 [9][n] (mean
// velocity, co-moments) updated in place, counter = SD.stat_counter.
int ref_mean_update(int prec, long n, const void* macro4, void* stats9, int counter)
{
	if (prec == 0)
		return mean_update_typed<double>(n, (const double*) macro4, (double*) stats9, counter);
	return mean_update_typed<float>(n, (const float*) macro4, (float*) stats9, counter);
}

// The reference's adjoint SRT collision (col_srt_adjoint.h:50-109) on n
// independent sites: fstar[n][27] updated in place, primary velocity u[n][3].
int ref_srt_adjoint_collision(long n, double* fstar, const double* u, double nu)
{
	using T = HarnessTraits<double>;
	for (long s = 0; s < n; s++) {
		HarnessAdjointKS<double> KS;
		for (int q = 0; q < 27; q++)
			KS.f[q] = fstar[s * 27 + q];
		KS.vx = u[s * 3 + 0];
		KS.vy = u[s * 3 + 1];
		KS.vz = u[s * 3 + 2];
		KS.lbmViscosity = nu;
		D3Q27_SRT_ADJOINT<T>::collision(KS);
		for (int q = 0; q < 27; q++)
			fstar[s * 27 + q] = KS.f[q];
	}
	return 0;
}

// The reference's adjoint data term D3Q27_EQ_ADJOINT::collisionWithData
// (eq_adjoint.h:30-33) for every direction: macro[n][8] = primary rho, vx,
// vy, vz and measured rho_m, vx_m, vy_m, vz_m; out[n][27].
int ref_adjoint_data_term(long n, const double* macro, double* out)
{
	using EQ = D3Q27_EQ_ADJOINT<HarnessTraits<double>>;
	for (long s = 0; s < n; s++) {
		const double* m = macro + s * 8;
		for (int q = 0; q < 27; q++)
			out[s * 27 + q] = EQ::collisionWithData(HCX[q], HCY[q], HCZ[q], m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7]);
	}
	return 0;
}


// Flags this build was compiled with: bit0 USE_GEIER_CUM_2017, bit1 USE_GEIER_CUM_ANTIALIAS.
int ref_cum_flags(void)
{
	int flags = 0;
#ifdef USE_GEIER_CUM_2017
	flags |= 1;
#endif
#ifdef USE_GEIER_CUM_ANTIALIAS
	flags |= 2;
#endif
	return flags;
}

// prec: 0 = double, 1 = float.  coll: 0 CUM, 1 SRT, 2 BGK, 3 MRT.
// eq: 0 = D3Q27_EQ (eq.h), 1 = D3Q27_EQ_INV_CUM (eq_inv_cum.h).
// f: [27][Z+2][Y+2][X+2] (x fastest), updated in place.  map: [Z][Y][X] GEO values.
// inflow profiles: [Z][Y] or NULL.  macro: [4][Z][Y][X] (rho, vx, vy, vz) or NULL.
#ifdef AB_PATTERN
	#define LBM_HARNESS_RUN ref_ab_run
#else
	#define LBM_HARNESS_RUN ref_aa_run
#endif
int LBM_HARNESS_RUN(int prec, int coll, int eq, long X, long Y, long Z, void* f, const short* map, double nu, double fx, double fy,
			   double fz, const double* vx, const double* vy, const double* vz, void* macro, long start_iter, int nsteps,
			   int nthreads, double* elapsed_s)
{
	if (prec == 0) {
		if (eq == 0)
			return dispatch_coll<double, D3Q27_EQ<HarnessTraits<double>>>(coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro,
																		  start_iter, nsteps, nthreads, elapsed_s);
		return dispatch_coll<double, D3Q27_EQ_INV_CUM<HarnessTraits<double>>>(coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz,
																			  macro, start_iter, nsteps, nthreads, elapsed_s);
	}
	if (eq == 0)
		return dispatch_coll<float, D3Q27_EQ<HarnessTraits<float>>>(coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro,
																	start_iter, nsteps, nthreads, elapsed_s);
	return dispatch_coll<float, D3Q27_EQ_INV_CUM<HarnessTraits<float>>>(coll, X, Y, Z, f, map, nu, fx, fy, fz, vx, vy, vz, macro,
																		start_iter, nsteps, nthreads, elapsed_s);
}

// Equilibrium populations on every site incl. the ghost layer, as
// LBM_BLOCK::setEquilibrium (lbm_block.hpp:248-278).  rho/vx/vy/vz are [Z][Y][X]
// fields for the interior (or NULL for the uniform state rho0, v0).
int ref_init_equilibrium(int prec, int eq, long X, long Y, long Z, void* f, const double* rho, const double* vx, const double* vy,
						 const double* vz, double rho0, double vx0, double vy0, double vz0)
{
	if (prec == 0) {
		if (eq == 0)
			return init_eq_typed<double, D3Q27_EQ<HarnessTraits<double>>>(X, Y, Z, (double*) f, rho, vx, vy, vz, rho0, vx0, vy0, vz0);
		return init_eq_typed<double, D3Q27_EQ_INV_CUM<HarnessTraits<double>>>(X, Y, Z, (double*) f, rho, vx, vy, vz, rho0, vx0, vy0,
																			  vz0);
	}
	if (eq == 0)
		return init_eq_typed<float, D3Q27_EQ<HarnessTraits<float>>>(X, Y, Z, (float*) f, rho, vx, vy, vz, rho0, vx0, vy0, vz0);
	return init_eq_typed<float, D3Q27_EQ_INV_CUM<HarnessTraits<float>>>(X, Y, Z, (float*) f, rho, vx, vy, vz, rho0, vx0, vy0, vz0);
}

// Per-site collision: computeDensityAndVelocity (common.h:17-50) then
// COLL::collision on n independent sites f[n][27]; macro_out[n][4] or NULL.
int ref_collide(int prec, int coll, int eq, long n, void* f, void* macro_out, double nu, double fx, double fy, double fz)
{
	if (prec == 0) {
		if (eq == 0)
			return collide_dispatch<double, D3Q27_EQ<HarnessTraits<double>>>(coll, n, f, macro_out, nu, fx, fy, fz);
		return collide_dispatch<double, D3Q27_EQ_INV_CUM<HarnessTraits<double>>>(coll, n, f, macro_out, nu, fx, fy, fz);
	}
	if (eq == 0)
		return collide_dispatch<float, D3Q27_EQ<HarnessTraits<float>>>(coll, n, f, macro_out, nu, fx, fy, fz);
	return collide_dispatch<float, D3Q27_EQ_INV_CUM<HarnessTraits<float>>>(coll, n, f, macro_out, nu, fx, fy, fz);
}

// Equilibrium of n sites, out[n][27].
int ref_equilibrium(int prec, int eq, long n, const double* rho, const double* vx, const double* vy, const double* vz, void* out)
{
	for (long s = 0; s < n; s++) {
		if (prec == 0) {
			double* o = (double*) out + s * 27;
			if (eq == 0)
				eq_into<double, D3Q27_EQ<HarnessTraits<double>>>(o, rho[s], vx[s], vy[s], vz[s]);
			else
				eq_into<double, D3Q27_EQ_INV_CUM<HarnessTraits<double>>>(o, rho[s], vx[s], vy[s], vz[s]);
		}
		else {
			float* o = (float*) out + s * 27;
			if (eq == 0)
				eq_into<float, D3Q27_EQ<HarnessTraits<float>>>(o, rho[s], vx[s], vy[s], vz[s]);
			else
				eq_into<float, D3Q27_EQ_INV_CUM<HarnessTraits<float>>>(o, rho[s], vx[s], vy[s], vz[s]);
		}
	}
	return 0;
}

}  // extern "C"
