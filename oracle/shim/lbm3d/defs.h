// Oracle-only replacement for TNL-LBM's include/lbm3d/defs.h.
//
// The reference's per-site operator headers (include/lbm3d/d3q27/*.h) include
// "lbm3d/defs.h", which pulls in TNL, MPI and the NDArray machinery.  None of
// that is needed to evaluate the per-site arithmetic, so this header restates
// only the pieces the operator headers reference:
//   - the A-A / A-B pattern switch and the DF buffer enum (defs.h:20-67)
//   - the D3Q27 kernel struct                             (defs.h:255-276)
//   - the plugin composition template LBM_CONFIG          (defs.h:288-310)
//   - the 27-direction enum, whose numbering is part of
//     the population-slot interface                        (defs.h:318-350)
// Test infrastructure only: the product library never includes it.
#pragma once

#include <cstdint>
#include <math.h>
#include <utility>

#include <TNL/Backend/Macros.h>

#if ! defined(AB_PATTERN) && ! defined(AA_PATTERN)
	#define AA_PATTERN
#endif

#define CUDA_HOSTDEV

#ifdef AB_PATTERN
// A-B pattern: read buffer and write buffer, swapped every step (defs.h:54-60)
enum : std::uint8_t
{
	df_cur,
	df_out,
	DFMAX
};
#else
// A-A pattern keeps a single in-place population buffer (defs.h:61-66)
enum : std::uint8_t
{
	df_cur,
	DFMAX
};
#endif

// KernelStruct - D3Q7 (field set and defaults as defs.h:244-252)
template <typename REAL>
struct D3Q7_KernelStruct
{
	static constexpr int Q = 7;
	REAL f[Q];
	REAL vz = 0, vx = 0, vy = 0;
	REAL phi = 1.0, lbmViscosity = 1.0;
};

// KernelStruct - D3Q27 (field set and defaults as defs.h:257-263)
template <typename REAL>
struct D3Q27_KernelStruct
{
	static constexpr int Q = 27;
	REAL f[Q];
	REAL fz = 0, fx = 0, fy = 0;
	REAL vz = 0, vx = 0, vy = 0;
	REAL rho = 1.0, lbmViscosity = 1.0;
};

template <
	typename _TRAITS,
	template <typename> class _KERNEL_STRUCT,
	typename _DATA,
	typename _COLL,
	typename _EQ,
	typename _STREAMING,
	template <typename> class _BC,
	typename _MACRO>
struct LBM_CONFIG
{
	using TRAITS = _TRAITS;
	template <typename REAL>
	using KernelStruct = _KERNEL_STRUCT<REAL>;
	using DATA = _DATA;
	using COLL = _COLL;
	using EQ = _EQ;
	using STREAMING = _STREAMING;
	using BC = _BC<LBM_CONFIG>;
	using MACRO = _MACRO;

	static constexpr int Q = KernelStruct<typename TRAITS::dreal>::Q;
};

// population directions; the numbering is the slot order of the DF arrays
enum : std::uint8_t
{
	zzz = 0,
	pzz = 1,
	mzz = 2,
	zpz = 3,
	zmz = 4,
	zzp = 5,
	zzm = 6,
	ppz = 7,
	mmz = 8,
	pmz = 9,
	mpz = 10,
	pzp = 11,
	mzm = 12,
	pzm = 13,
	mzp = 14,
	zpp = 15,
	zmm = 16,
	zpm = 17,
	zmp = 18,
	ppp = 19,
	mmm = 20,
	ppm = 21,
	mmp = 22,
	pmp = 23,
	mpm = 24,
	pmm = 25,
	mpp = 26,
};
