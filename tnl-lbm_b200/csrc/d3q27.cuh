// D3Q27 lattice constants and population storage formats for the sm_100a
// kernels.
//
// Direction numbering is the slot order of TNL-LBM's population arrays
// (include/lbm3d/defs.h:318-350): zzz, pzz, mzz, zpz, zmz, zzp, zzm, ppz,
// mmz, pmz, mpz, pzp, mzm, pzm, mzp, zpp, zmm, zpm, zmp, ppp, mmm, ppm, mmp,
// pmp, mpm, pmm, mpp.  Opposite directions are adjacent pairs (1,2), (3,4), ...
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace lbm {

enum Dir : int
{
	ZZZ, PZZ, MZZ, ZPZ, ZMZ, ZZP, ZZM, PPZ, MMZ, PMZ, MPZ, PZP, MZM, PZM, MZP,
	ZPP, ZMM, ZPM, ZMP, PPP, MMM, PPM, MMP, PMP, MPM, PMM, MPP
};

__host__ __device__ constexpr int cx(int q)
{
	constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
	return t[q];
}
__host__ __device__ constexpr int cy(int q)
{
	constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
	return t[q];
}
__host__ __device__ constexpr int cz(int q)
{
	constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1};
	return t[q];
}
__host__ __device__ constexpr int opp(int q)
{
	return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1);
}
// velocity components for a runtime direction index: (c + 1) packed in 2 bits
// per direction into one 64-bit constant, so that no table is materialised
__host__ __device__ constexpr unsigned long long pack_components(int axis)
{
	unsigned long long p = 0;
	for (int q = 0; q < 27; q++) {
		const int c = axis == 0 ? cx(q) : (axis == 1 ? cy(q) : cz(q));
		p |= (unsigned long long) (c + 1) << (2 * q);
	}
	return p;
}
__host__ __device__ __forceinline__ int cx_rt(int q)
{
	return (int) ((pack_components(0) >> (2 * q)) & 3ull) - 1;
}
__host__ __device__ __forceinline__ int cy_rt(int q)
{
	return (int) ((pack_components(1) >> (2 * q)) & 3ull) - 1;
}
__host__ __device__ __forceinline__ int cz_rt(int q)
{
	return (int) ((pack_components(2) >> (2 * q)) & 3ull) - 1;
}
// number of non-zero velocity components: 0 rest, 1 face, 2 edge, 3 corner
__host__ __device__ constexpr int nnz(int q)
{
	return (cx(q) != 0) + (cy(q) != 0) + (cz(q) != 0);
}
// direction index from components (used with compile-time arguments)
__host__ __device__ constexpr int dir(int x, int y, int z)
{
	int r = -1;
	for (int q = 0; q < 27; q++)
		if (cx(q) == x && cy(q) == y && cz(q) == z)
			r = q;
	return r;
}
// lattice weights w_q
__host__ __device__ constexpr double weight(int q)
{
	return nnz(q) == 0 ? 8.0 / 27.0 : nnz(q) == 1 ? 2.0 / 27.0 : nnz(q) == 2 ? 1.0 / 54.0 : 1.0 / 216.0;
}
// exact power-of-two scale applied to the FP16 deviations: the smallest 2^k
// with 2^k >= 1/w_q, so that (f_q - w_q) * 2^k stays in FP16's normal range
__host__ __device__ constexpr float half_scale(int q)
{
	return nnz(q) == 0 ? 4.0f : nnz(q) == 1 ? 16.0f : nnz(q) == 2 ? 64.0f : 256.0f;
}

// quantum of the 16-bit fixed-point deviation format (StoreI16S): the
// power of two that spreads the deviations |f_q - w_q| <= 0.42 w_q over the
// signed 16-bit range (32767 q = 0.42 w_q for every weight class)
__host__ __device__ constexpr float fixed_quantum(int q)
{
	return nnz(q) == 0 ? 0x1p-18f : nnz(q) == 1 ? 0x1p-20f : nnz(q) == 2 ? 0x1p-22f : 0x1p-24f;
}

// GEO site types of D3Q27_BC_All (include/lbm3d/d3q27/bc.h:17-43); the map
// stores these values as uint8
enum Geo : uint8_t
{
	GEO_FLUID = 0,
	GEO_WALL = 1,
	GEO_INFLOW = 2,
	GEO_INFLOW_LEFT = 3,
	GEO_INFLOW_BB_LEFT = 4,
	GEO_INFLOW_EQ_LEFT = 5,
	GEO_OUTFLOW_EQ = 6,
	GEO_OUTFLOW_RIGHT = 7,
	GEO_OUTFLOW_RIGHT_INTERP = 8,
	GEO_PERIODIC = 9,
	GEO_NOTHING = 10,
	GEO_SYM_TOP = 11,
	GEO_SYM_BOTTOM = 12,
	GEO_SYM_LEFT = 13,
	GEO_SYM_RIGHT = 14,
	GEO_SYM_BACK = 15,
	GEO_SYM_FRONT = 16,
};

// Groups of the two-site step (pair.cuh): a lattice row is cut into groups of
// PAIR_GROUP x-sites (32 bytes of a slot row in FP32, one DRAM sector, as the
// interior x = 0 of a row is 128-byte aligned; 16 bytes in the 16-bit
// formats), and a group whose sites are all GEO_FLUID or all GEO_PERIODIC
// runs in the two-site update.  Groups of 8 took the duct 1-3 % above groups
// of 16: half as many sites on the per-site path.
constexpr int PAIR_GROUP = 8;
enum : uint8_t
{
	PAIR_GROUP_REST = 0,
	PAIR_GROUP_FLUID = 1,
	PAIR_GROUP_PERIODIC = 2
};
// work item of the pair step with a map: a chunk of the rest-site list when
// this bit is set, else a tile of a row
constexpr unsigned PAIR_WORK_REST = 0x80000000u;

// ---------------------------------------------------------------------------
// population storage formats
//   F64   double  f_q
//   F32   float   f_q
//   F32S  float   f_q - w_q
//   F16S  half    (f_q - w_q) * half_scale(q)
//   BF16S bf16    f_q - w_q
//   F16SR, BF16SR as F16S and BF16S, rounded stochastically on store
//   I16S  int16   round((f_q - w_q) / fixed_quantum(q)), clamped to +-32767
// Every format is read into the compute type R and written back from it.
// ---------------------------------------------------------------------------
struct StoreF64
{
	using T = double;
	using R = double;
	template <int Q>
	__device__ static __forceinline__ R load(const T* p)
	{
		return __ldcs(p);
	}
	template <int Q>
	__device__ static __forceinline__ void store(T* p, R v)
	{
		__stcs(p, v);
	}
	template <int Q>
	__device__ static __forceinline__ R load_smem(const T* p)
	{
		return *p;
	}
};

struct StoreF32
{
	using T = float;
	using R = float;
	template <int Q>
	__device__ static __forceinline__ R load(const T* p)
	{
		return __ldcs(p);
	}
	template <int Q>
	__device__ static __forceinline__ void store(T* p, R v)
	{
		__stcs(p, v);
	}
	template <int Q>
	__device__ static __forceinline__ R load_smem(const T* p)
	{
		return *p;
	}
};

struct StoreF32S
{
	using T = float;
	using R = float;
	template <int Q>
	__device__ static __forceinline__ R load(const T* p)
	{
		return __ldcs(p) + (float) weight(Q);
	}
	template <int Q>
	__device__ static __forceinline__ void store(T* p, R v)
	{
		__stcs(p, v - (float) weight(Q));
	}
	template <int Q>
	__device__ static __forceinline__ R load_smem(const T* p)
	{
		return *p + (float) weight(Q);
	}
};

struct StoreF16S
{
	using T = __half;
	using R = float;
	template <int Q>
	__device__ static __forceinline__ R load(const T* p)
	{
		const unsigned short raw = __ldcs(reinterpret_cast<const unsigned short*>(p));
		return __half2float(__ushort_as_half(raw)) * (1.0f / half_scale(Q)) + (float) weight(Q);
	}
	// (v - w) * s as one fused multiply-add, v * s - w * s with w * s exact
	// (s a power of two): one rounding instead of two, one instruction less
	template <int Q>
	__device__ static __forceinline__ float scaled_deviation(R v)
	{
		return __fmaf_rn(v, half_scale(Q), -(float) weight(Q) * half_scale(Q));
	}
	template <int Q>
	__device__ static __forceinline__ void store(T* p, R v)
	{
		const __half h = __float2half_rn(scaled_deviation<Q>(v));
		__stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(h));
	}
	template <int Q>
	__device__ static __forceinline__ R load_smem(const T* p)
	{
		return __half2float(*p) * (1.0f / half_scale(Q)) + (float) weight(Q);
	}
};

// Stochastic rounding of a float to a 16-bit format that keeps the top
// 32 - DROP bits: a pseudo-random integer below 2^DROP is added to the bit
// pattern, then the low bits are cut (round toward zero), so that a value is
// rounded up with probability equal to its distance from the lower neighbour.
// The random bits come from a multiplicative hash of the value's own bit
// pattern (Knuth's golden-ratio constant): no generator state, reproducible
// results, and a different draw whenever the value changes from one step to
// the next.  The thresholds are uniform over the values a site takes, so the
// rounding error has zero mean and the storage error of a slowly varying
// field does not drift the way round-to-nearest does.
template <int DROP>
__device__ __forceinline__ float stochastic_round_bits(float x)
{
	const unsigned b = __float_as_uint(x);
	return __uint_as_float(b + ((b * 0x9E3779B1u) >> (32 - DROP)));
}

struct StoreF16SR : StoreF16S
{
	template <int Q>
	__device__ static __forceinline__ void store(T* p, R v)
	{
		// a normal half keeps 10 of the float's 23 mantissa bits: 13 are dropped
		const float x = stochastic_round_bits<13>(scaled_deviation<Q>(v));
		const __half h = __float2half_rz(x);
		__stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(h));
	}
};

struct StoreBF16S
{
	using T = __nv_bfloat16;
	using R = float;
	template <int Q>
	__device__ static __forceinline__ R load(const T* p)
	{
		const unsigned short raw = __ldcs(reinterpret_cast<const unsigned short*>(p));
		return __bfloat162float(__ushort_as_bfloat16(raw)) + (float) weight(Q);
	}
	template <int Q>
	__device__ static __forceinline__ void store(T* p, R v)
	{
		const __nv_bfloat16 h = __float2bfloat16_rn(v - (float) weight(Q));
		__stcs(reinterpret_cast<unsigned short*>(p), __bfloat16_as_ushort(h));
	}
	template <int Q>
	__device__ static __forceinline__ R load_smem(const T* p)
	{
		return __bfloat162float(*p) + (float) weight(Q);
	}
};

struct StoreBF16SR : StoreBF16S
{
	template <int Q>
	__device__ static __forceinline__ void store(T* p, R v)
	{
		// bfloat16 keeps 7 of the float's 23 mantissa bits: 16 are dropped, and
		// cutting them is exact truncation of the bit pattern
		const float x = stochastic_round_bits<16>(v - (float) weight(Q));
		const unsigned short h = (unsigned short) (__float_as_uint(x) >> 16);
		__stcs(reinterpret_cast<unsigned short*>(p), h);
	}
};

// 16-bit fixed-point deviations: the integer i = round((f - w) / q) with the
// power-of-two quantum q = fixed_quantum(Q), kept as the unsigned 16-bit
// pattern of i + 32768.  Over its range |f - w| <= 0.42 w every value carries
// the same absolute resolution q / 2 = 6.5e-6 w, where FP16 keeps 11
// significant bits of the deviation itself (a relative 2.4e-4): about 5x finer
// at the deviations of u = 0.05 flows (0.15 w), coarser only below 0.03 w.
// Deviations beyond the range are clamped (densities outside 1 +- 0.3 at low
// Mach number); a NaN is kept as the one pattern the clamp never produces
// (0, i = -32768) and read back as NaN, so the non-finite count of the sums
// still sees it.  The conversions are exact integer-float bit patterns: an
// integer below 2^16 ORed into the mantissa of 2^23 is the float 2^23 + u, and
// a float in [2^23, 2^24) has the integer part of its value in the low
// mantissa bits, so the round to nearest of the store is one addition.
struct StoreI16S
{
	using T = short;
	using R = float;
	static constexpr float BIAS = 8421376.0f;	// 2^23 + 2^15
	static constexpr float ROUND = 12615680.0f;	// 1.5 * 2^23 + 2^15
	// f from the stored pattern u = i + 2^15 (0: NaN)
	template <int Q>
	__device__ static __forceinline__ R from_raw(unsigned u)
	{
		const float i = __uint_as_float(0x4B000000u | u) - BIAS;  // exact
		const float f = __fmaf_rn(i, fixed_quantum(Q), (float) weight(Q));
		return u ? f : __uint_as_float(0x7FFFFFFFu);
	}
	// the stored pattern of f: (f - w) / q as one fused multiply-add (1 / q
	// and w / q exact), clamped, rounded to nearest by the magic addition
	template <int Q>
	__device__ static __forceinline__ unsigned to_raw(R v)
	{
		const float d = __fmaf_rn(v, 1.0f / fixed_quantum(Q), -(float) weight(Q) / fixed_quantum(Q));
		const unsigned u = __float_as_uint(fminf(fmaxf(d, -32767.0f), 32767.0f) + ROUND) & 0xFFFFu;
		return d == d ? u : 0u;
	}
	template <int Q>
	__device__ static __forceinline__ R load(const T* p)
	{
		return from_raw<Q>(__ldcs(reinterpret_cast<const unsigned short*>(p)));
	}
	template <int Q>
	__device__ static __forceinline__ void store(T* p, R v)
	{
		__stcs(reinterpret_cast<unsigned short*>(p), (unsigned short) to_raw<Q>(v));
	}
	template <int Q>
	__device__ static __forceinline__ R load_smem(const T* p)
	{
		return from_raw<Q>(*reinterpret_cast<const unsigned short*>(p));
	}
};

}  // namespace lbm
