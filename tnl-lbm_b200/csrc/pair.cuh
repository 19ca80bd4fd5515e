// Two-site A-A step for sm_100a: every thread updates the x-adjacent sites
// (x, x + 1) of one lattice row, and the cumulant collision of both runs on
// the packed FP32 instructions of sm_100 (add/mul/fma on .f32x2 operands,
// __fadd2_rn / __fmul2_rn / __ffma2_rn), which issue one instruction for two
// values.  The two sites share their y and z neighbour offsets, and the
// directions without an x component (and every direction of the even step)
// move both sites' populations with one 8-byte (FP32) or 4-byte (16-bit)
// access.
//
// The per-site algorithm is that of aa_step_kernel (aa_kernels.cuh): A-A
// read and write of streaming_AA.h, D3Q27_BC_All (bc.h) through
// apply_boundary, and the cumulant collision of col_cum.h.  On a lattice with
// a map, the groups of sites that are all GEO_FLUID (or all GEO_PERIODIC) take
// the two-site update and every other site the per-site update, both in one
// launch over a host-built work list; A-A sites are independent within a
// step, so the order of the work items does not change the result.
#pragma once

#include "aa_kernels.cuh"
#include "coll_params.cuh"
#include "launch.h"

namespace lbm {

// two FP32 lanes
struct F2
{
	float2 v;
	F2() = default;
	__host__ __device__ __forceinline__ F2(double a) : v{(float) a, (float) a} {}
	__host__ __device__ __forceinline__ F2(float a, float b) : v{a, b} {}
	__host__ __device__ __forceinline__ explicit F2(float2 a) : v(a) {}
};

__device__ __forceinline__ F2 operator+(F2 a, F2 b)
{
	return F2(__fadd2_rn(a.v, b.v));
}
__device__ __forceinline__ F2 operator-(F2 a)
{
	return F2(make_float2(-a.v.x, -a.v.y));
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b)
{
	return F2(__fadd2_rn(a.v, make_float2(-b.v.x, -b.v.y)));
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b)
{
	return F2(__fmul2_rn(a.v, b.v));
}
// per lane, IEEE division as the scalar form
__device__ __forceinline__ F2 operator/(F2 a, F2 b)
{
	return F2(a.v.x / b.v.x, a.v.y / b.v.y);
}
__device__ __forceinline__ F2& operator*=(F2& a, F2 b)
{
	a = a * b;
	return a;
}
__device__ __forceinline__ F2& operator+=(F2& a, F2 b)
{
	a = a + b;
	return a;
}
__device__ __forceinline__ F2& operator-=(F2& a, F2 b)
{
	a = a - b;
	return a;
}
// a * b + c, one rounding per lane
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c)
{
	return F2(__ffma2_rn(a.v, b.v, c.v));
}
__device__ __forceinline__ F2 fabs(F2 a)
{
	return F2(fabsf(a.v.x), fabsf(a.v.y));
}
// per lane, correctly rounded as the scalar form
__device__ __forceinline__ F2 sqrt(F2 a)
{
	return F2(sqrtf(a.v.x), sqrtf(a.v.y));
}
// 1 / rho of the SRT forcing per lane, 1 where rho = 0 (inv_rho_or_one)
__device__ __forceinline__ F2 inv_rho_or_one(const Site<F2>& s)
{
	return F2(s.rho.v.x == 0.0f ? 1.0f : s.ir.v.x, s.rho.v.y == 0.0f ? 1.0f : s.ir.v.y);
}
template <>
__device__ __forceinline__ F2 rcp<F2>(F2 x)
{
	return F2(__frcp_rn(x.v.x), __frcp_rn(x.v.y));
}
template <>
__device__ __forceinline__ F2 div_approx<F2>(F2 a, F2 b)
{
	return F2(__fdividef(a.v.x, b.v.x), __fdividef(a.v.y, b.v.y));
}

// Chimera transforms of collide_cumulant with the multiply-adds written out
// (the compiler fuses a * b + c only for scalar operands), in the order of the
// scalar forms.
__device__ __forceinline__ void chim_fwd(F2& m, F2& z, F2& p, F2 u, F2 u2)
{
	const F2 s = p + m, d = p - m;
	const F2 k0 = s + z;
	m = k0;
	z = fma2(-u, k0, d);
	p = fma2(u2, k0, fma2(-(u + u), d, s));
}
__device__ __forceinline__ void chim_bwd(F2& a, F2& b, F2& c, F2 u, F2 u2)
{
	const F2 k0 = a, k1 = b, k2 = c;
	const F2 s = fma2(k0, u2, fma2(u + u, k1, k2));
	const F2 hd = F2(0.5) * fma2(u, k0, k1);
	a = fma2(s, F2(0.5), -hd);
	b = k0 - s;
	c = fma2(s, F2(0.5), hd);
}

// ---------------------------------------------------------------------------
// two-site accesses per storage format: load2 / store2 move the populations
// of sites (x, x + 1) at p, p + 1 (p 8-byte aligned for FP32, 4-byte for the
// 16-bit formats); Q is the slot, as for the scalar S::load / S::store
// ---------------------------------------------------------------------------
template <typename S>
struct PairIO;

template <>
struct PairIO<StoreF32>
{
	template <int Q>
	__device__ static __forceinline__ F2 load2(const float* p)
	{
		return F2(__ldcs(reinterpret_cast<const float2*>(p)));
	}
	template <int Q>
	__device__ static __forceinline__ void store2(float* p, F2 v)
	{
		__stcs(reinterpret_cast<float2*>(p), v.v);
	}
};

template <>
struct PairIO<StoreF32S>
{
	template <int Q>
	__device__ static __forceinline__ F2 load2(const float* p)
	{
		return F2(__ldcs(reinterpret_cast<const float2*>(p))) + F2(weight(Q));
	}
	template <int Q>
	__device__ static __forceinline__ void store2(float* p, F2 v)
	{
		__stcs(reinterpret_cast<float2*>(p), (v - F2(weight(Q))).v);
	}
};

template <>
struct PairIO<StoreF16S>
{
	template <int Q>
	__device__ static __forceinline__ F2 load2(const __half* p)
	{
		const F2 h(__half22float2(__ldcs(reinterpret_cast<const __half2*>(p))));
		return fma2(h, F2(1.0 / half_scale(Q)), F2(weight(Q)));
	}
	// (v - w) * s as v * s - w * s, as StoreF16S::scaled_deviation
	template <int Q>
	__device__ static __forceinline__ F2 scaled_deviation(F2 v)
	{
		return fma2(v, F2(half_scale(Q)), F2(-(float) weight(Q) * half_scale(Q)));
	}
	template <int Q>
	__device__ static __forceinline__ void store2(__half* p, F2 v)
	{
		__stcs(reinterpret_cast<__half2*>(p), __float22half2_rn(scaled_deviation<Q>(v).v));
	}
};

template <>
struct PairIO<StoreF16SR> : PairIO<StoreF16S>
{
	template <int Q>
	__device__ static __forceinline__ void store2(__half* p, F2 v)
	{
		const F2 d = scaled_deviation<Q>(v);
		const __half lo = __float2half_rz(stochastic_round_bits<13>(d.v.x));
		const __half hi = __float2half_rz(stochastic_round_bits<13>(d.v.y));
		__stcs(reinterpret_cast<__half2*>(p), __halves2half2(lo, hi));
	}
};

template <>
struct PairIO<StoreBF16S>
{
	template <int Q>
	__device__ static __forceinline__ F2 load2(const __nv_bfloat16* p)
	{
		return F2(__bfloat1622float2(__ldcs(reinterpret_cast<const __nv_bfloat162*>(p)))) + F2(weight(Q));
	}
	template <int Q>
	__device__ static __forceinline__ void store2(__nv_bfloat16* p, F2 v)
	{
		__stcs(reinterpret_cast<__nv_bfloat162*>(p), __float22bfloat162_rn((v - F2(weight(Q))).v));
	}
};

template <>
struct PairIO<StoreBF16SR> : PairIO<StoreBF16S>
{
	template <int Q>
	__device__ static __forceinline__ void store2(__nv_bfloat16* p, F2 v)
	{
		const F2 d = v - F2(weight(Q));
		const unsigned lo = __float_as_uint(stochastic_round_bits<16>(d.v.x)) >> 16;
		const unsigned hi = __float_as_uint(stochastic_round_bits<16>(d.v.y)) & 0xffff0000u;
		__stcs(reinterpret_cast<unsigned*>(p), lo | hi);
	}
};

template <>
struct PairIO<StoreI16S>
{
	// both sites' patterns from one 32-bit word: each 16-bit half into the
	// mantissa of 2^23 (byte permutes), the bias off as one packed addition
	template <int Q>
	__device__ static __forceinline__ F2 load2(const short* p)
	{
		const unsigned w = __ldcs(reinterpret_cast<const unsigned*>(p));
		const F2 x(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7610)), __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7632)));
		const F2 f = fma2(x - F2(StoreI16S::BIAS), F2(fixed_quantum(Q)), F2(weight(Q)));
		const float nan = __uint_as_float(0x7FFFFFFFu);
		return F2((w & 0xFFFFu) ? f.v.x : nan, (w >> 16) ? f.v.y : nan);  // pattern 0: NaN
	}
	template <int Q>
	__device__ static __forceinline__ void store2(short* p, F2 v)
	{
		const F2 d = fma2(v, F2(1.0f / fixed_quantum(Q)), F2(-(float) weight(Q) / fixed_quantum(Q)));
		const F2 c(fminf(fmaxf(d.v.x, -32767.0f), 32767.0f), fminf(fmaxf(d.v.y, -32767.0f), 32767.0f));
		const F2 t = c + F2(StoreI16S::ROUND);
		const unsigned lo = d.v.x == d.v.x ? __float_as_uint(t.v.x) & 0xFFFFu : 0u;  // NaN: pattern 0
		const unsigned hi = d.v.y == d.v.y ? __float_as_uint(t.v.y) << 16 : 0u;
		__stcs(reinterpret_cast<unsigned*>(p), lo | hi);
	}
};

// x offsets of a pair: the left neighbour of site x and the right neighbour
// of site x + 1 (the other two are the pair's own sites); periodic sites wrap
struct PairX
{
	int left;	// -1, or X - 1 for a periodic site at x = 0
	int right;	// +1, or -(X - 1) for a periodic site at x + 1 = X - 1
};

// A-A read of both sites with shared y and z offsets (o.y, o.z of either site)
template <typename S, bool ODD>
__device__ __forceinline__ void pair_read(const typename S::T* __restrict__ f, long long sq, long long base, const Offsets& o,
										  PairX px, Site<F2>& s)
{
	using IO = PairIO<S>;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (!ODD)
				s.f[q] = IO::template load2<q>(f + q * sq + base);
			else {
				// direction q of site x comes from slot opp(q) of site x - c_q
				const typename S::T* c = f + opp(q) * sq + base + o.y[1 - cy(q)] + o.z[1 - cz(q)];
				if constexpr (cx(q) == 0)
					s.f[q] = IO::template load2<opp(q)>(c);
				else if constexpr (cx(q) > 0)
					s.f[q] = F2(S::template load<opp(q)>(c + px.left), S::template load<opp(q)>(c));
				else
					s.f[q] = F2(S::template load<opp(q)>(c + 1), S::template load<opp(q)>(c + 1 + px.right));
			}
		}
	);
}

// A-A write of both sites, the mirror of pair_read
template <typename S, bool ODD>
__device__ __forceinline__ void pair_write(typename S::T* __restrict__ f, long long sq, long long base, const Offsets& o, PairX px,
										   const Site<F2>& s)
{
	using IO = PairIO<S>;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (!ODD)
				IO::template store2<opp(q)>(f + opp(q) * sq + base, s.f[q]);
			else {
				// direction q of site x goes to slot q of site x + c_q
				typename S::T* c = f + q * sq + base + o.y[1 + cy(q)] + o.z[1 + cz(q)];
				if constexpr (cx(q) == 0)
					IO::template store2<q>(c, s.f[q]);
				else if constexpr (cx(q) > 0) {
					S::template store<q>(c + 1, s.f[q].v.x);
					S::template store<q>(c + 1 + px.right, s.f[q].v.y);
				}
				else {
					S::template store<q>(c + px.left, s.f[q].v.x);
					S::template store<q>(c, s.f[q].v.y);
				}
			}
		}
	);
}

// Addresses of the two-site kernels without 64-bit multiplies: the byte
// offsets q sq sizeof(T) of the 27 slot rows of a lattice row come from the
// kernel parameters (constant-bank operands), the rows of the pair's three z
// planes from three pointers, and the y neighbours from three offsets, so an
// access is one pointer plus two offsets.  (Formed as f + q * sq + ..., every
// access took 64-bit integer multiply-adds, which run on the FMA pipe that
// the 16-bit formats' collision already fills.)
struct PairSlots
{
	int b[27];
};

inline PairSlots make_pair_slots(long long sq, int elem)
{
	PairSlots ps;
	for (int q = 0; q < 27; q++)
		ps.b[q] = (int) (q * sq * elem);
	return ps;
}

struct PairAt
{
	char* P[3];		   // row (y, x of the first site) in planes z - 1, z, z + 1
	long long oy[3];   // byte offsets of rows y - 1, y, y + 1 from row y
	int left, right;   // x offsets (elements) of the pair's outer neighbours, as PairX
};

// neighbours of the pair (x, x + 1) of row (y, z) of the population array f
// (element size E bytes, strides in elements): periodic sites wrap in x and
// y (wrap) and in z (wrap && zwrap), all others reach the ghost layer
__device__ __forceinline__ PairAt pair_at_of(char* f, long long E, int sy, int sz, int x0, int X, int Y, int Z, int x, int y,
											 int z, bool wrap, bool zwrap)
{
	PairAt at;
	const int zm = (wrap && zwrap && z == 0) ? Z - 1 : z - 1;
	const int zp = (wrap && zwrap && z == Z - 1) ? 0 : z + 1;
	const long long ry = (long long) (y + 1) * sy + x0 + x;
	at.P[0] = f + ((long long) (zm + 1) * sz + ry) * E;
	at.P[1] = f + ((long long) (z + 1) * sz + ry) * E;
	at.P[2] = f + ((long long) (zp + 1) * sz + ry) * E;
	at.oy[0] = (long long) ((wrap && y == 0) ? Y - 1 : -1) * sy * E;
	at.oy[1] = 0;
	at.oy[2] = (long long) ((wrap && y == Y - 1) ? -(Y - 1) : 1) * sy * E;
	at.left = (wrap && x == 0) ? X - 1 : -1;
	at.right = (wrap && x + 1 == X - 1) ? -(X - 1) : 1;
	return at;
}

template <typename T>
__device__ __forceinline__ PairAt pair_at(const StepArgs<T, float>& a, int x, int y, int z, bool wrap)
{
	return pair_at_of(reinterpret_cast<char*>(a.f), (long long) sizeof(T), a.sy, a.sz, a.x0, a.X, a.Y, a.Z, x, y, z, wrap,
					  a.zwrap != 0);
}

// pair_read with the addresses of PairAt / PairSlots
template <typename S, bool ODD>
__device__ __forceinline__ void pair_read_at(const PairAt& at, const PairSlots& ps, Site<F2>& s)
{
	using T = typename S::T;
	using IO = PairIO<S>;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (!ODD)
				s.f[q] = IO::template load2<q>(reinterpret_cast<const T*>(at.P[1] + ps.b[q]));
			else {
				// direction q of site x comes from slot opp(q) of site x - c_q
				const T* c = reinterpret_cast<const T*>(at.P[1 - cz(q)] + at.oy[1 - cy(q)] + ps.b[opp(q)]);
				if constexpr (cx(q) == 0)
					s.f[q] = IO::template load2<opp(q)>(c);
				else if constexpr (cx(q) > 0)
					s.f[q] = F2(S::template load<opp(q)>(c + at.left), S::template load<opp(q)>(c));
				else
					s.f[q] = F2(S::template load<opp(q)>(c + 1), S::template load<opp(q)>(c + 1 + at.right));
			}
		}
	);
}

// pair_write with the addresses of PairAt / PairSlots
template <typename S, bool ODD>
__device__ __forceinline__ void pair_write_at(const PairAt& at, const PairSlots& ps, const Site<F2>& s)
{
	using T = typename S::T;
	using IO = PairIO<S>;
	static_for<27>(
		[&](auto Qc)
		{
			constexpr int q = decltype(Qc)::value;
			if constexpr (!ODD)
				IO::template store2<opp(q)>(reinterpret_cast<T*>(at.P[1] + ps.b[opp(q)]), s.f[q]);
			else {
				// direction q of site x goes to slot q of site x + c_q
				T* c = reinterpret_cast<T*>(at.P[1 + cz(q)] + at.oy[1 + cy(q)] + ps.b[q]);
				if constexpr (cx(q) == 0)
					IO::template store2<q>(c, s.f[q]);
				else if constexpr (cx(q) > 0) {
					S::template store<q>(c + 1, s.f[q].v.x);
					S::template store<q>(c + 1 + at.right, s.f[q].v.y);
				}
				else {
					S::template store<q>(c + at.left, s.f[q].v.x);
					S::template store<q>(c, s.f[q].v.y);
				}
			}
		}
	);
}

// outputs of an observation step for both sites (step_outputs of the scalar
// kernel); in = site inside the lattice; the warp's partial sums go to slot
// `slot` of nslots
template <typename T>
__device__ __forceinline__ void pair_outputs(const StepArgs<T, float>& a, bool inA, bool inB, long long site, const Site<F2>& s,
											 long long slot, long long nslots)
{
	if (a.macro) {
		const long long n = (long long) a.X * a.Y * a.Z;
		const F2 m[4] = {s.rho, s.vx, s.vy, s.vz};
#pragma unroll
		for (int k = 0; k < 4; k++) {
			if (inA)
				a.macro[k * n + site] = m[k].v.x;
			if (inB)
				a.macro[k * n + site + 1] = m[k].v.y;
		}
	}
	if (a.partials) {
		double red[NRED] = {0, 0, 0, 0, 0, 0};
		if (inA) {
			const double rho = s.rho.v.x, vx = s.vx.v.x, vy = s.vy.v.x, vz = s.vz.v.x;
			red[0] = rho;
			red[1] = rho * vx;
			red[2] = rho * vy;
			red[3] = rho * vz;
			red[4] = rho * (vx * vx + vy * vy + vz * vz);
			red[5] = isfinite(rho) ? 0.0 : 1.0;
		}
		if (inB) {
			const double rho = s.rho.v.y, vx = s.vx.v.y, vy = s.vy.v.y, vz = s.vz.v.y;
			red[0] += rho;
			red[1] += rho * vx;
			red[2] += rho * vy;
			red[3] += rho * vz;
			red[4] += rho * (vx * vx + vy * vy + vz * vz);
			red[5] += isfinite(rho) ? 0.0 : 1.0;
		}
		warp_reduce_store(red, a.partials, slot, nslots);
	}
}

// The update of the pair (x, x + 1) of row (y, z), cumulant collision on two
// lanes.  Without a map (GENERAL = false) every site is periodic and X is
// even.  With a map, the lattice rows are cut into groups of PAIR_GROUP sites
// (whole DRAM sectors of every slot row); groups[row * ceil(X / PAIR_GROUP) +
// x / PAIR_GROUP] is PAIR_GROUP_FLUID or PAIR_GROUP_PERIODIC when every site
// of the group has that type, and only those groups are updated here; the
// sites of the other groups (boundaries, obstacles, the lattice ends) take
// rest_update, one thread per site.  OUT: the macro field and the partial sums
// of the pair, the warp's sums in slot `slot` of nslots.  Every thread of the
// warp calls it (threads past the lattice with x >= X).
template <int COLL, int CUMF>
struct BuiltinCollision;
// true for the built-in collisions, false for a collision plugin's struct
template <typename C>
struct is_builtin_collision : std::false_type
{
};
template <int COLL, int CUMF>
struct is_builtin_collision<BuiltinCollision<COLL, CUMF>> : std::true_type
{
};

template <typename S, typename C, bool ODD, bool GENERAL, bool OUT>
__device__ __forceinline__ void pair_update(const StepArgs<typename S::T, float>& a, const CollParams<F2>& p2,
											const PairSlots& ps, const uint8_t* __restrict__ groups, int x, int y, int z,
											long long slot, long long nslots)
{
	bool act = x < a.X && y < a.Y;
	long long site = 0;
	Site<F2> s;
	PairAt at;
	if (act) {
		site = ((long long) z * a.Y + y) * a.X + x;
		if constexpr (GENERAL) {
			// a pair away from every lattice face has the same neighbours
			// whether it wraps or not: its loads are issued together with the
			// group flag's (and are discarded if the group is not a pair group)
			const bool inner = x > 0 && x + 2 < a.X && y > 0 && y < a.Y - 1 && z > 0 && z < a.Z - 1;
			if (inner) {
				at = pair_at(a, x, y, z, false);
				pair_read_at<S, ODD>(at, ps, s);
			}
			const int gx = (a.X + PAIR_GROUP - 1) / PAIR_GROUP;
			const uint8_t g = groups[((long long) z * a.Y + y) * gx + x / PAIR_GROUP];
			act = g != PAIR_GROUP_REST;
			if (act && !inner) {
				at = pair_at(a, x, y, z, g == PAIR_GROUP_PERIODIC);
				pair_read_at<S, ODD>(at, ps, s);
			}
		}
		else {
			at = pair_at(a, x, y, z, true);
			pair_read_at<S, ODD>(at, ps, s);
		}
		if (act)
			density_velocity(s, p2);
	}
	if constexpr (OUT && GENERAL) {
		// the work kernel: populations first, sums after the stores
		if (act) {
			C::template collision<F2>(s, p2);
			pair_write_at<S, ODD>(at, ps, s);
		}
		pair_outputs(a, act, act, site, s, slot, nslots);
		return;
	}
	else if constexpr (OUT)
		pair_outputs(a, act, act, site, s, slot, nslots);  // no map: before the collision (fewer live registers)
	else if constexpr (!GENERAL || sizeof(typename S::T) == 2 || !is_builtin_collision<C>::value)
		// keeps the collision after the loads (fewer live registers).  The work
		// kernel of 32-bit storage with a built-in collision runs without it:
		// its odd step then compiles without spills (80 bytes with it) and the
		// duct's FP32 step is 1.6 % faster (cumulant and MRT).  The 16-bit
		// formats are 1.2 % faster with it, and a collision plugin (4 blocks per
		// SM) 15 %
		__syncwarp();
	if (!act)
		return;
	C::template collision<F2>(s, p2);
	pair_write_at<S, ODD>(at, ps, s);
}

// The per-site update of aa_step_kernel for entry i of a host-built site list
// rest[i] = row << 32 | x with row = z Y + y (entries i >= n: no site);
// GEO_NOTHING sites only give their outputs.  OUT: macro field and partial
// sums, the warp's in slot `slot` of nslots.  Every thread of the warp calls it.
template <typename S, typename C, bool ODD, bool OUT>
__device__ __forceinline__ void rest_update(const StepArgs<typename S::T, float>& a, const unsigned long long* __restrict__ rest,
											long long n, long long i, long long slot, long long nslots)
{
	const bool in = i < n;
	if (!OUT && !in)
		return;
	Site<float> s;
	s.rho = 1.0f;
	s.vx = s.vy = s.vz = 0.0f;
	Offsets o;
	long long base = 0, site = 0;
	bool rw = false, coll = false;
	if (in) {
		const unsigned long long e = rest[i];
		const unsigned row = (unsigned) (e >> 32);
		const int x = (int) (e & 0xffffffffu);
		const int y = (int) (row % (unsigned) a.Y);
		const int z = (int) (row / (unsigned) a.Y);
		site = (long long) row * a.X + x;
		const uint8_t geo = a.map[site];
		if (geo != GEO_NOTHING) {
			const bool wrap = geo == GEO_PERIODIC;
			base = (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + x;
			o = neighbour_offsets(wrap, wrap && a.zwrap, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
			aa_read<S, ODD>(a.f, a.sq, base, o, s.f);
			coll = apply_boundary(s, geo, a, z, y);
			rw = true;
		}
	}
	if constexpr (OUT) {
		if (in && a.macro) {
			const long long nsites = (long long) a.X * a.Y * a.Z;
			a.macro[site] = s.rho;
			a.macro[nsites + site] = s.vx;
			a.macro[2 * nsites + site] = s.vy;
			a.macro[3 * nsites + site] = s.vz;
		}
		if (a.partials) {
			double red[NRED] = {0, 0, 0, 0, 0, 0};
			if (in) {
				const double rho = s.rho, vx = s.vx, vy = s.vy, vz = s.vz;
				red[0] = rho;
				red[1] = rho * vx;
				red[2] = rho * vy;
				red[3] = rho * vz;
				red[4] = rho * (vx * vx + vy * vy + vz * vz);
				red[5] = isfinite(rho) ? 0.0 : 1.0;
			}
			warp_reduce_store(red, a.partials, slot, nslots);
		}
	}
	if (!rw)
		return;
	if (coll)
		C::template collision<float>(s, a.p);
	aa_write<S, ODD>(a.f, a.sq, base, o, s.f);
}

// One A-A step of a lattice without a map, two sites per thread: thread
// (t, y) of the grid owns sites x = 2t and 2t + 1 of row (y, z = blockIdx.z).
template <typename S, typename C, bool ODD, bool OUT, int MINB>
__global__ void __launch_bounds__(128, MINB) aa_pair_kernel(const StepArgs<typename S::T, float> a, const CollParams<F2> p2,
															 const PairSlots ps, long long red_slots)
{
	if constexpr (OUT)
		launch_dependents();
	const int wpb = (blockDim.x * blockDim.y) >> 5;
	const long long block = blockIdx.x + (long long) gridDim.x * (blockIdx.y + (long long) gridDim.y * blockIdx.z);
	const long long slot = block * wpb + ((threadIdx.x + blockDim.x * threadIdx.y) >> 5);
	pair_update<S, C, ODD, false, OUT>(a, p2, ps, nullptr, 2 * (int) (blockIdx.x * blockDim.x + threadIdx.x),
										  blockIdx.y * blockDim.y + threadIdx.y, blockIdx.z, slot, red_slots);
}

// One A-A step of a lattice with a map in one launch of 128-thread blocks, each
// taking one item of a host-built work list, in z-plane order: a tile of 256
// x-sites of one row through pair_update (item = row * tiles_x + tile), or 128
// entries of the rest-site list through rest_update (item = PAIR_WORK_REST |
// chunk).  A plane's rest chunks come first and its pair tiles after them, so
// the rest sites run while the pair tiles around them are in flight and share
// their DRAM sectors through L2.  Warp w of block b writes partial-sum slot 4 b + w.
template <typename S, typename C, bool ODD, bool OUT, int MINB>
__global__ void __launch_bounds__(128, MINB)
	aa_pair_work_kernel(const StepArgs<typename S::T, float> a, const CollParams<F2> p2, const PairSlots ps,
						const uint8_t* __restrict__ groups, const unsigned* __restrict__ work,
						const unsigned long long* __restrict__ rest, long long nrest, int tiles_x)
{
	if constexpr (OUT)
		launch_dependents();
	const unsigned w = work[blockIdx.x];
	const long long slot = (long long) blockIdx.x * 4 + (threadIdx.x >> 5);
	const long long nslots = (long long) gridDim.x * 4;
	if (w & PAIR_WORK_REST) {
		rest_update<S, C, ODD, OUT>(a, rest, nrest, (long long) (w & ~PAIR_WORK_REST) * 128 + threadIdx.x, slot, nslots);
	}
	else {
		const unsigned row = w / (unsigned) tiles_x;
		const int x = (int) (w - row * (unsigned) tiles_x) * 256 + 2 * (int) threadIdx.x;
		pair_update<S, C, ODD, true, OUT>(a, p2, ps, groups, x, (int) (row % (unsigned) a.Y), (int) (row / (unsigned) a.Y),
											 slot, nslots);
	}
}

// Resident 128-thread blocks per SM requested for the pair kernel (register
// cap 65536 / (128 n)): the largest counts that compile without spills
// (-Xptxas -v on sm_100a).
template <typename T, int COLL, bool ODD>
constexpr int pair_minb()
{
	// even steps fit 96 registers without spills; odd steps spill up to 32
	// bytes at 96 in some variants and still run faster than at 4 blocks
	// (116-128 registers): duct
	// 25.2 GLUPS, Taylor-Green 512^3 27.5 against 27.2 at equal clocks.  The
	// even step of the 16-bit formats runs 6 blocks (80 registers, 8-32 bytes
	// of spills): duct F16S 35.2 against 34.4 GLUPS at 5
	if (COLL == COLL_SRT || COLL == COLL_BGK)
		return 4;
	return sizeof(T) == 2 && !ODD ? 6 : 5;
}
// A built-in collision of the COLL slot as a collision type of the two-site
// kernels (the shape a collision plugin's struct has, plugin.cuh), with its
// resident blocks per SM
template <int COLL, int CUMF>
struct BuiltinCollision
{
	template <typename R>
	__device__ static __forceinline__ void collision(Site<R>& s, const CollParams<R>& p)
	{
		collide<R, COLL, CUMF>(s, p);
	}
	template <typename T, bool ODD>
	static constexpr int pair_minb()
	{
		return lbm::pair_minb<T, COLL, ODD>();
	}
};

// One A-A step of collision type C (BuiltinCollision, or a collision
// plugin's struct) through aa_pair_kernel (no map) or aa_pair_work_kernel (a
// map); cudaErrorNotSupported for periodic lattices of odd width and for
// storage geometries the two-site accesses cannot align to.
template <typename S, typename C>
cudaError_t pair_step_with(const StepLaunch& L)
{
	using T = typename S::T;
	static_assert(sizeof(typename S::R) == 4, "the pair kernel computes in FP32");
	const bool general = L.map != nullptr;
	const bool out = L.macro || L.partials;
	// observation steps with the macro field run the work list that holds the
	// GEO_NOTHING sites (they output rho = 1, u = 0); a sums-only step runs
	// the plain list, and the finish kernel adds those sites' rho = 1 each
	const PairWork& W = L.macro ? L.pair_work_out : L.pair_work;
	if (general ? (!W.work || !L.pair_groups || W.nwork < 1) : (L.g.X % 2 != 0))
		return cudaErrorNotSupported;
	// 8- and 4-byte alignment of every pair's first site
	if ((L.g.x0 | L.g.sq | L.g.sy | L.g.sz) & 1)
		return cudaErrorNotSupported;
	StepArgs<T, float> a;
	a.f = (T*) L.g.f;
	a.sq = L.g.sq;
	a.sy = L.g.sy;
	a.sz = L.g.sz;
	a.x0 = L.g.x0;
	a.X = L.g.X;
	a.Y = L.g.Y;
	a.Z = L.g.Z;
	a.map = L.map;
	a.in_vx = (const float*) L.inflow[0];
	a.in_vy = (const float*) L.inflow[1];
	a.in_vz = (const float*) L.inflow[2];
	a.macro = (float*) L.macro;
	a.partials = L.partials;
	a.zwrap = L.distributed_z ? 0 : 1;
	a.p = make_coll_params<float>(L.p);
	const CollParams<F2> p2 = make_coll_params<F2>(L.p);
	// every slot offset of a lattice row fits 32 bits (sq < 2^26 elements)
	if (27ll * L.g.sq * (long long) sizeof(T) >= (1ll << 31))
		return cudaErrorNotSupported;
	const PairSlots ps = make_pair_slots(L.g.sq, (int) sizeof(T));
	const dim3 block = general ? dim3(128, 1, 1) : L.block;
	const int pairs = (L.g.X + 1) / 2;
	const dim3 grid = general ? dim3((unsigned) W.nwork, 1, 1)
							  : dim3((pairs + block.x - 1) / block.x, (L.g.Y + block.y - 1) / block.y, L.g.Z);
	// one partial-sum slot per warp
	const long long red_slots = (long long) grid.x * grid.y * grid.z * ((block.x * block.y) / 32);
	if (L.blocks_out)
		*L.blocks_out = red_slots;
	if (L.nothing_skipped)
		*L.nothing_skipped = general && L.partials && !L.macro;
	if (L.dry_run)
		return cudaSuccess;
	const int tiles_x = (pairs + 127) / 128;
	auto launch = [&](auto odd)
	{
		constexpr bool ODD = decltype(odd)::value;
		constexpr int MINB = C::template pair_minb<T, ODD>();
		if (general) {
			if (out)
				aa_pair_work_kernel<S, C, ODD, true, MINB>
					<<<grid, block, 0, L.stream>>>(a, p2, ps, L.pair_groups, W.work, W.rest, W.nrest, tiles_x);
			else
				aa_pair_work_kernel<S, C, ODD, false, MINB>
					<<<grid, block, 0, L.stream>>>(a, p2, ps, L.pair_groups, W.work, W.rest, W.nrest, tiles_x);
		}
		else if (out)
			aa_pair_kernel<S, C, ODD, true, MINB><<<grid, block, 0, L.stream>>>(a, p2, ps, red_slots);
		else
			aa_pair_kernel<S, C, ODD, false, MINB><<<grid, block, 0, L.stream>>>(a, p2, ps, red_slots);
	};
	if (L.odd)
		launch(std::true_type{});
	else
		launch(std::false_type{});
	return cudaGetLastError();
}

// One A-A step of the lattice's built-in collision on the two-site kernels;
// cudaErrorNotSupported where they do not apply (see pair_step_with)
template <typename S>
cudaError_t pair_step(const StepLaunch& L)
{
	switch (L.coll) {
		case COLL_SRT:
			return pair_step_with<S, BuiltinCollision<COLL_SRT, 0>>(L);
		case COLL_BGK:
			return pair_step_with<S, BuiltinCollision<COLL_BGK, 0>>(L);
		case COLL_MRT:
			return pair_step_with<S, BuiltinCollision<COLL_MRT, 0>>(L);
		case COLL_CUM:
			switch (L.cum_flags) {
				case 0:
					return pair_step_with<S, BuiltinCollision<COLL_CUM, 0>>(L);
				case CUM_ANTIALIAS:
					return pair_step_with<S, BuiltinCollision<COLL_CUM, CUM_ANTIALIAS>>(L);
				case CUM_2017 | CUM_ANTIALIAS:
					return pair_step_with<S, BuiltinCollision<COLL_CUM, CUM_2017 | CUM_ANTIALIAS>>(L);
				default:
					return cudaErrorInvalidValue;
			}
		default:
			return cudaErrorNotSupported;
	}
}

}  // namespace lbm

// defines cudaError_t lbm::FN(const StepLaunch&) for storage S
#define LBM_DEFINE_PAIR_STEP(FN, S)     \
	namespace lbm {                     \
	cudaError_t FN(const StepLaunch& L) \
	{                                   \
		return pair_step<S>(L);         \
	}                                   \
	}
