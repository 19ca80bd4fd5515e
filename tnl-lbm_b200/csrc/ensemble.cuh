// Ensemble step: many independent periodic lattices of different sizes and
// viscosities advanced by one persistent launch per A-A step.
//
// The reference runs one lattice per solver instance (one LBM_BLOCK per
// rank, include/lbm3d/lbm_block.h), so an ensemble there is a sequence of
// runs.  Small lattices (32^3 = 32768 sites) fill a fraction of a B200, so
// here all members share one launch: the sites of every member are cut into
// tiles of TPB consecutive sites (x fastest, rows wrap into the next row), a
// tile never spans two members, and a persistent grid walks the tile list.
// Each thread updates one site of a tile with the per-site code of the
// single-lattice kernel (aa_read, density_velocity, collide, aa_write), with
// the member's collision constants; the results equal the single-lattice
// kernel's bit for bit.
//
// Member table (device, one EnsMember per member): storage geometry of the
// member's own allocation region (same layout as a single lattice: ghost
// layer, 128-byte aligned rows), its collision constants, its first tile,
// and the constants of the division-free decode of a site index.
#pragma once

#include "aa_kernels.cuh"
#include "pair.cuh"

namespace lbm {

// Division by an invariant integer with a multiply-high (Granlund and
// Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994): for d >= 1, l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (umulhi(m, n) + n) >> l for every n < 2^31.
struct FastDiv
{
	unsigned m;
	int l;
	int d;
};

inline FastDiv make_fast_div(int d)
{
	int l = 0;
	while ((1ll << l) < d)
		l++;
	const unsigned long long m = ((1ull << 32) * ((1ull << l) - (unsigned long long) d)) / (unsigned long long) d + 1ull;
	return FastDiv{(unsigned) m, l, d};
}

__device__ __forceinline__ unsigned fast_div(unsigned n, const FastDiv& f)
{
	return (__umulhi(f.m, n) + n) >> f.l;
}

template <typename T, typename R>
struct EnsMember
{
	T* f;
	long long sq;
	int sy, sz, x0;
	int X, Y, Z;
	int n;			   // sites, X * Y * Z < 2^31
	long long tile0;   // first tile of the member in the ensemble's tile list
	FastDiv dx, dy;	   // division by X and by Y
	CollParams<R> p;
	CollParams<F2> p2;	// the same constants in both lanes (two-site kernel)
};

// One A-A step of every member.  OUT: per-tile FP64 partial sums
// (partials[k * ntiles + tile]) of the sums of lbm_get_sums.
template <typename S, int COLL, int CUMF, bool ODD, bool OUT, int TPB, int MINB>
__global__ void __launch_bounds__(TPB, MINB)
	ens_step_kernel(const EnsMember<typename S::T, typename S::R>* __restrict__ members, const int* __restrict__ tile_member,
					long long ntiles, double* __restrict__ partials)
{
	using T = typename S::T;
	using R = typename S::R;
	// the current member's table entry, staged in shared memory: its fields are
	// read where they are used instead of occupying registers
	__shared__ EnsMember<T, R> M;
	constexpr int WORDS = (int) (sizeof(EnsMember<T, R>) / 4);
	static_assert(sizeof(EnsMember<T, R>) % 4 == 0 && WORDS <= TPB, "member entry size");
	int cur = -1;
	for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
		const int m = tile_member[t];
		if (m != cur) {
			__syncthreads();  // every thread is done with the previous entry
			if ((int) threadIdx.x < WORDS)
				reinterpret_cast<unsigned*>(&M)[threadIdx.x] = reinterpret_cast<const unsigned*>(members + m)[threadIdx.x];
			__syncthreads();
			cur = m;
		}
		const unsigned i = (unsigned) ((t - M.tile0) * TPB) + threadIdx.x;
		double red[NRED] = {0, 0, 0, 0, 0, 0};
		if (i < (unsigned) M.n) {
			const unsigned row = fast_div(i, M.dx);
			const int x = (int) (i - row * (unsigned) M.X);
			const unsigned z = fast_div(row, M.dy);
			const int y = (int) (row - z * (unsigned) M.Y);
			const CollParams<R>& p = M.p;
			T* const f = M.f;
			const long long sq = M.sq;
			const long long base = (long long) (z + 1) * M.sz + (long long) (y + 1) * M.sy + M.x0 + x;
			const Offsets o = neighbour_offsets(true, x, (int) y, (int) z, M.X, M.Y, M.Z, M.sy, M.sz);
			Site<R> s;
			aa_read<S, ODD>(f, sq, base, o, s.f);
			density_velocity(s, p);
			collide<R, COLL, CUMF>(s, p);
			aa_write<S, ODD>(f, sq, base, o, s.f);
			if constexpr (OUT) {
				const double rho = (double) s.rho, vx = (double) s.vx, vy = (double) s.vy, vz = (double) s.vz;
				red[0] = rho;
				red[1] = rho * vx;
				red[2] = rho * vy;
				red[3] = rho * vz;
				red[4] = rho * (vx * vx + vy * vy + vz * vz);
				red[5] = isfinite(rho) ? 0.0 : 1.0;
			}
		}
		if constexpr (OUT) {
			// block sum in a fixed order, one partial per tile
#pragma unroll
			for (int k = 0; k < NRED; k++)
#pragma unroll
				for (int off = 16; off > 0; off >>= 1)
					red[k] += __shfl_down_sync(0xffffffffu, red[k], off);
			__shared__ double wsum[TPB / 32][NRED];
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			if (lane == 0)
#pragma unroll
				for (int k = 0; k < NRED; k++)
					wsum[warp][k] = red[k];
			__syncthreads();
			if (threadIdx.x < NRED) {
				double acc = 0;
#pragma unroll
				for (int w = 0; w < TPB / 32; w++)
					acc += wsum[w][threadIdx.x];
				partials[threadIdx.x * ntiles + t] = acc;
			}
			__syncthreads();
		}
	}
}

// One A-A step of every member, two x-adjacent sites per thread (grid policy
// 3): tiles of 256 sites, 128 threads, the per-pair code of aa_pair_kernel
// with the member's constants.  The grid walks the tile list with a stride
// of the grid size, so the blocks resident at one time work on neighbouring
// tiles and share the rows they touch through L2 (contiguous ranges per
// block ran 7 % slower on 64 members).  Every member's X is even, so a tile's pairs
// never straddle two rows.  OUT: per-tile FP64 partial sums as
// ens_step_kernel's.
template <typename S, int COLL, int CUMF, bool ODD, bool OUT, int MINB>
__global__ void __launch_bounds__(128, MINB)
	ens_pair_kernel(const EnsMember<typename S::T, float>* __restrict__ members, const int* __restrict__ tile_member,
					long long ntiles, double* __restrict__ partials)
{
	using T = typename S::T;
	__shared__ EnsMember<T, float> M;
	// byte offsets of the current member's 27 slot rows (pair_read_at reads
	// them from shared memory instead of multiplying per access)
	__shared__ PairSlots ps;
	constexpr int WORDS = (int) (sizeof(EnsMember<T, float>) / 4);
	static_assert(sizeof(EnsMember<T, float>) % 4 == 0 && WORDS <= 128, "member entry size");
	int cur = -1;
	for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
		const int m = tile_member[t];
		if (m != cur) {
			__syncthreads();
			if ((int) threadIdx.x < WORDS)
				reinterpret_cast<unsigned*>(&M)[threadIdx.x] = reinterpret_cast<const unsigned*>(members + m)[threadIdx.x];
			if (threadIdx.x < 27)
				ps.b[threadIdx.x] = (int) (threadIdx.x * members[m].sq * (long long) sizeof(T));
			__syncthreads();
			cur = m;
		}
		const unsigned i = (unsigned) ((t - M.tile0) * 256) + 2 * threadIdx.x;
		const bool act = i < (unsigned) M.n;
		Site<F2> s;
		PairAt at;
		if (act) {
			const unsigned row = fast_div(i, M.dx);
			const int x = (int) (i - row * (unsigned) M.X);
			const unsigned z = fast_div(row, M.dy);
			const int y = (int) (row - z * (unsigned) M.Y);
			at = pair_at_of(reinterpret_cast<char*>(M.f), sizeof(T), M.sy, M.sz, M.x0, M.X, M.Y, M.Z, x, y, (int) z, true, true);
			pair_read_at<S, ODD>(at, ps, s);
			density_velocity(s, M.p2);
		}
		__syncwarp();  // keeps the collision after the loads (fewer live registers)
		double red[NRED] = {0, 0, 0, 0, 0, 0};
		if (act) {
			if constexpr (OUT) {
#pragma unroll
				for (int l = 0; l < 2; l++) {
					const double rho = l ? s.rho.v.y : s.rho.v.x, vx = l ? s.vx.v.y : s.vx.v.x;
					const double vy = l ? s.vy.v.y : s.vy.v.x, vz = l ? s.vz.v.y : s.vz.v.x;
					red[0] += rho;
					red[1] += rho * vx;
					red[2] += rho * vy;
					red[3] += rho * vz;
					red[4] += rho * (vx * vx + vy * vy + vz * vz);
					red[5] += isfinite(rho) ? 0.0 : 1.0;
				}
			}
			collide<F2, COLL, CUMF>(s, M.p2);
			pair_write_at<S, ODD>(at, ps, s);
		}
		if constexpr (OUT) {
#pragma unroll
			for (int k = 0; k < NRED; k++)
#pragma unroll
				for (int off = 16; off > 0; off >>= 1)
					red[k] += __shfl_down_sync(0xffffffffu, red[k], off);
			__shared__ double wsum[4][NRED];
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			if (lane == 0)
#pragma unroll
				for (int k = 0; k < NRED; k++)
					wsum[warp][k] = red[k];
			__syncthreads();
			if (threadIdx.x < NRED)
				partials[threadIdx.x * ntiles + t] = ((wsum[0][threadIdx.x] + wsum[1][threadIdx.x]) + wsum[2][threadIdx.x])
												   + wsum[3][threadIdx.x];
			__syncthreads();
		}
	}
}

}  // namespace lbm
