// Persistent, warp-specialised A-A step kernel for sm_100a.
//
// Each CTA has TX threads, one lattice site per thread, and walks over row
// tiles (TX consecutive sites of one (y, z) row) in a grid-stride loop.  For
// every tile, lanes 0..26 of warp 0 issue 27 bulk copies (cp.async.bulk, one
// per population direction) of the rows the tile's A-A read needs into a
// STAGES-deep shared-memory ring, signalled by mbarrier transaction counts; a
// stage is refilled as soon as all warps have released it.  All threads read
// their 27 values from shared memory, apply boundary conditions and the
// collision, and store to HBM with ordinary coalesced stores.  No warp is set
// aside as a producer, so every register of the CTA does site work.  The number of bytes in flight per SM is set by
// the ring depth, not by the registers a thread can spare for loads.
//
// Odd step: direction q of the site at x comes from slot opp(q) of the site
// x - c_q.  Its row is (y - c_qy, z - c_qz); its x range is shifted by -c_qx,
// which is not a 16-byte aligned start, so the copy takes an aligned window
// [xs - A, xs + n + A) with A = 16 bytes / element and the consumer indexes it
// at A - c_qx + tid.  Even step: the site's own 27 slots, an aligned window
// [xs, xs + n).
//
// Every location a tile reads belongs to one of its own sites (A-A ownership),
// so no other CTA writes it during the step; the A-element margins of an odd
// window may be written concurrently by the neighbouring tiles, and are never
// used.  Sites whose neighbours wrap around a periodic face cannot take their
// values from the window; they re-read the affected populations directly from
// HBM (aa_read), which is the same read the direct kernel does.
//
// Waits on mbarriers are bounded; a timeout sets LBM_STATUS_TIMEOUT in the
// device status word, stops the tile loop and still drains the copies this
// CTA has issued before it exits.  The tile loop's waits take their bound
// from the launch (wait_limit tries, WAIT_LIMIT by default), so that a test
// can make them run out while copies are in flight; the drain always waits
// with the full bound, so no copy lands after the CTA has exited.
#pragma once

#include "aa_kernels.cuh"

namespace lbm {

constexpr int STATUS_TIMEOUT = 1;
// iterations of mbarrier.try_wait before giving up (each try waits for a
// hardware-defined interval, so this bounds a wait to seconds)
constexpr long long WAIT_LIMIT = 1ll << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
	return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(ok)
		: "r"(smem_u32(bar)), "r"(parity)
		: "memory");
	return ok != 0;
}

// bounded wait on one phase of an mbarrier (at most `limit` tries); false on
// timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = WAIT_LIMIT)
{
	for (long long i = 0; i < limit; i++)
		if (mbar_try_wait(bar, parity))
			return true;
	return false;
}

// bulk copy global -> shared completing on an mbarrier (no multicast)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
				 "l"(src), "r"(bytes), "r"(smem_u32(bar))
				 : "memory");
}

// Tile t of the grid-stride walk, decomposed as t = (z*Y + y)*tiles_x + xt.
// Consecutive tiles of one CTA differ by gridDim.x, so the cursor is advanced
// with additions and at most two carries instead of 64-bit divisions.
struct TileCursor
{
	int xt, y, z;
};

struct TileStride
{
	int dxt, dy, dz;
};

__device__ __forceinline__ TileCursor tile_at(long long t, int tiles_x, int Y)
{
	TileCursor c;
	c.xt = (int) (t % tiles_x);
	const long long row = t / tiles_x;
	c.y = (int) (row % Y);
	c.z = (int) (row / Y);
	return c;
}

__device__ __forceinline__ TileStride tile_stride(long long g, int tiles_x, int Y)
{
	const TileCursor c = tile_at(g, tiles_x, Y);
	return TileStride{c.xt, c.y, c.z};
}

__device__ __forceinline__ void tile_advance(TileCursor& c, const TileStride& d, int tiles_x, int Y)
{
	c.xt += d.dxt;
	int carry = 0;
	if (c.xt >= tiles_x) {
		c.xt -= tiles_x;
		carry = 1;
	}
	c.y += d.dy + carry;
	carry = 0;
	if (c.y >= Y) {
		c.y -= Y;
		carry = 1;
	}
	c.z += d.dz + carry;
}

template <typename T, int TX, bool ODD>
struct TileShape
{
	static constexpr int A = 16 / (int) sizeof(T);	 // elements per 16 bytes
	static constexpr int W = ODD ? TX + 2 * A : TX;	 // window width in elements
	static constexpr int ROW_BYTES = W * (int) sizeof(T);
	static constexpr int MAP_BYTES = TX + 32;		 // map row of the tile, from a 16-byte aligned start
	static constexpr int STAGE_BYTES = 27 * ROW_BYTES + MAP_BYTES;
};

template <typename T, int TX, bool ODD, int STAGES>
constexpr int tile_smem_bytes()
{
	return STAGES * TileShape<T, TX, ODD>::STAGE_BYTES + 2 * STAGES * 8;
}

// Issue the 27 bulk copies of one tile into stage s (called by warp 0; lane q
// copies the window of slot q).
template <typename S, bool ODD, bool GENERAL, int TX, int STAGES>
__device__ __forceinline__ void issue_tile(const StepArgs<typename S::T, typename S::R>& a, typename S::T* ring,
										   uint64_t* full, int s, const TileCursor& c, int lane)
{
	using T = typename S::T;
	using Shape = TileShape<T, TX, ODD>;
	constexpr int A = Shape::A;
	constexpr int W = Shape::W;
	const int y = c.y, z = c.z;
	const int xs = c.xt * TX;
	const int n = min(TX, a.X - xs);
	const int n_al = (n + A - 1) / A * A;
	const uint32_t bytes = (uint32_t) ((ODD ? n_al + 2 * A : n_al) * (int) sizeof(T));
	// periodic lattice, odd step: the x neighbours of the row's first and last
	// sites wrap around.  When X is a multiple of A, the 16-byte margins of the
	// window come from the other end of the row instead of the ghost columns;
	// the main copy then leaves those margins out, so no two copies of a stage
	// write the same bytes.
	const bool wrap_margins = ODD && !GENERAL && (a.X % A) == 0;
	const bool left = wrap_margins && xs == 0;
	const bool right = wrap_margins && xs + n == a.X;
	const int lo = left ? A : 0;
	const int hi = right ? A + n_al : n_al + 2 * A;
	// map row of the tile (general kernels): 16-byte aligned source window
	uint32_t map_bytes = 0;
	long long map_src = 0;
	if (GENERAL) {
		const long long m0 = ((long long) z * a.Y + y) * a.X + xs;
		map_src = m0 & ~15ll;
		map_bytes = (uint32_t) ((m0 - map_src + n + 15) & ~15ll);
	}
	if (lane == 0)
		mbar_arrive_expect_tx(&full[s], 27 * bytes + map_bytes);
	__syncwarp();
	unsigned char* stage = reinterpret_cast<unsigned char*>(ring) + (long long) s * Shape::STAGE_BYTES;
	T* win = reinterpret_cast<T*>(stage);
	if (lane < 27) {
		const int q = lane;
		if (ODD) {
			// slot q of the sites x + c_q: read there by site x as direction opp(q)
			int yy = y + cy_rt(q), zz = z + cz_rt(q);
			if (!GENERAL) {
				yy = yy < 0 ? a.Y - 1 : (yy >= a.Y ? 0 : yy);
				zz = zz < 0 ? a.Z - 1 : (zz >= a.Z ? 0 : zz);
			}
			const long long row = (long long) q * a.sq + (long long) (zz + 1) * a.sz + (long long) (yy + 1) * a.sy + a.x0;
			// window element j holds site xs - A + j
			bulk_g2s(win + q * W + lo, a.f + row + xs - A + lo, (uint32_t) ((hi - lo) * (int) sizeof(T)), &full[s]);
			if (left)  // window [0, A) <- sites [X - A, X)
				bulk_g2s(win + q * W, a.f + row + a.X - A, 16u, &full[s]);
			if (right)	// window [A + n, 2A + n) <- sites [0, A)
				bulk_g2s(win + q * W + A + n_al, a.f + row, 16u, &full[s]);
		}
		else {
			const long long src = (long long) q * a.sq + (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + xs;
			bulk_g2s(win + q * W, a.f + src, bytes, &full[s]);
		}
	}
	else if (GENERAL && lane == 27) {
		bulk_g2s(stage + 27 * Shape::ROW_BYTES, a.map + map_src, map_bytes, &full[s]);
	}
}

template <typename S, int COLL, int CUMF, bool ODD, bool GENERAL, int TX, int STAGES>
__global__ void __launch_bounds__(TX, LBM_TILE_MINB)
	aa_tile_kernel(const StepArgs<typename S::T, typename S::R> a, int* status, long long ntiles, int tiles_x,
				   long long wait_limit)
{
	using R = typename S::R;
	using T = typename S::T;
	using Shape = TileShape<T, TX, ODD>;
	constexpr int A = Shape::A;
	constexpr int W = Shape::W;
	constexpr int WARPS = TX / 32;

	extern __shared__ __align__(128) unsigned char smem_raw[];
	T* ring = reinterpret_cast<T*>(smem_raw);
	uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + STAGES * Shape::STAGE_BYTES);
	uint64_t* empty = full + STAGES;

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const bool warp0 = tid < 32;

	if (tid == 0) {
		for (int s = 0; s < STAGES; s++) {
			mbar_init(&full[s], 1);
			mbar_init(&empty[s], WARPS);
		}
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();

	const long long my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
	double red[NRED] = {0, 0, 0, 0, 0, 0};
	bool timed_out = false;
	long long issued = 0;
	const TileStride stride = tile_stride(gridDim.x, tiles_x, a.Y);
	TileCursor cur = tile_at(blockIdx.x, tiles_x, a.Y);	  // tile consumed in iteration i
	TileCursor pre = cur;									  // next tile warp 0 copies

	// prologue: warp 0 fills the ring
	if (warp0) {
		for (long long i = 0; i < STAGES && i < my_tiles; i++) {
			issue_tile<S, ODD, GENERAL, TX, STAGES>(a, ring, full, (int) i, pre, lane);
			tile_advance(pre, stride, tiles_x, a.Y);
		}
		issued = my_tiles < STAGES ? my_tiles : STAGES;
	}

	int s = 0;
	uint32_t phase = 0;
	for (long long i = 0; i < my_tiles; i++) {
		if (i > 0) {
			tile_advance(cur, stride, tiles_x, a.Y);
			if (++s == STAGES) {
				s = 0;
				phase ^= 1u;
			}
		}
		if (!mbar_wait(&full[s], phase, wait_limit)) {
			timed_out = true;
			break;
		}
		const int y = cur.y;
		const int z = cur.z;
		const int x = cur.xt * TX + tid;
		const bool active = x < a.X;
		const unsigned char* stage = reinterpret_cast<const unsigned char*>(ring) + (long long) s * Shape::STAGE_BYTES;
		const T* st = reinterpret_cast<const T*>(stage);
		uint8_t geo = GEO_PERIODIC;
		if constexpr (GENERAL) {
			const long long m0 = ((long long) z * a.Y + y) * a.X + cur.xt * TX;
			if (active)
				geo = stage[27 * Shape::ROW_BYTES + (int) (m0 & 15) + tid];
		}

		Site<R> site;
		// slot q's window holds direction opp(q) of the tile's sites (odd step)
		// or direction q (even step)
		if (active) {
			static_for<27>(
				[&](auto Qc)
				{
					constexpr int q = decltype(Qc)::value;
					if constexpr (ODD)
						site.f[q] = S::template load_smem<opp(q)>(st + opp(q) * W + A - cx(q) + tid);
					else
						site.f[q] = S::template load_smem<q>(st + q * W + tid);
				}
			);
		}
		__syncwarp();
		if (lane == 0)
			mbar_arrive(&empty[s]);
		// warp 0 refills stage s with tile i + STAGES once every warp has read it
		if (warp0 && i + STAGES < my_tiles) {
			bool ok = true;
			if (lane == 0)
				ok = mbar_wait(&empty[s], phase, wait_limit);
			ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
			if (!ok) {
				timed_out = true;
				break;
			}
			issue_tile<S, ODD, GENERAL, TX, STAGES>(a, ring, full, s, pre, lane);
			tile_advance(pre, stride, tiles_x, a.Y);
			issued = i + STAGES + 1;
		}
		if (!active)
			continue;

		const long long base = (long long) (z + 1) * a.sz + (long long) (y + 1) * a.sy + a.x0 + x;
		const long long sidx = ((long long) z * a.Y + y) * a.X + x;
		const bool wrap = !GENERAL || geo == GEO_PERIODIC;
		const Offsets o = neighbour_offsets(wrap, wrap && a.zwrap, x, y, z, a.X, a.Y, a.Z, a.sy, a.sz);
		if constexpr (ODD) {
			// sites on a periodic face: the wrapped neighbours are not in the window
			bool face;
			if constexpr (GENERAL)
				face = wrap && (x == 0 || x == a.X - 1 || y == 0 || y == a.Y - 1 || z == 0 || z == a.Z - 1);
			else
				face = (a.X % A) != 0 && (x == 0 || x == a.X - 1);
			if (face)
				aa_read<S, true>(a.f, a.sq, base, o, site.f);
		}
		bool store = true, coll = true;
		if constexpr (GENERAL) {
			if (geo == GEO_NOTHING) {
				site.rho = R(1);
				site.vx = site.vy = site.vz = R(0);
				store = false;
				coll = false;
			}
			else {
				coll = apply_boundary(site, geo, a, z, y);
			}
		}
		else {
			density_velocity(site, a.p);
		}
		if (coll)
			collide<R, COLL, CUMF>(site, a.p);
		if (store)
			aa_write<S, ODD>(a.f, a.sq, base, o, site.f);
		if (a.macro) {
			const long long nsites = (long long) a.X * a.Y * a.Z;
			a.macro[sidx] = site.rho;
			a.macro[nsites + sidx] = site.vx;
			a.macro[2 * nsites + sidx] = site.vy;
			a.macro[3 * nsites + sidx] = site.vz;
		}
		if (a.partials) {
			const double rho = (double) site.rho, vx = (double) site.vx, vy = (double) site.vy, vz = (double) site.vz;
			red[0] += rho;
			red[1] += rho * vx;
			red[2] += rho * vy;
			red[3] += rho * vz;
			red[4] += rho * (vx * vx + vy * vy + vz * vz);
			red[5] += isfinite(rho) ? 0.0 : 1.0;
		}
	}
	if (timed_out && lane == 0)
		atomicOr(status, STATUS_TIMEOUT);
	// drain: no copy issued by this CTA may land after it exits (only reachable
	// with copies outstanding after a timeout)
	if (warp0 && lane == 0) {
		const long long first = issued > STAGES ? issued - STAGES : 0;
		for (long long i = first; i < issued; i++)
			mbar_wait(&full[(int) (i % STAGES)], (uint32_t) ((i / STAGES) & 1));
	}
	if (a.partials)
		block_reduce_store<R>(red, a.partials);
}

}  // namespace lbm
