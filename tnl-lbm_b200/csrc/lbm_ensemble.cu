// C-ABI of ensembles of periodic lattices (declared in include/tnl_lbm_b200.h,
// lbm_ensemble_*).
//
// All members live in one device allocation, each with the layout of a single
// lattice (ghost layer, 128-byte aligned rows).  The sites of every member are
// cut into tiles of `tile_sites` consecutive sites; a tile list maps each tile
// to its member, and the member table (ensemble.cuh) carries each member's
// geometry and collision constants.  One launch per A-A step covers every
// member; plain steps are replayed from CUDA graphs of GRAPH_STEPS steps.
//
// The reference has no counterpart: a TNL-LBM user advances one lattice per
// solver instance (State::SimUpdate, include/lbm3d/state.hpp:1297-1314).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tnl_lbm_b200.h"
#include "host_common.h"
#include "launch.h"

namespace lbm {
int record_error(int code, const char* msg);
PairStepFn pair_step_of(int storage);  // lbm_abi.cu
}

namespace {

int efail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int efail(int code, const char* fmt, ...)
{
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	return lbm::record_error(code, buf);
}

#define ENS_CUDA(call)                                                                                    \
	do {                                                                                                  \
		cudaError_t err_ = (call);                                                                        \
		if (err_ != cudaSuccess)                                                                          \
			return efail(LBM_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_), __FILE__, \
						 __LINE__);                                                                       \
	} while (0)

constexpr int NRED = lbm::NRED_HOST;

// per-member sums: block m adds the partials of tiles [tile0[m], tile0[m+1])
// in a fixed order into out[m * NRED + k]
__global__ void __launch_bounds__(256) ens_finish_kernel(const double* __restrict__ partials, long long ntiles,
														  const long long* __restrict__ tile0, double* __restrict__ out)
{
	__shared__ double sh[256];
	const int m = blockIdx.x;
	const long long b = tile0[m], e = tile0[m + 1];
	for (int k = 0; k < NRED; k++) {
		double v = 0;
		for (long long t = b + threadIdx.x; t < e; t += 256)
			v += partials[k * ntiles + t];
		sh[threadIdx.x] = v;
		__syncthreads();
		for (int s = 128; s > 0; s >>= 1) {
			if ((int) threadIdx.x < s)
				sh[threadIdx.x] += sh[threadIdx.x + s];
			__syncthreads();
		}
		if (threadIdx.x == 0)
			out[(long long) m * NRED + k] = sh[0];
		__syncthreads();
	}
}

}  // namespace

struct lbm_ensemble_t
{
	static constexpr int GRAPH_STEPS = 16;

	int count = 0;
	int storage = 0, collision = 0, cum_flags = 0, equilibrium = 0, device = 0, use_graphs = 1;
	const lbm::StorageOps* ops = nullptr;
	std::vector<lbm::Geometry> g;
	std::vector<lbm::CollParamsD> p;
	void* pops = nullptr;
	size_t pop_bytes = 0;
	cudaStream_t stream = nullptr;
	int tile_sites = 128;
	int grid_policy = 0;
	long long ntiles = 0;
	std::vector<long long> tile0;  // [count + 1]
	void* members_dev = nullptr;
	int* tile_member_dev = nullptr;
	long long* tile0_dev = nullptr;
	double* partials = nullptr;	 // [NRED][ntiles]
	double* sums_host = nullptr;	 // pinned [count][NRED]
	double* sums_mapped = nullptr;	 // device address of sums_host
	bool sums_valid = false;
	long long iteration = 0;
	cudaGraphExec_t graph = nullptr;
	// grid policy 2: one stream per lane, members round-robin over the lanes
	std::vector<cudaStream_t> lanes;
	std::vector<cudaEvent_t> joins;
	cudaEvent_t fork = nullptr;
	static constexpr int MAX_LANES = 64;

	void drop_graph()
	{
		if (graph) {
			cudaGraphExecDestroy(graph);
			graph = nullptr;
		}
	}
	void free_tiles()
	{
		cudaFree(members_dev);
		cudaFree(tile_member_dev);
		cudaFree(tile0_dev);
		cudaFree(partials);
		members_dev = nullptr;
		tile_member_dev = nullptr;
		tile0_dev = nullptr;
		partials = nullptr;
	}
};

namespace {

// grid policy 3 (persistent two-site kernel): FP32 arithmetic, every member
// of even width
bool ens_pair_ok(lbm_ensemble e)
{
	if (e->ops->compute_size != 4)
		return false;
	for (int m = 0; m < e->count; m++)
		if (e->g[m].X % 2 != 0)
			return false;
	return true;
}

int echeck(lbm_ensemble e)
{
	if (!e)
		return efail(LBM_ERR_INVALID, "null ensemble handle");
	if (cudaSetDevice(e->device) != cudaSuccess)
		return efail(LBM_ERR_CUDA, "cudaSetDevice(%d) failed", e->device);
	return LBM_OK;
}

// tile list, member table and partial-sum scratch for the current tile size
int build_tiles(lbm_ensemble e)
{
	e->drop_graph();
	e->free_tiles();
	const int tpb = e->tile_sites;
	e->tile0.assign(e->count + 1, 0);
	for (int m = 0; m < e->count; m++) {
		const long long n = (long long) e->g[m].X * e->g[m].Y * e->g[m].Z;
		e->tile0[m + 1] = e->tile0[m] + (n + tpb - 1) / tpb;
	}
	e->ntiles = e->tile0[e->count];
	std::vector<int> tile_member((size_t) e->ntiles);
	for (int m = 0; m < e->count; m++)
		for (long long t = e->tile0[m]; t < e->tile0[m + 1]; t++)
			tile_member[(size_t) t] = m;
	const size_t eb = e->ops->ens_entry_bytes;
	std::vector<unsigned char> table(eb * e->count);
	for (int m = 0; m < e->count; m++)
		e->ops->ens_entry(table.data() + eb * m, e->g[m], e->p[m], e->tile0[m]);
	ENS_CUDA(cudaMalloc(&e->members_dev, table.size()));
	ENS_CUDA(cudaMalloc(&e->tile_member_dev, sizeof(int) * tile_member.size()));
	ENS_CUDA(cudaMalloc(&e->tile0_dev, sizeof(long long) * e->tile0.size()));
	ENS_CUDA(cudaMalloc(&e->partials, sizeof(double) * NRED * e->ntiles));
	ENS_CUDA(cudaMemcpyAsync(e->members_dev, table.data(), table.size(), cudaMemcpyHostToDevice, e->stream));
	ENS_CUDA(cudaMemcpyAsync(e->tile_member_dev, tile_member.data(), sizeof(int) * tile_member.size(), cudaMemcpyHostToDevice,
							 e->stream));
	ENS_CUDA(cudaMemcpyAsync(e->tile0_dev, e->tile0.data(), sizeof(long long) * e->tile0.size(), cudaMemcpyHostToDevice,
							 e->stream));
	ENS_CUDA(cudaStreamSynchronize(e->stream));
	return LBM_OK;
}

int ensure_lanes(lbm_ensemble e)
{
	if (!e->lanes.empty())
		return LBM_OK;
	const int n = e->count < lbm_ensemble_t::MAX_LANES ? e->count : lbm_ensemble_t::MAX_LANES;
	ENS_CUDA(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
	for (int i = 0; i < n; i++) {
		cudaStream_t st = nullptr;
		cudaEvent_t ev = nullptr;
		ENS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
		e->lanes.push_back(st);
		ENS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
		e->joins.push_back(ev);
	}
	return LBM_OK;
}

// grid policy 2: every member runs the single-lattice step (the two-site
// kernel where it applies, else the direct kernel) on its lane; the lanes fork from and join into the ensemble's stream, so under
// graph capture the members become independent branches
int ens_launch_members(lbm_ensemble e)
{
	if (int rc = ensure_lanes(e))
		return rc;
	const int nl = (int) e->lanes.size();
	ENS_CUDA(cudaEventRecord(e->fork, e->stream));
	for (int i = 0; i < nl; i++)
		ENS_CUDA(cudaStreamWaitEvent(e->lanes[i], e->fork, 0));
	for (int m = 0; m < e->count; m++) {
		const lbm::Geometry& g = e->g[m];
		lbm::StepLaunch L{};
		L.g = g;
		L.p = e->p[m];
		L.coll = e->collision;
		L.cum_flags = e->cum_flags;
		L.odd = (e->iteration % 2) != 0;
		const int bx = g.X >= 128 ? 128 : ((g.X + 31) / 32) * 32;
		L.block = dim3(bx, 128 / bx, 1);
		L.grid = dim3((g.X + bx - 1) / bx, (g.Y + L.block.y - 1) / L.block.y, g.Z);
		L.stream = e->lanes[m % nl];
		L.kernel = lbm::KERNEL_DIRECT;
		// the two-site kernel where it applies (FP32 arithmetic, even X)
		cudaError_t err = cudaErrorNotSupported;
		if (const lbm::PairStepFn pair = lbm::pair_step_of(e->storage))
			err = pair(L);
		if (err == cudaErrorNotSupported)
			err = e->ops->step(L);
		if (err != cudaSuccess)
			return efail(LBM_ERR_CUDA, "member %d step launch failed: %s", m, cudaGetErrorString(err));
	}
	for (int i = 0; i < nl; i++) {
		ENS_CUDA(cudaEventRecord(e->joins[i], e->lanes[i]));
		ENS_CUDA(cudaStreamWaitEvent(e->stream, e->joins[i], 0));
	}
	return LBM_OK;
}

int ens_launch(lbm_ensemble e, bool sums, bool dry_run = false)
{
	if (e->grid_policy == 2 && !sums) {
		if (dry_run)
			return LBM_OK;
		if (int rc = ens_launch_members(e))
			return rc;
		e->iteration++;
		return LBM_OK;
	}
	lbm::EnsLaunch L{};
	L.members = e->members_dev;
	L.tile_member = e->tile_member_dev;
	L.ntiles = e->ntiles;
	L.tpb = e->tile_sites;
	L.pair = e->grid_policy == 3;
	L.grid = e->grid_policy == 1 ? e->ntiles : 0;
	L.partials = sums ? e->partials : nullptr;
	L.coll = e->collision;
	L.cum_flags = e->cum_flags;
	L.odd = (e->iteration % 2) != 0;
	L.stream = e->stream;
	L.dry_run = dry_run;
	const cudaError_t err = e->ops->ens_step(L);
	if (err != cudaSuccess)
		return efail(LBM_ERR_CUDA, "ensemble step launch failed: %s", cudaGetErrorString(err));
	if (!dry_run)
		e->iteration++;
	return LBM_OK;
}

int ens_build_graph(lbm_ensemble e)
{
	e->drop_graph();
	const long long saved = e->iteration;
	// resolve per-kernel launch facts outside of the capture
	for (int parity = 0; parity < 2; parity++) {
		e->iteration = parity;
		if (int rc = ens_launch(e, false, true)) {
			e->iteration = saved;
			return rc;
		}
	}
	e->iteration = 0;  // the graph starts at an even step
	cudaGraph_t graph = nullptr;
	ENS_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
	int rc = LBM_OK;
	for (int s = 0; s < lbm_ensemble_t::GRAPH_STEPS && rc == LBM_OK; s++)
		rc = ens_launch(e, false);
	const cudaError_t end = cudaStreamEndCapture(e->stream, &graph);
	e->iteration = saved;
	if (rc != LBM_OK) {
		if (graph)
			cudaGraphDestroy(graph);
		return rc;
	}
	if (end != cudaSuccess)
		return efail(LBM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(end));
	const cudaError_t inst = cudaGraphInstantiate(&e->graph, graph, 0);
	cudaGraphDestroy(graph);
	if (inst != cudaSuccess) {
		e->graph = nullptr;
		return efail(LBM_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(inst));
	}
	return LBM_OK;
}

int ens_plain_steps(lbm_ensemble e, long long n)
{
	while (n > 0 && (e->iteration % 2) != 0) {
		if (int rc = ens_launch(e, false))
			return rc;
		n--;
	}
	if (e->use_graphs && n >= lbm_ensemble_t::GRAPH_STEPS) {
		if (!e->graph)
			if (int rc = ens_build_graph(e))
				return rc;
		while (n >= lbm_ensemble_t::GRAPH_STEPS) {
			ENS_CUDA(cudaGraphLaunch(e->graph, e->stream));
			e->iteration += lbm_ensemble_t::GRAPH_STEPS;
			n -= lbm_ensemble_t::GRAPH_STEPS;
		}
	}
	while (n > 0) {
		if (int rc = ens_launch(e, false))
			return rc;
		n--;
	}
	return LBM_OK;
}

size_t dense_count(const lbm::Geometry& g, int layout)
{
	const long long gh = layout == LBM_LAYOUT_GHOST ? 2 : 0;
	return (size_t) 27 * (g.X + gh) * (g.Y + gh) * (g.Z + gh);
}

int ens_init(lbm_ensemble e, const lbm::InitSpec& spec)
{
	for (int m = 0; m < e->count; m++) {
		const cudaError_t err = e->ops->init_eq(e->g[m], spec, e->stream);
		if (err != cudaSuccess)
			return efail(LBM_ERR_CUDA, "init kernel failed: %s", cudaGetErrorString(err));
	}
	e->iteration = 0;
	e->sums_valid = false;
	ENS_CUDA(cudaStreamSynchronize(e->stream));
	return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_ensemble_create(const lbm_ensemble_desc* d, lbm_ensemble* out)
{
	if (!d || !out)
		return efail(LBM_ERR_INVALID, "null argument");
	*out = nullptr;
	if (d->count < 1 || d->count > LBM_ENSEMBLE_MAX_MEMBERS)
		return efail(LBM_ERR_INVALID, "member count %d outside 1 .. %d", d->count, LBM_ENSEMBLE_MAX_MEMBERS);
	if (!d->X || !d->Y || !d->Z || !d->viscosity)
		return efail(LBM_ERR_INVALID, "null size or viscosity array");
	if (d->storage < 0 || d->storage >= lbm::ST_COUNT)
		return efail(LBM_ERR_INVALID, "unknown storage %d", d->storage);
	if (d->collision < LBM_COLL_CUM || d->collision > LBM_COLL_MRT)
		return efail(LBM_ERR_INVALID, "unknown collision %d", d->collision);
	if (d->collision == LBM_COLL_CUM && d->cum_flags != 0 && d->cum_flags != LBM_CUM_ANTIALIAS
		&& d->cum_flags != (LBM_CUM_GEIER_2017 | LBM_CUM_ANTIALIAS))
		return efail(LBM_ERR_UNSUPPORTED, "cumulant flags %d: the 2017 variant requires the anti-aliasing terms", d->cum_flags);
	if (d->equilibrium != LBM_EQ_SECOND_ORDER && d->equilibrium != LBM_EQ_INV_CUM)
		return efail(LBM_ERR_INVALID, "unknown equilibrium %d", d->equilibrium);
	for (int m = 0; m < d->count; m++) {
		if (d->X[m] < 1 || d->Y[m] < 1 || d->Z[m] < 1)
			return efail(LBM_ERR_INVALID, "member %d: sizes must be positive", m);
		if ((long long) d->X[m] * d->Y[m] * d->Z[m] >= (1ll << 31) || d->X[m] > 65535 * 4 || d->Y[m] > 65535
			|| d->Z[m] > 65535)
			return efail(LBM_ERR_SIZE, "member %d: %d x %d x %d sites exceed the member limit (2^31 sites)", m, d->X[m],
						 d->Y[m], d->Z[m]);
		if (!(d->viscosity[m] > 0.0) || !std::isfinite(d->viscosity[m]))
			return efail(LBM_ERR_INVALID, "member %d: viscosity must be positive and finite", m);
	}
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
		return efail(LBM_ERR_CUDA, "no CUDA device available");
	if (d->device < 0 || d->device >= ndev)
		return efail(LBM_ERR_INVALID, "device %d out of range", d->device);
	ENS_CUDA(cudaSetDevice(d->device));

	lbm_ensemble e = new lbm_ensemble_t();
	e->count = d->count;
	e->storage = d->storage;
	e->collision = d->collision;
	e->cum_flags = d->cum_flags;
	e->equilibrium = d->equilibrium;
	e->device = d->device;
	e->use_graphs = d->use_graphs;
	e->ops = &lbm::storage_ops(d->storage);
	const int es = e->ops->elem_size;
	e->g.resize(e->count);
	e->p.resize(e->count);
	std::vector<size_t> offset(e->count);
	size_t total = 0;
	for (int m = 0; m < e->count; m++) {
		e->g[m] = lbm::make_geometry(d->X[m], d->Y[m], d->Z[m], es);
		offset[m] = total;
		total += (lbm::geometry_elems(e->g[m]) * es + 255) / 256 * 256;
		lbm::CollParamsD& p = e->p[m];
		p = lbm::CollParamsD{};
		lbm::cumulant_rates(d->viscosity[m], p);
		p.nu = d->viscosity[m];
		p.eq = d->equilibrium;
	}
	e->pop_bytes = total;
	auto cleanup = [&](int rc) {
		lbm_ensemble_destroy(e);
		return rc;
	};
	if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
		return cleanup(efail(LBM_ERR_CUDA, "stream creation failed"));
	cudaError_t err = cudaMalloc(&e->pops, total);
	if (err != cudaSuccess)
		return cleanup(efail(LBM_ERR_CUDA, "population allocation of %zu bytes failed: %s", total, cudaGetErrorString(err)));
	if (cudaMemsetAsync(e->pops, 0, total, e->stream) != cudaSuccess)
		return cleanup(efail(LBM_ERR_CUDA, "population memset failed"));
	for (int m = 0; m < e->count; m++)
		e->g[m].f = (char*) e->pops + offset[m];
	if (cudaHostAlloc(&e->sums_host, sizeof(double) * NRED * e->count, cudaHostAllocMapped) != cudaSuccess
		|| cudaHostGetDevicePointer((void**) &e->sums_mapped, e->sums_host, 0) != cudaSuccess)
		return cleanup(efail(LBM_ERR_CUDA, "reduction buffers allocation failed"));
	if (int rc = build_tiles(e))
		return cleanup(rc);
	*out = e;
	return LBM_OK;
}

int lbm_ensemble_destroy(lbm_ensemble e)
{
	if (!e)
		return LBM_OK;
	cudaSetDevice(e->device);
	if (e->stream)
		cudaStreamSynchronize(e->stream);
	e->drop_graph();
	e->free_tiles();
	cudaFree(e->pops);
	cudaFreeHost(e->sums_host);
	for (cudaStream_t st : e->lanes)
		cudaStreamDestroy(st);
	for (cudaEvent_t ev : e->joins)
		cudaEventDestroy(ev);
	if (e->fork)
		cudaEventDestroy(e->fork);
	if (e->stream)
		cudaStreamDestroy(e->stream);
	delete e;
	return LBM_OK;
}

int lbm_ensemble_init_taylor_green(lbm_ensemble e, double u0, double rho0)
{
	if (int rc = echeck(e))
		return rc;
	lbm::InitSpec spec{};
	spec.mode = 2;
	spec.eq = e->equilibrium;
	spec.rho0 = rho0;
	spec.u0 = u0;
	return ens_init(e, spec);
}

int lbm_ensemble_init_equilibrium(lbm_ensemble e, double rho0, double vx0, double vy0, double vz0)
{
	if (int rc = echeck(e))
		return rc;
	lbm::InitSpec spec{};
	spec.mode = 0;
	spec.eq = e->equilibrium;
	spec.rho0 = rho0;
	spec.vx0 = vx0;
	spec.vy0 = vy0;
	spec.vz0 = vz0;
	return ens_init(e, spec);
}

int lbm_ensemble_set_populations(lbm_ensemble e, int member, const void* host, int layout, int dtype)
{
	if (int rc = echeck(e))
		return rc;
	if (member < 0 || member >= e->count)
		return efail(LBM_ERR_INVALID, "member %d out of range", member);
	if (!host || (layout != 0 && layout != 1) || (dtype != 0 && dtype != 1))
		return efail(LBM_ERR_INVALID, "bad arguments");
	const size_t bytes = dense_count(e->g[member], layout) * (dtype == 0 ? 8 : 4);
	void* dev = nullptr;
	ENS_CUDA(cudaMallocAsync(&dev, bytes, e->stream));
	ENS_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, e->stream));
	const cudaError_t err = e->ops->unpack(e->g[member], dev, dtype, layout, e->stream);
	cudaFreeAsync(dev, e->stream);
	if (err != cudaSuccess)
		return efail(LBM_ERR_CUDA, "unpack failed: %s", cudaGetErrorString(err));
	e->sums_valid = false;
	ENS_CUDA(cudaStreamSynchronize(e->stream));
	return LBM_OK;
}

int lbm_ensemble_get_populations(lbm_ensemble e, int member, void* host, int layout, int dtype)
{
	if (int rc = echeck(e))
		return rc;
	if (member < 0 || member >= e->count)
		return efail(LBM_ERR_INVALID, "member %d out of range", member);
	if (!host || (layout != 0 && layout != 1) || (dtype != 0 && dtype != 1))
		return efail(LBM_ERR_INVALID, "bad arguments");
	const size_t bytes = dense_count(e->g[member], layout) * (dtype == 0 ? 8 : 4);
	void* dev = nullptr;
	ENS_CUDA(cudaMallocAsync(&dev, bytes, e->stream));
	const cudaError_t err = e->ops->pack(e->g[member], dev, dtype, layout, e->stream);
	if (err != cudaSuccess) {
		cudaFreeAsync(dev, e->stream);
		return efail(LBM_ERR_CUDA, "pack failed: %s", cudaGetErrorString(err));
	}
	ENS_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, e->stream));
	cudaFreeAsync(dev, e->stream);
	ENS_CUDA(cudaStreamSynchronize(e->stream));
	return LBM_OK;
}

int lbm_ensemble_step(lbm_ensemble e, int64_t nsteps, int flags)
{
	if (int rc = echeck(e))
		return rc;
	if (nsteps < 0 || (nsteps == 0 && flags))
		return efail(LBM_ERR_INVALID, "nsteps must be positive when flags are given");
	if (flags & ~LBM_STEP_SUMS)
		return efail(LBM_ERR_UNSUPPORTED, "ensembles provide LBM_STEP_SUMS only");
	if (nsteps == 0)
		return LBM_OK;
	const bool sums = (flags & LBM_STEP_SUMS) != 0;
	if (int rc = ens_plain_steps(e, nsteps - (sums ? 1 : 0)))
		return rc;
	e->sums_valid = false;
	if (sums) {
		if (int rc = ens_launch(e, true))
			return rc;
		// written straight into the mapped pinned buffer
		ens_finish_kernel<<<e->count, 256, 0, e->stream>>>(e->partials, e->ntiles, e->tile0_dev, e->sums_mapped);
		ENS_CUDA(cudaGetLastError());
		e->sums_valid = true;
	}
	return LBM_OK;
}

int lbm_ensemble_get_sums(lbm_ensemble e, double* out)
{
	if (int rc = echeck(e))
		return rc;
	if (!out)
		return efail(LBM_ERR_INVALID, "null output");
	if (!e->sums_valid)
		return efail(LBM_ERR_INVALID, "no sums: call lbm_ensemble_step with LBM_STEP_SUMS first");
	ENS_CUDA(cudaStreamSynchronize(e->stream));
	memcpy(out, e->sums_host, sizeof(double) * NRED * e->count);
	return LBM_OK;
}

int64_t lbm_ensemble_iteration(lbm_ensemble e)
{
	return e ? e->iteration : -1;
}

int lbm_ensemble_get_stream(lbm_ensemble e, void** stream)
{
	if (!e || !stream)
		return efail(LBM_ERR_INVALID, "null argument");
	*stream = (void*) e->stream;
	return LBM_OK;
}

int lbm_ensemble_synchronize(lbm_ensemble e)
{
	if (int rc = echeck(e))
		return rc;
	ENS_CUDA(cudaStreamSynchronize(e->stream));
	ENS_CUDA(cudaGetLastError());
	return LBM_OK;
}

int lbm_ensemble_set_shape(lbm_ensemble e, int tile_sites, int grid_policy)
{
	if (int rc = echeck(e))
		return rc;
	if ((tile_sites != 128 && tile_sites != 256) || grid_policy < 0 || grid_policy > 3)
		return efail(LBM_ERR_INVALID, "launch shape: tile_sites 128 or 256, grid_policy 0, 1, 2 or 3");
	if (grid_policy == 3 && (tile_sites != 256 || !ens_pair_ok(e)))
		return efail(LBM_ERR_UNSUPPORTED,
					 "grid policy 3 (two-site kernel) needs tile_sites 256, FP32 arithmetic and members of even width");
	if (tile_sites != e->tile_sites) {
		ENS_CUDA(cudaStreamSynchronize(e->stream));
		e->tile_sites = tile_sites;
		e->sums_valid = false;
		if (int rc = build_tiles(e))
			return rc;
	}
	e->grid_policy = grid_policy;
	e->drop_graph();
	return LBM_OK;
}

int lbm_ensemble_get_shape(lbm_ensemble e, int* tile_sites, int* grid_policy)
{
	if (!e || !tile_sites || !grid_policy)
		return efail(LBM_ERR_INVALID, "null argument");
	*tile_sites = e->tile_sites;
	*grid_policy = e->grid_policy;
	return LBM_OK;
}

int lbm_ensemble_autotune(lbm_ensemble e, int ntrials)
{
	if (int rc = echeck(e))
		return rc;
	if (ntrials < 1)
		return efail(LBM_ERR_INVALID, "ntrials must be positive");
	void* backup = nullptr;
	ENS_CUDA(cudaMalloc(&backup, e->pop_bytes));
	ENS_CUDA(cudaMemcpyAsync(backup, e->pops, e->pop_bytes, cudaMemcpyDeviceToDevice, e->stream));
	const long long it0 = e->iteration;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	float best = 1e30f;
	int best_tile = e->tile_sites, best_grid = e->grid_policy;
	int rc = LBM_OK;
	// every candidate timed the way plain steps run: graph replays when graphs
	// are on (the first replay builds and warms the graph)
	const long long chunk = e->use_graphs ? lbm_ensemble_t::GRAPH_STEPS : 2;
	for (int tile : {128, 256}) {
		for (int gp : {0, 1, 2, 3}) {
			if (gp == 2 && tile != 128)
				continue;  // the tile size does not apply to per-member launches
			if (gp == 3 && (tile != 256 || !ens_pair_ok(e)))
				continue;
			if ((rc = lbm_ensemble_set_shape(e, tile, gp)))
				break;
			e->iteration = it0 + (it0 % 2);	 // timed steps start at an even step
			rc = ens_plain_steps(e, chunk);
			cudaEventRecord(e0, e->stream);
			if (rc == LBM_OK)
				rc = ens_plain_steps(e, chunk * ntrials);
			cudaEventRecord(e1, e->stream);
			cudaEventSynchronize(e1);
			float ms = 0;
			cudaEventElapsedTime(&ms, e0, e1);
			if (rc == LBM_OK && ms < best) {
				best = ms;
				best_tile = tile;
				best_grid = gp;
			}
		}
		if (rc)
			break;
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	e->iteration = it0;
	cudaMemcpyAsync(e->pops, backup, e->pop_bytes, cudaMemcpyDeviceToDevice, e->stream);
	cudaStreamSynchronize(e->stream);
	cudaFree(backup);
	if (rc)
		return rc;
	const cudaError_t err = cudaGetLastError();
	if (err != cudaSuccess)
		return efail(LBM_ERR_CUDA, "ensemble autotune failed: %s", cudaGetErrorString(err));
	e->sums_valid = false;
	return lbm_ensemble_set_shape(e, best_tile, best_grid);
}

}  // extern "C"
