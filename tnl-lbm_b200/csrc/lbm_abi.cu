// C-ABI of the B200 hot path (declared in include/tnl_lbm_b200.h).
//
// Owns the device state of one lattice (populations with ghost layer, map,
// inflow profiles, macro field, reduction scratch), computes the per-viscosity
// collision constants once on the host, and drives the even/odd A-A kernels
// from a host loop or from captured CUDA graphs.  Mirrors the host side of the
// reference's time step: LBM::updateKernelData (include/lbm3d/lbm.hpp:307-323)
// and State::SimUpdate (include/lbm3d/state.hpp:1235-1314).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tnl_lbm_b200.h"
#include "d3q27.cuh"
#include "host_common.h"
#include "lattice.h"
#include "launch.h"

namespace lbm {
const StorageOps& storage_ops_f64();
const StorageOps& storage_ops_f32();
const StorageOps& storage_ops_f32s();
const StorageOps& storage_ops_f16s();
const StorageOps& storage_ops_bf16s();
const StorageOps& storage_ops_f16sr();
const StorageOps& storage_ops_bf16sr();
const StorageOps& storage_ops_i16s();

const StorageOps& storage_ops(int storage)
{
	switch (storage) {
		case ST_F64:
			return storage_ops_f64();
		case ST_F32:
			return storage_ops_f32();
		case ST_F32S:
			return storage_ops_f32s();
		case ST_F16S:
			return storage_ops_f16s();
		case ST_F16SR:
			return storage_ops_f16sr();
		case ST_BF16SR:
			return storage_ops_bf16sr();
		case ST_I16S:
			return storage_ops_i16s();
		default:
			return storage_ops_bf16s();
	}
}

// the two-site step of a storage, or null (FP64 arithmetic)
PairStepFn pair_step_of(int storage)
{
	switch (storage) {
		case ST_F32:
			return pair_step_f32;
		case ST_F32S:
			return pair_step_f32s;
		case ST_F16S:
			return pair_step_f16s;
		case ST_F16SR:
			return pair_step_f16sr;
		case ST_BF16S:
			return pair_step_bf16s;
		case ST_BF16SR:
			return pair_step_bf16sr;
		case ST_I16S:
			return pair_step_i16s;
		default:
			return nullptr;
	}
}
}  // namespace lbm

namespace {

thread_local std::string g_error = "no error";

int fail(int code, const char* fmt, ...)
{
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	g_error = buf;
	return code;
}

#define LBM_CUDA(call)                                                                                   \
	do {                                                                                                 \
		cudaError_t err_ = (call);                                                                       \
		if (err_ != cudaSuccess)                                                                         \
			return fail(LBM_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_), __FILE__, \
						__LINE__);                                                                       \
	} while (0)

bool site_type_supported(uint8_t g)
{
	switch (g) {
		case lbm::GEO_FLUID:
		case lbm::GEO_WALL:
		case lbm::GEO_INFLOW:
		case lbm::GEO_INFLOW_LEFT:
		case lbm::GEO_INFLOW_EQ_LEFT:
		case lbm::GEO_OUTFLOW_EQ:
		case lbm::GEO_PERIODIC:
		case lbm::GEO_NOTHING:
		case lbm::GEO_SYM_TOP:
		case lbm::GEO_SYM_BOTTOM:
		case lbm::GEO_SYM_LEFT:
		case lbm::GEO_SYM_RIGHT:
		case lbm::GEO_SYM_BACK:
		case lbm::GEO_SYM_FRONT:
			return true;
		default:
			return false;
	}
}

// collision plugins registered by lbm_register_collision, by id - LBM_COLL_PLUGIN_FIRST
struct CollisionPlugin
{
	lbm_collision_launcher launch = nullptr;
	std::string name;
};
std::mutex g_plugins_mutex;
CollisionPlugin g_plugins[LBM_COLL_PLUGIN_LAST - LBM_COLL_PLUGIN_FIRST + 1];

bool plugin_id(int id)
{
	return id >= LBM_COLL_PLUGIN_FIRST && id <= LBM_COLL_PLUGIN_LAST;
}

}  // namespace

namespace lbm {
// lets other translation units of the library set the message of lbm_last_error()
int record_error(int code, const char* msg)
{
	return fail(code, "%s", msg);
}
}  // namespace lbm


namespace {

int check(lbm_handle h)
{
	if (!h)
		return fail(LBM_ERR_INVALID, "null handle");
	if (cudaSetDevice(h->d.device) != cudaSuccess)
		return fail(LBM_ERR_CUDA, "cudaSetDevice(%d) failed", h->d.device);
	return LBM_OK;
}

// one slot of partial sums: [NRED][blocks] partials and the finish scratch
size_t partials_slot_doubles(long long blocks)
{
	return (size_t) blocks * lbm::NRED_HOST + lbm::finish_scratch_doubles();
}
// slot s of the partial sums
double* partials_of(lbm_handle h, int s)
{
	return h->partials + (size_t) s * partials_slot_doubles(h->partials_cap);
}
int ensure_partials(lbm_handle h, long long blocks)
{
	if (blocks <= h->partials_cap)
		return LBM_OK;
	if (h->partials) {
		// a finish kernel may still read the old slots
		LBM_CUDA(cudaStreamSynchronize(h->finish_stream));
		cudaFree(h->partials);
	}
	h->partials = nullptr;
	h->partials_cap = 0;
	LBM_CUDA(cudaMalloc(&h->partials, 2 * partials_slot_doubles(blocks) * sizeof(double)));
	h->partials_cap = blocks;
	return LBM_OK;
}

int ensure_macro(lbm_handle h)
{
	if (h->macro)
		return LBM_OK;
	LBM_CUDA(cudaMalloc(&h->macro, (size_t) 4 * h->sites() * h->ops->compute_size));
	return LBM_OK;
}

int launch_step(lbm_handle h, bool macro, bool sums, bool dry_run = false)
{
	lbm::StepLaunch L{};
	L.g = h->g;
	L.map = h->d.periodic ? nullptr : h->map;
	for (int k = 0; k < 3; k++)
		L.inflow[k] = h->inflow[k];
	L.macro = macro ? h->macro : nullptr;
	// the slot of the sums ring this step fills; the finish kernel that last
	// read the slot (two observation steps ago) must be done with it
	const int sums_slot = h->sums_last ^ 1;
	L.partials = sums ? partials_of(h, sums_slot) : nullptr;
	if (sums && !dry_run)
		LBM_CUDA(cudaStreamWaitEvent(h->stream, h->sums_ev[sums_slot], 0));
	L.p = h->p;
	L.coll = h->d.collision;
	L.cum_flags = h->d.cum_flags;
	L.odd = (h->iteration % 2) != 0;
	L.grid = h->grid();
	L.block = h->block();
	L.stream = h->stream;
	L.kernel = h->kernel;
	L.status = h->status_dev;
	L.wait_limit = h->wait_limit;
	long long blocks = 0;
	L.blocks_out = &blocks;
	bool nothing_skipped = false;
	L.nothing_skipped = &nothing_skipped;
	L.dry_run = dry_run;
	L.f_out = h->f_out;
	L.split_tiles = h->split_tiles;
	L.split_n[0] = h->split_n[0];
	L.split_n[1] = h->split_n[1];
	L.split_tiles_x = h->split_tiles_x;
	L.pair_groups = h->pair_groups;
	L.pair_work = lbm::PairWork{h->pair_work[0], h->pair_nwork[0], h->pair_rest[0], h->pair_nrest[0]};
	L.pair_work_out = lbm::PairWork{h->pair_work[1], h->pair_nwork[1], h->pair_rest[1], h->pair_nrest[1]};
	L.distributed_z = h->distributed_z;
	const bool ab = h->streaming == LBM_STREAMING_AB;
	if (h->ade) {
		h->ade->launch.phi = macro ? h->ade->phi_buf : nullptr;
		L.ade = &h->ade->launch;
		if (!dry_run)
			h->ade->phi_valid = macro;
	}
	if (h->plugin) {  // a registered collision: its own direct kernel
		const int32_t rc = h->plugin(&L, h->d.storage);
		if (rc != 0)
			return fail(LBM_ERR_CUDA, "collision plugin %d step launch failed: %s", h->d.collision,
						cudaGetErrorString((cudaError_t) rc));
		if (dry_run)
			return LBM_OK;
		h->last_blocks = blocks;
		h->last_nothing_skipped = nothing_skipped;
		h->iteration++;
		return LBM_OK;
	}
	cudaError_t err = cudaErrorNotSupported;
	// the two-site coupled step (FP32 storage, plain steps of a lattice with a map)
	if (h->ade && h->kernel == lbm::KERNEL_PAIR && h->d.storage == lbm::ST_F32 && !macro && !sums) {
		if (h->ade->pair_dirty)
			if (int rc = lbm::ade_build_pair(h))
				return rc;
		err = lbm::ade_pair_step_f32(L);
	}
	// the two-site kernel where it applies (FP32 arithmetic),
	// else the direct kernel
	if (!h->ade && !ab && h->kernel == lbm::KERNEL_PAIR)
		if (const lbm::PairStepFn pair = lbm::pair_step_of(h->d.storage))
			err = pair(L);
	if (err == cudaErrorNotSupported)
		err = h->ade ? h->ops->ade_step(L) : (ab ? h->ops->ab_step(L) : h->ops->step(L));
	if (err != cudaSuccess)
		return fail(LBM_ERR_CUDA, "step kernel launch failed: %s", cudaGetErrorString(err));
	if (dry_run)
		return LBM_OK;
	h->last_blocks = blocks;
	h->last_nothing_skipped = nothing_skipped;
	h->iteration++;
	if (ab)	 // pointer rotation of lbm.hpp:314-322
		std::swap(h->g.f, h->f_out);
	return LBM_OK;
}

// A-B: ghost and GEO_NOTHING entries are never written, so both buffers must
// hold the same values; called after every write of the populations
int sync_ab_buffers(lbm_handle h)
{
	if (h->streaming == LBM_STREAMING_AB && h->f_out)
		LBM_CUDA(cudaMemcpyAsync(h->f_out, h->g.f, h->pop_bytes, cudaMemcpyDeviceToDevice, h->stream));
	return LBM_OK;
}

// the graph slot captured with the current population buffer and inlet
// profiles, or null
lbm_lattice::GraphSlot* current_graph(lbm_handle h)
{
	for (lbm_lattice::GraphSlot& g : h->graphs)
		if (g.exec && g.f == h->g.f && g.inflow[0] == h->inflow[0] && g.inflow[1] == h->inflow[1]
			&& g.inflow[2] == h->inflow[2])
			return &g;
	return nullptr;
}

int build_graph(lbm_handle h)
{
	lbm_lattice::GraphSlot& slot = h->graphs[h->graph_next];
	if (slot.exec)
		cudaGraphExecDestroy(slot.exec);
	slot = lbm_lattice::GraphSlot{};
	const long long saved = h->iteration;
	// resolve per-kernel launch attributes outside of the capture
	for (int parity = 0; parity < 2; parity++) {
		h->iteration = parity;
		int rc = launch_step(h, false, false, true);
		if (rc) {
			h->iteration = saved;
			return rc;
		}
	}
	h->iteration = 0;  // graph starts at an even step
	cudaGraph_t graph = nullptr;
	LBM_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
	int rc = LBM_OK;
	for (int s = 0; s < lbm_lattice::GRAPH_STEPS && rc == LBM_OK; s++)
		rc = launch_step(h, false, false);
	const cudaError_t end = cudaStreamEndCapture(h->stream, &graph);
	h->iteration = saved;
	if (rc != LBM_OK) {
		if (graph)
			cudaGraphDestroy(graph);
		return rc;
	}
	if (end != cudaSuccess)
		return fail(LBM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(end));
	const cudaError_t inst = cudaGraphInstantiate(&slot.exec, graph, 0);
	cudaGraphDestroy(graph);
	if (inst != cudaSuccess) {
		slot.exec = nullptr;
		return fail(LBM_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(inst));
	}
	slot.f = h->g.f;
	for (int k = 0; k < 3; k++)
		slot.inflow[k] = h->inflow[k];
	h->graph_next ^= 1;
	return LBM_OK;
}

int run_plain_steps(lbm_handle h, long long n)
{
	while (n > 0 && (h->iteration % 2) != 0) {
		int rc = launch_step(h, false, false);
		if (rc)
			return rc;
		n--;
	}
	if (h->d.use_graphs && n >= lbm_lattice::GRAPH_STEPS) {
		lbm_lattice::GraphSlot* g = current_graph(h);
		if (!g) {
			if (int rc = build_graph(h))
				return rc;
			g = current_graph(h);
		}
		while (n >= lbm_lattice::GRAPH_STEPS) {
			LBM_CUDA(cudaGraphLaunch(g->exec, h->stream));
			h->iteration += lbm_lattice::GRAPH_STEPS;
			n -= lbm_lattice::GRAPH_STEPS;
		}
	}
	while (n > 0) {
		int rc = launch_step(h, false, false);
		if (rc)
			return rc;
		n--;
	}
	return LBM_OK;
}

}  // namespace

extern "C" {

const char* lbm_last_error(void)
{
	return g_error.c_str();
}

int lbm_register_collision(int32_t id, lbm_collision_launcher launcher, int32_t abi_version, const char* name)
{
	if (!plugin_id(id))
		return fail(LBM_ERR_INVALID, "collision plugin id %d outside %d .. %d", id, LBM_COLL_PLUGIN_FIRST,
					LBM_COLL_PLUGIN_LAST);
	if (abi_version != LBM_PLUGIN_ABI_VERSION)
		return fail(LBM_ERR_UNSUPPORTED, "collision plugin built for plugin ABI %d, the library has %d", abi_version,
					LBM_PLUGIN_ABI_VERSION);
	std::lock_guard<std::mutex> lock(g_plugins_mutex);
	CollisionPlugin& slot = g_plugins[id - LBM_COLL_PLUGIN_FIRST];
	slot.launch = launcher;
	slot.name = launcher ? (name ? name : "") : "";
	return LBM_OK;
}

const char* lbm_collision_name(int32_t id)
{
	if (!plugin_id(id))
		return nullptr;
	std::lock_guard<std::mutex> lock(g_plugins_mutex);
	const CollisionPlugin& slot = g_plugins[id - LBM_COLL_PLUGIN_FIRST];
	return slot.launch ? slot.name.c_str() : nullptr;
}

const char* lbm_version(void)
{
	return "tnl-lbm-b200 0.1 (sm_100a, D3Q27 A-A)";
}

int lbm_create(const lbm_desc* desc, lbm_handle* out)
{
	if (!desc || !out)
		return fail(LBM_ERR_INVALID, "null argument");
	*out = nullptr;
	const lbm_desc& d = *desc;
	if (d.X < 1 || d.Y < 1 || d.Z < 1)
		return fail(LBM_ERR_INVALID, "lattice sizes must be positive (got %d x %d x %d)", d.X, d.Y, d.Z);
	if (d.X > 65535 * 4 || d.Y > 65535 || d.Z > 65535)
		return fail(LBM_ERR_SIZE, "lattice sizes beyond the launch limits");
	if (d.storage < 0 || d.storage >= lbm::ST_COUNT)
		return fail(LBM_ERR_INVALID, "unknown storage %d", d.storage);
	lbm_collision_launcher plugin = nullptr;
	if (plugin_id(d.collision)) {
		{
			std::lock_guard<std::mutex> lock(g_plugins_mutex);
			plugin = g_plugins[d.collision - LBM_COLL_PLUGIN_FIRST].launch;
		}
		if (!plugin)
			return fail(LBM_ERR_INVALID, "no collision plugin registered under id %d", d.collision);
		if (plugin(nullptr, d.storage) != 0)
			return fail(LBM_ERR_UNSUPPORTED, "collision plugin %d was not built for storage %d", d.collision, d.storage);
		if (d.cum_flags != 0)
			return fail(LBM_ERR_INVALID, "cumulant flags %d given for a collision plugin", d.cum_flags);
	}
	else if (d.collision < LBM_COLL_CUM || d.collision > LBM_COLL_MRT)
		return fail(LBM_ERR_INVALID, "unknown collision %d", d.collision);
	if (d.collision == LBM_COLL_CUM && d.cum_flags != 0 && d.cum_flags != LBM_CUM_ANTIALIAS
		&& d.cum_flags != (LBM_CUM_GEIER_2017 | LBM_CUM_ANTIALIAS))
		return fail(LBM_ERR_UNSUPPORTED, "cumulant flags %d: the 2017 variant requires the anti-aliasing terms", d.cum_flags);
	if (d.equilibrium != LBM_EQ_SECOND_ORDER && d.equilibrium != LBM_EQ_INV_CUM)
		return fail(LBM_ERR_INVALID, "unknown equilibrium %d", d.equilibrium);
	if (!(d.viscosity > 0.0) || !std::isfinite(d.viscosity))
		return fail(LBM_ERR_INVALID, "viscosity must be positive and finite (state.hpp:1240-1245)");
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
		return fail(LBM_ERR_CUDA, "no CUDA device available");
	if (d.device < 0 || d.device >= ndev)
		return fail(LBM_ERR_INVALID, "device %d out of range", d.device);
	LBM_CUDA(cudaSetDevice(d.device));

	lbm_lattice* h = new lbm_lattice();
	h->d = d;
	h->plugin = plugin;
	h->ops = &lbm::storage_ops(d.storage);
	const int es = h->ops->elem_size;
	h->g = lbm::make_geometry(d.X, d.Y, d.Z, es);
	h->pop_bytes = lbm::geometry_elems(h->g) * es;
	lbm::cumulant_rates(d.viscosity, h->p);
	h->p.nu = d.viscosity;
	h->p.fx = d.fx;
	h->p.fy = d.fy;
	h->p.fz = d.fz;
	h->p.eq = d.equilibrium;

	auto cleanup = [&](int rc) {
		lbm_destroy(h);
		return rc;
	};
	if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
		return cleanup(fail(LBM_ERR_CUDA, "stream creation failed"));
	cudaError_t e = cudaMalloc(&h->g.f, h->pop_bytes);
	if (e != cudaSuccess)
		return cleanup(fail(LBM_ERR_CUDA, "population allocation of %zu bytes failed: %s", h->pop_bytes, cudaGetErrorString(e)));
	if (cudaMemsetAsync(h->g.f, 0, h->pop_bytes, h->stream) != cudaSuccess)
		return cleanup(fail(LBM_ERR_CUDA, "population memset failed"));
	// the tile kernel copies map rows from 16-byte aligned windows that can end
	// up to 15 bytes past the last site: pad the allocation
	if (!d.periodic
		&& (cudaMalloc(&h->map, (size_t) h->sites() + 64) != cudaSuccess
			|| cudaMemsetAsync(h->map, 0, (size_t) h->sites() + 64, h->stream) != cudaSuccess))
		return cleanup(fail(LBM_ERR_CUDA, "map allocation failed"));
	// the finish stream at the highest priority: its few blocks take the first
	// SM slots that the next step's blocks free instead of queueing behind
	// them (at the default priority the end-to-end step was slower)
	int top = 0;
	if (cudaHostAlloc(&h->sums_host, 2 * lbm::NRED_HOST * sizeof(double), cudaHostAllocMapped) != cudaSuccess
		|| cudaEventCreateWithFlags(&h->sums_ev[0], cudaEventDisableTiming) != cudaSuccess
		|| cudaEventCreateWithFlags(&h->sums_ev[1], cudaEventDisableTiming) != cudaSuccess
		|| cudaHostGetDevicePointer((void**) &h->sums_mapped, h->sums_host, 0) != cudaSuccess
		|| cudaMalloc(&h->finish_arrived, 2 * sizeof(unsigned)) != cudaSuccess
		|| cudaMemsetAsync(h->finish_arrived, 0, 2 * sizeof(unsigned), h->stream) != cudaSuccess
		|| cudaDeviceGetStreamPriorityRange(nullptr, &top) != cudaSuccess
		|| cudaStreamCreateWithPriority(&h->finish_stream, cudaStreamNonBlocking, top) != cudaSuccess
		|| cudaEventCreateWithFlags(&h->step_ev[0], cudaEventDisableTiming) != cudaSuccess
		|| cudaEventCreateWithFlags(&h->step_ev[1], cudaEventDisableTiming) != cudaSuccess)
		return cleanup(fail(LBM_ERR_CUDA, "reduction buffers allocation failed"));
	if (cudaMalloc(&h->status_dev, sizeof(int)) != cudaSuccess || cudaMemsetAsync(h->status_dev, 0, sizeof(int), h->stream) != cudaSuccess)
		return cleanup(fail(LBM_ERR_CUDA, "status word allocation failed"));
	cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, d.device);
	int rc = ensure_partials(h, h->max_step_blocks());
	if (rc)
		return cleanup(rc);
	*out = h;
	return LBM_OK;
}

int lbm_destroy(lbm_handle h)
{
	if (!h)
		return LBM_OK;
	cudaSetDevice(h->d.device);
	if (h->stream)
		cudaStreamSynchronize(h->stream);
	h->drop_graph();
	lbm::adjoint_free(h->adjoint);
	lbm::ade_free(h->ade);
	cudaFree(h->g.f);
	cudaFree(h->f_out);
	cudaFree(h->split_tiles);
	for (int k = 0; k < 2; k++) {
		cudaFree(h->pair_rest[k]);
		cudaFree(h->pair_work[k]);
	}
	cudaFree(h->pair_groups);
	cudaFree(h->stats);
	cudaFree(h->map);
	if (h->upload_stream)
		cudaStreamSynchronize(h->upload_stream);
	for (auto& set : h->inflow_buf)
		for (void* p : set)
			cudaFree(p);
	cudaFree(h->macro);
	if (h->inflow_host)
		cudaFreeHost(h->inflow_host);
	for (cudaEvent_t ev : {h->inflow_ready, h->inflow_free[0], h->inflow_free[1], h->inflow_staged[0], h->inflow_staged[1]})
		if (ev)
			cudaEventDestroy(ev);
	if (h->upload_stream)
		cudaStreamDestroy(h->upload_stream);
	if (h->halo_ev)
		cudaEventDestroy(h->halo_ev);
	if (h->finish_stream)
		cudaStreamSynchronize(h->finish_stream);
	cudaFree(h->partials);
	cudaFree(h->finish_arrived);
	cudaFree(h->status_dev);
	if (h->sums_host)
		cudaFreeHost(h->sums_host);
	for (cudaEvent_t ev : {h->sums_ev[0], h->sums_ev[1], h->step_ev[0], h->step_ev[1]})
		if (ev)
			cudaEventDestroy(ev);
	if (h->finish_stream)
		cudaStreamDestroy(h->finish_stream);
	if (h->stream)
		cudaStreamDestroy(h->stream);
	delete h;
	return LBM_OK;
}

int lbm_set_map(lbm_handle h, const uint8_t* map)
{
	if (int rc = check(h))
		return rc;
	if (h->d.periodic)
		return fail(LBM_ERR_INVALID, "periodic lattice has no map");
	if (!map)
		return fail(LBM_ERR_INVALID, "null map");
	const long long n = h->sites();
	for (long long i = 0; i < n; i++)
		if (!site_type_supported(map[i])
			&& !(h->streaming == LBM_STREAMING_AB
				 && (map[i] == lbm::GEO_INFLOW_BB_LEFT || map[i] == lbm::GEO_OUTFLOW_RIGHT
					 || map[i] == lbm::GEO_OUTFLOW_RIGHT_INTERP)))
			return fail(LBM_ERR_UNSUPPORTED,
						"site type %d at index %lld is not provided by the A-A kernels (reads a slot another site writes "
						"in the same pass, or belongs to the adjoint set)",
						(int) map[i], i);
	LBM_CUDA(cudaMemcpyAsync(h->map, map, (size_t) n, cudaMemcpyHostToDevice, h->stream));
	LBM_CUDA(cudaStreamSynchronize(h->stream));
	h->map_host.assign(map, map + n);
	h->map_set = true;
	h->nothing_sites = 0;
	for (size_t i = 0; i < n; i++)
		h->nothing_sites += map[i] == lbm::GEO_NOTHING;
	if (h->ade)
		h->ade->pair_dirty = true;  // the coupled pair step's lists follow the flow map
	// tiles of 128 x-sites for the split step: fluid-only ones first
	{
		const int tx = (h->d.X + 127) / 128;
		std::vector<unsigned> fluid, other;
		for (long long row = 0; row < (long long) h->d.Y * h->d.Z; row++)
			for (int t = 0; t < tx; t++) {
				bool all = (t + 1) * 128 <= h->d.X;
				for (int i = 0; all && i < 128; i++)
					all = map[row * h->d.X + t * 128 + i] == lbm::GEO_FLUID;
				(all ? fluid : other).push_back((unsigned) (row * tx + t));
			}
		cudaFree(h->split_tiles);
		h->split_tiles = nullptr;
		const size_t nt = fluid.size() + other.size();
		if (nt > 0xffffffffull)
			return fail(LBM_ERR_SIZE, "too many tiles for the split step");
		fluid.insert(fluid.end(), other.begin(), other.end());
		LBM_CUDA(cudaMalloc(&h->split_tiles, nt * sizeof(unsigned)));
		LBM_CUDA(cudaMemcpyAsync(h->split_tiles, fluid.data(), nt * sizeof(unsigned), cudaMemcpyHostToDevice, h->stream));
		LBM_CUDA(cudaStreamSynchronize(h->stream));
		h->split_n[0] = (long long) (nt - other.size());
		h->split_n[1] = (long long) other.size();
		h->split_tiles_x = tx;
		// groups of the two-site step (PAIR_GROUP sites of a row: all
		// GEO_FLUID, all GEO_PERIODIC, or the rest), the sites of the rest
		// groups in row order (without GEO_NOTHING sites for plain steps, with
		// them for observation steps, where they give their outputs), and the
		// work lists: per z plane the chunks of 128 rest sites that start in it,
		// then the plane's tiles of 256 x-sites that hold a pair group
		const int X = h->d.X, Y = h->d.Y, Z = h->d.Z;
		const int gx = (X + lbm::PAIR_GROUP - 1) / lbm::PAIR_GROUP;
		const int tiles_x = ((X + 1) / 2 + 127) / 128;
		std::vector<uint8_t> groups((size_t) gx * Y * Z);
		std::vector<unsigned long long> rest[2];
		for (long long row = 0; row < (long long) Y * Z; row++)
			for (int k = 0; k < gx; k++) {
				const int x0 = k * lbm::PAIR_GROUP;
				const uint8_t first = map[row * X + x0];
				bool same = x0 + lbm::PAIR_GROUP <= X && (first == lbm::GEO_FLUID || first == lbm::GEO_PERIODIC);
				for (int x = x0 + 1; same && x < x0 + lbm::PAIR_GROUP; x++)
					same = map[row * X + x] == first;
				groups[row * gx + k] = !same ? lbm::PAIR_GROUP_REST
										: (first == lbm::GEO_PERIODIC ? lbm::PAIR_GROUP_PERIODIC : lbm::PAIR_GROUP_FLUID);
				if (!same)
					for (int x = x0; x < x0 + lbm::PAIR_GROUP && x < X; x++) {
						const unsigned long long e = (unsigned long long) row << 32 | (unsigned) x;
						if (map[row * X + x] != lbm::GEO_NOTHING)
							rest[0].push_back(e);
						rest[1].push_back(e);
					}
			}
		std::vector<unsigned> work[2];
		for (int k = 0; k < 2; k++) {
			const long long nchunks = ((long long) rest[k].size() + 127) / 128;
			if (nchunks > (long long) (lbm::PAIR_WORK_REST - 1) || (long long) Y * Z * tiles_x >= (long long) lbm::PAIR_WORK_REST)
				return fail(LBM_ERR_SIZE, "lattice too large for the pair step's work list");
			long long c = 0;
			for (int z = 0; z < Z; z++) {
				// the chunks whose first site lies in plane z, ahead of the plane's
				// tiles: the slower per-site work starts first and the tiles fill in
				// around it (duct 26.7 -> 28.3 GLUPS against chunks after the tiles)
				while (c < nchunks && (long long) (rest[k][(size_t) c * 128] >> 32) / Y <= z)
					work[k].push_back(lbm::PAIR_WORK_REST | (unsigned) c++);
				for (int y = 0; y < Y; y++) {
					const long long row = (long long) z * Y + y;
					for (int t = 0; t < tiles_x; t++) {
						bool any = false;
						for (int g = t * 256 / lbm::PAIR_GROUP; !any && g < gx && g < (t + 1) * 256 / lbm::PAIR_GROUP; g++)
							any = groups[row * gx + g] != lbm::PAIR_GROUP_REST;
						if (any)
							work[k].push_back((unsigned) (row * tiles_x + t));
					}
				}
			}
		}
		cudaFree(h->pair_groups);
		h->pair_groups = nullptr;
		LBM_CUDA(cudaMalloc(&h->pair_groups, groups.size()));
		LBM_CUDA(cudaMemcpyAsync(h->pair_groups, groups.data(), groups.size(), cudaMemcpyHostToDevice, h->stream));
		for (int k = 0; k < 2; k++) {
			cudaFree(h->pair_rest[k]);
			cudaFree(h->pair_work[k]);
			h->pair_rest[k] = nullptr;
			h->pair_work[k] = nullptr;
			h->pair_nrest[k] = (long long) rest[k].size();
			h->pair_nwork[k] = (long long) work[k].size();
			LBM_CUDA(cudaMalloc(&h->pair_rest[k], (rest[k].empty() ? 1 : rest[k].size()) * sizeof(unsigned long long)));
			LBM_CUDA(cudaMalloc(&h->pair_work[k], (work[k].empty() ? 1 : work[k].size()) * sizeof(unsigned)));
			if (!rest[k].empty())
				LBM_CUDA(cudaMemcpyAsync(h->pair_rest[k], rest[k].data(), rest[k].size() * sizeof(unsigned long long),
										 cudaMemcpyHostToDevice, h->stream));
			if (!work[k].empty())
				LBM_CUDA(cudaMemcpyAsync(h->pair_work[k], work[k].data(), work[k].size() * sizeof(unsigned),
										 cudaMemcpyHostToDevice, h->stream));
		}
		LBM_CUDA(cudaStreamSynchronize(h->stream));
		h->drop_graph();
	}
	return LBM_OK;
}

int lbm_get_map(lbm_handle h, uint8_t* map)
{
	if (int rc = check(h))
		return rc;
	if (!map)
		return fail(LBM_ERR_INVALID, "null map");
	if (h->d.periodic || h->map_host.empty())
		return fail(LBM_ERR_INVALID, "no map: the lattice is periodic or lbm_set_map was not called");
	std::memcpy(map, h->map_host.data(), h->map_host.size());
	return LBM_OK;
}

int lbm_set_inflow(lbm_handle h, const double* vx, const double* vy, const double* vz)
{
	if (int rc = check(h))
		return rc;
	const double* src[3] = {vx, vy, vz};
	const size_t n = (size_t) h->d.Y * h->d.Z;
	const int cs = h->ops->compute_size;
	if (!h->upload_stream) {
		LBM_CUDA(cudaMallocHost(&h->inflow_host, 2 * 3 * n * cs));
		LBM_CUDA(cudaStreamCreateWithFlags(&h->upload_stream, cudaStreamNonBlocking));
		for (cudaEvent_t* ev : {&h->inflow_ready, &h->inflow_free[0], &h->inflow_free[1], &h->inflow_staged[0], &h->inflow_staged[1]})
			LBM_CUDA(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
	}
	// upload into the set that is not current, from staging slot b: the
	// slot's previous copies (two calls ago) are normally long done, and the
	// set's last readers are the steps queued before it stopped being current
	const int b = h->inflow_cur ^ 1;
	LBM_CUDA(cudaEventSynchronize(h->inflow_staged[b]));
	if (h->inflow_free_valid[b])
		LBM_CUDA(cudaStreamWaitEvent(h->upload_stream, h->inflow_free[b], 0));
	void* next[3] = {nullptr, nullptr, nullptr};
	for (int k = 0; k < 3; k++) {
		if (!src[k])
			continue;  // a null component reads as zero
		if (!h->inflow_buf[b][k])
			LBM_CUDA(cudaMalloc(&h->inflow_buf[b][k], n * cs));
		unsigned char* stage = (unsigned char*) h->inflow_host + (size_t) (3 * b + k) * n * cs;
		if (cs == 8)
			std::memcpy(stage, src[k], n * 8);
		else
			for (size_t i = 0; i < n; i++)
				((float*) stage)[i] = (float) src[k][i];
		LBM_CUDA(cudaMemcpyAsync(h->inflow_buf[b][k], stage, n * cs, cudaMemcpyHostToDevice, h->upload_stream));
		next[k] = h->inflow_buf[b][k];
	}
	LBM_CUDA(cudaEventRecord(h->inflow_staged[b], h->upload_stream));
	LBM_CUDA(cudaEventRecord(h->inflow_ready, h->upload_stream));
	// later work on the lattice's stream sees the new profiles; the current
	// set is free once the work queued so far is done
	LBM_CUDA(cudaStreamWaitEvent(h->stream, h->inflow_ready, 0));
	LBM_CUDA(cudaEventRecord(h->inflow_free[h->inflow_cur], h->stream));
	h->inflow_free_valid[h->inflow_cur] = true;
	h->inflow_cur = b;
	for (int k = 0; k < 3; k++)
		h->inflow[k] = next[k];
	return LBM_OK;
}

int lbm_set_viscosity(lbm_handle h, double nu)
{
	if (int rc = check(h))
		return rc;
	if (!(nu > 0.0) || !std::isfinite(nu))
		return fail(LBM_ERR_INVALID, "viscosity must be positive and finite");
	h->d.viscosity = nu;
	lbm::cumulant_rates(nu, h->p);
	h->p.nu = nu;
	h->drop_graph();
	return LBM_OK;
}

int lbm_init_equilibrium(lbm_handle h, const double* rho, const double* vx, const double* vy, const double* vz, double rho0,
						 double vx0, double vy0, double vz0)
{
	if (int rc = check(h))
		return rc;
	const bool fields = rho || vx || vy || vz;
	if (fields && !(rho && vx && vy && vz))
		return fail(LBM_ERR_INVALID, "either all four fields or none");
	lbm::InitSpec spec{};
	spec.mode = fields ? 1 : 0;
	spec.eq = h->d.equilibrium;
	spec.rho0 = rho0;
	spec.vx0 = vx0;
	spec.vy0 = vy0;
	spec.vz0 = vz0;
	double* dev = nullptr;
	const size_t n = (size_t) h->sites();
	if (fields) {
		LBM_CUDA(cudaMallocAsync((void**) &dev, 4 * n * sizeof(double), h->stream));
		const double* src[4] = {rho, vx, vy, vz};
		for (int k = 0; k < 4; k++)
			LBM_CUDA(cudaMemcpyAsync(dev + k * n, src[k], n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
		spec.rho = dev;
		spec.vx = dev + n;
		spec.vy = dev + 2 * n;
		spec.vz = dev + 3 * n;
	}
	const cudaError_t e = h->ops->init_eq(h->g, spec, h->stream);
	if (dev)
		cudaFreeAsync(dev, h->stream);
	if (e != cudaSuccess)
		return fail(LBM_ERR_CUDA, "init kernel failed: %s", cudaGetErrorString(e));
	if (int rc = sync_ab_buffers(h))
		return rc;
	LBM_CUDA(cudaStreamSynchronize(h->stream));
	h->iteration = 0;
	h->macro_valid = h->sums_valid = false;
	return LBM_OK;
}

int lbm_init_taylor_green(lbm_handle h, double u0, double rho0)
{
	if (int rc = check(h))
		return rc;
	lbm::InitSpec spec{};
	spec.mode = 2;
	spec.eq = h->d.equilibrium;
	spec.rho0 = rho0;
	spec.u0 = u0;
	const cudaError_t e = h->ops->init_eq(h->g, spec, h->stream);
	if (e != cudaSuccess)
		return fail(LBM_ERR_CUDA, "init kernel failed: %s", cudaGetErrorString(e));
	if (int rc = sync_ab_buffers(h))
		return rc;
	LBM_CUDA(cudaStreamSynchronize(h->stream));
	h->iteration = 0;
	h->macro_valid = h->sums_valid = false;
	return LBM_OK;
}

static size_t dense_count(lbm_handle h, int layout)
{
	const int gh = layout == LBM_LAYOUT_GHOST ? 2 : 0;
	return (size_t) 27 * (h->d.X + gh) * (size_t) (h->d.Y + gh) * (h->d.Z + gh);
}

int lbm_set_populations(lbm_handle h, const void* host, int layout, int dtype)
{
	if (int rc = check(h))
		return rc;
	if (!host || (layout != 0 && layout != 1) || (dtype != 0 && dtype != 1))
		return fail(LBM_ERR_INVALID, "bad arguments");
	const size_t bytes = dense_count(h, layout) * (dtype == 0 ? 8 : 4);
	void* dev = nullptr;
	LBM_CUDA(cudaMallocAsync(&dev, bytes, h->stream));
	LBM_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, h->stream));
	const cudaError_t e = h->ops->unpack(h->g, dev, dtype, layout, h->stream);
	cudaFreeAsync(dev, h->stream);
	if (e != cudaSuccess)
		return fail(LBM_ERR_CUDA, "unpack failed: %s", cudaGetErrorString(e));
	if (int rc = sync_ab_buffers(h))
		return rc;
	LBM_CUDA(cudaStreamSynchronize(h->stream));
	return LBM_OK;
}

int lbm_get_populations(lbm_handle h, void* host, int layout, int dtype)
{
	if (int rc = check(h))
		return rc;
	if (!host || (layout != 0 && layout != 1) || (dtype != 0 && dtype != 1))
		return fail(LBM_ERR_INVALID, "bad arguments");
	const size_t bytes = dense_count(h, layout) * (dtype == 0 ? 8 : 4);
	void* dev = nullptr;
	LBM_CUDA(cudaMallocAsync(&dev, bytes, h->stream));
	const cudaError_t e = h->ops->pack(h->g, dev, dtype, layout, h->stream);
	if (e != cudaSuccess) {
		cudaFreeAsync(dev, h->stream);
		return fail(LBM_ERR_CUDA, "pack failed: %s", cudaGetErrorString(e));
	}
	LBM_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, h->stream));
	cudaFreeAsync(dev, h->stream);
	LBM_CUDA(cudaStreamSynchronize(h->stream));
	return LBM_OK;
}

// FP64 sums of the observation step just launched, written by the finish
// kernel straight into the next slot of the mapped pinned ring; the slot's
// event lets a reader wait for this step alone
int finish_observation(lbm_handle h)
{
	const int slot = h->sums_last ^ 1;
	const long long nb = h->last_blocks;
	const double mass_offset = h->last_nothing_skipped ? (double) h->nothing_sites : 0.0;
	double* part = partials_of(h, slot);
	// on the finish stream: the lattice's next step does not wait for it
	LBM_CUDA(cudaEventRecord(h->step_ev[slot], h->stream));
	LBM_CUDA(cudaStreamWaitEvent(h->finish_stream, h->step_ev[slot], 0));
	const cudaError_t e = lbm::finish_sums(part, nb, part + nb * lbm::NRED_HOST, h->finish_arrived + slot,
										   h->sums_mapped + slot * lbm::NRED_HOST, h->finish_stream, mass_offset);
	if (e != cudaSuccess)
		return fail(LBM_ERR_CUDA, "sum finish failed: %s", cudaGetErrorString(e));
	LBM_CUDA(cudaEventRecord(h->sums_ev[slot], h->finish_stream));
	h->sums_iter[slot] = h->iteration;
	h->sums_last = slot;
	return LBM_OK;
}

int lbm_step(lbm_handle h, int64_t nsteps, int flags)
{
	if (int rc = check(h))
		return rc;
	if (nsteps < 0 || (nsteps == 0 && flags))
		return fail(LBM_ERR_INVALID, "nsteps must be positive when flags are given");
	if (!h->d.periodic && !h->map_set)
		return fail(LBM_ERR_INVALID, "lbm_set_map must be called before stepping a non-periodic lattice");
	if (nsteps == 0)
		return LBM_OK;
	const bool macro = (flags & LBM_STEP_MACRO) != 0;
	const bool sums = (flags & LBM_STEP_SUMS) != 0;
	if (h->stats) {
		// D3Q27_MACRO_Mean computes in every iteration (macro.h:113): every step
		// outputs the macro field and updates the statistics
		int rc = ensure_macro(h);
		if (rc || (sums && (rc = ensure_partials(h, h->max_step_blocks()))))
			return rc;
		for (int64_t i = 0; i < nsteps; i++) {
			const bool last_sums = sums && i == nsteps - 1;
			if ((rc = launch_step(h, true, last_sums)))
				return rc;
			const cudaError_t e =
				lbm::stats_update(h->macro, h->stats, h->ops->compute_size, h->sites(), (int) h->stats_count, h->stream);
			if (e != cudaSuccess)
				return fail(LBM_ERR_CUDA, "statistics update failed: %s", cudaGetErrorString(e));
			h->stats_count++;
		}
		if (sums && (rc = finish_observation(h)))
			return rc;
		h->macro_valid = true;
		h->sums_valid = sums;
		return LBM_OK;
	}
	int rc = run_plain_steps(h, nsteps - ((macro || sums) ? 1 : 0));
	if (rc)
		return rc;
	if (macro || sums) {
		if (macro && (rc = ensure_macro(h)))
			return rc;
		if (sums && (rc = ensure_partials(h, h->max_step_blocks())))
			return rc;
		if ((rc = launch_step(h, macro, sums)))
			return rc;
		if (sums && (rc = finish_observation(h)))
			return rc;
		h->macro_valid = macro;
		h->sums_valid = sums;
	}
	else {
		h->macro_valid = h->sums_valid = false;
	}
	return LBM_OK;
}

int64_t lbm_iteration(lbm_handle h)
{
	return h ? h->iteration : -1;
}

int lbm_set_iteration(lbm_handle h, int64_t iteration)
{
	if (int rc = check(h))
		return rc;
	if (iteration < 0)
		return fail(LBM_ERR_INVALID, "iteration must be non-negative");
	h->iteration = iteration;
	return LBM_OK;
}

int lbm_get_macro(lbm_handle h, double* host)
{
	if (int rc = check(h))
		return rc;
	if (!host)
		return fail(LBM_ERR_INVALID, "null output");
	if (!h->macro_valid)
		return fail(LBM_ERR_INVALID, "no macro field: run lbm_step with LBM_STEP_MACRO first");
	const size_t n = 4 * (size_t) h->sites();
	if (h->ops->compute_size == 8) {
		LBM_CUDA(cudaMemcpyAsync(host, h->macro, n * 8, cudaMemcpyDeviceToHost, h->stream));
		LBM_CUDA(cudaStreamSynchronize(h->stream));
	}
	else {
		std::vector<float> tmp(n);
		LBM_CUDA(cudaMemcpyAsync(tmp.data(), h->macro, n * 4, cudaMemcpyDeviceToHost, h->stream));
		LBM_CUDA(cudaStreamSynchronize(h->stream));
		for (size_t i = 0; i < n; i++)
			host[i] = tmp[i];
	}
	return LBM_OK;
}

int lbm_get_sums(lbm_handle h, double* out)
{
	if (int rc = check(h))
		return rc;
	if (!out)
		return fail(LBM_ERR_INVALID, "null output");
	if (!h->sums_valid)
		return fail(LBM_ERR_INVALID, "no sums: run lbm_step with LBM_STEP_SUMS first");
	return lbm_get_sums_of(h, h->sums_iter[h->sums_last], out);
}

int lbm_get_sums_of(lbm_handle h, int64_t iteration, double* out)
{
	if (int rc = check(h))
		return rc;
	if (!out)
		return fail(LBM_ERR_INVALID, "null output");
	int slot = -1;
	for (int k = 0; k < 2; k++)
		if (h->sums_iter[k] == iteration && iteration >= 0)
			slot = k;
	if (slot < 0)
		return fail(LBM_ERR_INVALID, "no sums of iteration %lld: the last two observation steps ended at %lld and %lld",
					(long long) iteration, h->sums_iter[h->sums_last], h->sums_iter[h->sums_last ^ 1]);
	// wait for that step's finish kernel only, not for work queued after it
	LBM_CUDA(cudaEventSynchronize(h->sums_ev[slot]));
	std::memcpy(out, h->sums_host + slot * lbm::NRED_HOST, lbm::NRED_HOST * sizeof(double));
	if (out[5] != 0.0)
		return fail(LBM_ERR_NONFINITE, "%.0f sites with a non-finite density", out[5]);
	return LBM_OK;
}

int lbm_enstrophy_sum(lbm_handle h, double* out)
{
	if (int rc = check(h))
		return rc;
	if (!out)
		return fail(LBM_ERR_INVALID, "null output");
	if (!h->macro_valid)
		return fail(LBM_ERR_INVALID, "no macro field: run lbm_step with LBM_STEP_MACRO first");
	long long nb = 0;
	const long long need = (long long) ((h->d.X + 127) / 128) * h->d.Y * h->d.Z;
	if (int rc = ensure_partials(h, need))
		return rc;
	double* dres = nullptr;
	LBM_CUDA(cudaMallocAsync((void**) &dres, lbm::NRED_HOST * sizeof(double), h->stream));
	// slot 0 and its counter, once the finish kernels in flight are done
	for (cudaEvent_t ev : h->sums_ev)
		LBM_CUDA(cudaStreamWaitEvent(h->stream, ev, 0));
	double* part = partials_of(h, 0);
	cudaError_t e = lbm::enstrophy_partials(h->macro, h->ops->compute_size, h->d.X, h->d.Y, h->d.Z, part, &nb, h->stream);
	if (e == cudaSuccess)
		e = lbm::finish_sums(part, nb, part + nb * lbm::NRED_HOST, h->finish_arrived, dres, h->stream);
	double res[lbm::NRED_HOST];
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(res, dres, sizeof(res), cudaMemcpyDeviceToHost, h->stream);
	cudaFreeAsync(dres, h->stream);
	if (e != cudaSuccess)
		return fail(LBM_ERR_CUDA, "enstrophy reduction failed: %s", cudaGetErrorString(e));
	LBM_CUDA(cudaStreamSynchronize(h->stream));
	*out = res[0];
	return LBM_OK;
}

int lbm_synchronize(lbm_handle h)
{
	if (int rc = check(h))
		return rc;
	LBM_CUDA(cudaStreamSynchronize(h->stream));
	LBM_CUDA(cudaStreamSynchronize(h->finish_stream));
	return LBM_OK;
}

int lbm_set_block(lbm_handle h, int bx, int by)
{
	if (int rc = check(h))
		return rc;
	if (bx == 0 && by == 0) {
		h->bx = h->by = 0;
	}
	else {
		if (bx < 32 || bx % 32 != 0 || by < 1 || bx * by > 128)
			return fail(LBM_ERR_INVALID, "block (%d, %d): bx must be a multiple of 32 and bx*by <= 128", bx, by);
		h->bx = bx;
		h->by = by;
	}
	h->drop_graph();
	return ensure_partials(h, h->max_step_blocks());
}

int lbm_get_block(lbm_handle h, int* bx, int* by)
{
	if (int rc = check(h))
		return rc;
	const dim3 b = h->block();
	if (bx)
		*bx = (int) b.x;
	if (by)
		*by = (int) b.y;
	return LBM_OK;
}

int lbm_autotune(lbm_handle h, int ntrials)
{
	if (int rc = check(h))
		return rc;
	if (!h->d.periodic && !h->map_set)
		return fail(LBM_ERR_INVALID, "lbm_set_map must be called before autotuning");
	if (ntrials < 2)
		ntrials = 2;
	ntrials += ntrials % 2;
	void* backup = nullptr;
	LBM_CUDA(cudaMalloc(&backup, h->pop_bytes));
	LBM_CUDA(cudaMemcpyAsync(backup, h->g.f, h->pop_bytes, cudaMemcpyDeviceToDevice, h->stream));
	const long long it0 = h->iteration;
	static const int cands[][2] = {{128, 1}, {64, 2}, {32, 4}, {64, 1}, {32, 2}};
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	float best = 1e30f;
	int bbx = 0, bby = 0;
	int best_kernel = lbm::KERNEL_DIRECT;
	const int obx = h->bx, oby = h->by;
	// the direct and the two-site kernel take the block shape
	const bool pair_ok = lbm::pair_step_of(h->d.storage) && h->streaming == LBM_STREAMING_AA;
	// a collision plugin runs its own one-site or two-site kernels: the tile
	// and split kernels are not candidates
	for (auto& c : cands) {
		if (c[0] > 32 && c[0] / 2 >= h->d.X)
			continue;  // far wider than the lattice
		h->bx = c[0];
		h->by = c[1];
		if (ensure_partials(h, h->max_step_blocks()))
			break;
		for (int k : {(int) lbm::KERNEL_DIRECT, (int) lbm::KERNEL_PAIR}) {
			if (k == lbm::KERNEL_PAIR && !pair_ok)
				continue;
			h->kernel = k;
			// warm-up pair, then timed steps
			launch_step(h, false, false);
			launch_step(h, false, false);
			cudaEventRecord(e0, h->stream);
			for (int s = 0; s < ntrials; s++)
				launch_step(h, false, false);
			cudaEventRecord(e1, h->stream);
			cudaEventSynchronize(e1);
			float ms = 0;
			cudaEventElapsedTime(&ms, e0, e1);
			if (ms < best) {
				best = ms;
				bbx = c[0];
				bby = c[1];
				best_kernel = k;
			}
		}
	}
	// the tile kernel and, with a map, the split step (the block shape does
	// not apply to them)
	for (int k : {(int) lbm::KERNEL_TILE, (int) lbm::KERNEL_SPLIT}) {
		if ((k == lbm::KERNEL_SPLIT && !h->split_tiles) || h->plugin)
			continue;
		h->kernel = k;
		launch_step(h, false, false);
		launch_step(h, false, false);
		cudaEventRecord(e0, h->stream);
		for (int s = 0; s < ntrials; s++)
			launch_step(h, false, false);
		cudaEventRecord(e1, h->stream);
		cudaEventSynchronize(e1);
		float ms = 0;
		cudaEventElapsedTime(&ms, e0, e1);
		if (ms < best) {
			best = ms;
			best_kernel = k;
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	h->iteration = it0;
	cudaMemcpyAsync(h->g.f, backup, h->pop_bytes, cudaMemcpyDeviceToDevice, h->stream);
	sync_ab_buffers(h);
	cudaStreamSynchronize(h->stream);
	cudaFree(backup);
	const cudaError_t err = cudaGetLastError();
	if (err != cudaSuccess) {
		h->bx = obx;
		h->by = oby;
		return fail(LBM_ERR_CUDA, "autotune failed: %s", cudaGetErrorString(err));
	}
	h->bx = bbx;
	h->by = bby;
	h->kernel = best_kernel;
	h->drop_graph();
	return ensure_partials(h, h->max_step_blocks());
}

int lbm_set_statistics(lbm_handle h, int enable)
{
	if (int rc = check(h))
		return rc;
	LBM_CUDA(cudaStreamSynchronize(h->stream));
	cudaFree(h->stats);
	h->stats = nullptr;
	h->stats_count = 0;
	if (enable) {
		const size_t bytes = (size_t) 9 * h->sites() * h->ops->compute_size;
		LBM_CUDA(cudaMalloc(&h->stats, bytes));
		LBM_CUDA(cudaMemsetAsync(h->stats, 0, bytes, h->stream));
		LBM_CUDA(cudaStreamSynchronize(h->stream));
	}
	return LBM_OK;
}

int lbm_get_statistics(lbm_handle h, double* out, int64_t* count)
{
	if (int rc = check(h))
		return rc;
	if (!h->stats)
		return fail(LBM_ERR_INVALID, "statistics are not enabled (lbm_set_statistics)");
	if (!out || !count)
		return fail(LBM_ERR_INVALID, "null output");
	const size_t n = (size_t) 9 * h->sites();
	const int cs = h->ops->compute_size;
	if (cs == 8) {
		LBM_CUDA(cudaMemcpyAsync(out, h->stats, n * 8, cudaMemcpyDeviceToHost, h->stream));
		LBM_CUDA(cudaStreamSynchronize(h->stream));
	}
	else {
		std::vector<float> tmp(n);
		LBM_CUDA(cudaMemcpyAsync(tmp.data(), h->stats, n * 4, cudaMemcpyDeviceToHost, h->stream));
		LBM_CUDA(cudaStreamSynchronize(h->stream));
		for (size_t i = 0; i < n; i++)
			out[i] = tmp[i];
	}
	*count = h->stats_count;
	return LBM_OK;
}

int lbm_set_streaming(lbm_handle h, int streaming)
{
	if (int rc = check(h))
		return rc;
	if (streaming != LBM_STREAMING_AA && streaming != LBM_STREAMING_AB)
		return fail(LBM_ERR_INVALID, "unknown streaming pattern %d", streaming);
	if (streaming == h->streaming)
		return LBM_OK;
	if (h->ade)
		return fail(LBM_ERR_UNSUPPORTED, "the coupled scalar runs on A-A lattices only (lbm_ade_disable first)");
	if (h->plugin)
		return fail(LBM_ERR_UNSUPPORTED, "a collision plugin runs with A-A streaming only");
	if (streaming == LBM_STREAMING_AA) {
		for (uint8_t g : h->map_host)
			if (!site_type_supported(g))
				return fail(LBM_ERR_UNSUPPORTED, "the map holds site type %d, which only the A-B pattern provides", (int) g);
		LBM_CUDA(cudaStreamSynchronize(h->stream));
		cudaFree(h->f_out);
		h->f_out = nullptr;
	}
	else {
		LBM_CUDA(cudaMalloc(&h->f_out, h->pop_bytes));
		LBM_CUDA(cudaMemcpyAsync(h->f_out, h->g.f, h->pop_bytes, cudaMemcpyDeviceToDevice, h->stream));
		LBM_CUDA(cudaStreamSynchronize(h->stream));
	}
	h->streaming = streaming;
	h->drop_graph();
	return LBM_OK;
}

int lbm_get_streaming(lbm_handle h, int* streaming)
{
	if (!h || !streaming)
		return fail(LBM_ERR_INVALID, "null argument");
	*streaming = h->streaming;
	return LBM_OK;
}

int lbm_set_kernel(lbm_handle h, int kernel)
{
	if (int rc = check(h))
		return rc;
	if (kernel != LBM_KERNEL_DIRECT && kernel != LBM_KERNEL_TILE && kernel != LBM_KERNEL_SPLIT && kernel != LBM_KERNEL_PAIR)
		return fail(LBM_ERR_INVALID, "unknown kernel %d", kernel);
	if (h->plugin && kernel != LBM_KERNEL_DIRECT && kernel != LBM_KERNEL_PAIR)
		return fail(LBM_ERR_UNSUPPORTED, "a collision plugin runs the one-site or the two-site kernel (LBM_KERNEL_DIRECT, LBM_KERNEL_PAIR)");
	h->kernel = kernel;
	h->drop_graph();
	return LBM_OK;
}

int lbm_get_kernel(lbm_handle h, int* kernel)
{
	if (int rc = check(h))
		return rc;
	if (!kernel)
		return fail(LBM_ERR_INVALID, "null output");
	*kernel = h->kernel;
	return LBM_OK;
}

int lbm_status(lbm_handle h, int* status)
{
	if (int rc = check(h))
		return rc;
	if (!status)
		return fail(LBM_ERR_INVALID, "null output");
	LBM_CUDA(cudaMemcpyAsync(status, h->status_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
	LBM_CUDA(cudaMemsetAsync(h->status_dev, 0, sizeof(int), h->stream));
	LBM_CUDA(cudaStreamSynchronize(h->stream));
	return LBM_OK;
}

int lbm_set_wait_limit(lbm_handle h, int64_t tries)
{
	if (int rc = check(h))
		return rc;
	h->wait_limit = tries < 0 ? -1 : tries;
	h->drop_graph();
	return LBM_OK;
}

int lbm_device_view_get(lbm_handle h, lbm_device_view* out)
{
	if (int rc = check(h))
		return rc;
	if (!out)
		return fail(LBM_ERR_INVALID, "null output");
	out->populations = h->g.f;
	out->sq = h->g.sq;
	out->sy = h->g.sy;
	out->sz = h->g.sz;
	out->x0 = h->g.x0;
	out->elem_size = h->ops->elem_size;
	out->macro = h->macro;
	out->macro_elem_size = h->ops->compute_size;
	out->stream = (void*) h->stream;
	return LBM_OK;
}

}  // extern "C"
