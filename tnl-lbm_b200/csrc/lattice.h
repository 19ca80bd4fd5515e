// Host-side state of one lattice handle (lbm_handle of the C-ABI), shared by
// the translation units that implement the C-ABI (lbm_abi.cu, lbm_adjoint.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tnl_lbm_b200.h"
#include "launch.h"

namespace lbm {
struct AdjointState;  // lbm_adjoint.cu
void adjoint_free(AdjointState*);

// coupled D3Q7 scalar (lbm_ade.cu)
struct AdeState
{
	AdeLaunch launch{};				// device buffers and parameters of the coupled step
	std::vector<uint8_t> map_host;	// host copy of the accepted ADE map
	void* phi_buf = nullptr;		// phi of the last observation step
	bool phi_valid = false;
	// two-site coupled step: group flags, rest-site list and work list,
	// rebuilt before the next pair step after either map changes
	uint8_t* pair_groups = nullptr;
	unsigned long long* pair_rest = nullptr;
	unsigned* pair_work = nullptr;
	bool pair_dirty = true;
};
int ade_build_pair(lbm_lattice* h);  // lbm_ade.cu
void ade_free(AdeState*);
}  // namespace lbm

struct lbm_lattice
{
	lbm_desc d{};
	const lbm::StorageOps* ops = nullptr;
	lbm::Geometry g{};
	size_t pop_bytes = 0;
	cudaStream_t stream = nullptr;
	uint8_t* map = nullptr;
	bool map_set = false;
	// inlet profiles.  Two device sets: the steps read the current one
	// (inflow[], a null component reads as zero); lbm_set_inflow uploads into
	// the other set on upload_stream, so that the copy overlaps the steps
	// still reading the current set, and makes it current
	void* inflow[3] = {nullptr, nullptr, nullptr};
	void* inflow_buf[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
	int inflow_cur = 0;
	cudaStream_t upload_stream = nullptr;
	cudaEvent_t inflow_ready = nullptr;						 // an upload has landed (upload_stream)
	cudaEvent_t inflow_free[2] = {nullptr, nullptr};		 // set b no longer read (recorded on stream)
	bool inflow_free_valid[2] = {false, false};
	void* inflow_host = nullptr;							 // pinned staging [2][3][Z Y], compute type
	cudaEvent_t inflow_staged[2] = {nullptr, nullptr};		 // staging slot b copied out (upload_stream)
	void* macro = nullptr;
	bool macro_valid = false;
	double* partials = nullptr;
	long long partials_cap = 0;	 // in blocks
	double* sums_host = nullptr;  // pinned [2][NRED]: the sums of the last two observation steps
	double* sums_mapped = nullptr;	// device address of sums_host (written by the finish kernel)
	cudaEvent_t sums_ev[2] = {nullptr, nullptr};  // recorded after each slot's finish kernel
	long long sums_iter[2] = {-1, -1};			  // iteration at which each slot's step ended
	int sums_last = 1;							  // slot of the last observation step
	unsigned* finish_arrived = nullptr;	 // [2] arrival counters of the finish kernel per slot, zero between launches
	// The finish kernel of sums slot s runs on finish_stream (highest
	// priority) after step_ev[s], the end of its observation step on stream,
	// so that the lattice's next step does not wait for it; sums_ev[s] then
	// marks the slot's sums ready.  Each slot has its own partials (partials
	// holds two slots).
	cudaStream_t finish_stream = nullptr;
	cudaEvent_t step_ev[2] = {nullptr, nullptr};
	bool sums_valid = false;
	long long iteration = 0;
	int bx = 0, by = 0;	 // 0: default
	int kernel = lbm::KERNEL_DIRECT;
	lbm_collision_launcher plugin = nullptr;  // a registered collision (desc.collision >= LBM_COLL_PLUGIN_FIRST)
	int sms = 148;
	int* status_dev = nullptr;	// STATUS_* bits set by the kernels
	long long wait_limit = -1;	// tile kernel's loop waits (lbm_set_wait_limit); negative: the default
	long long last_blocks = 0;	// partial-sum slots of the last step launch
	long long nothing_sites = 0;  // GEO_NOTHING sites of the map
	// the last step's partial sums leave out its GEO_NOTHING sites (each adds
	// rho = 1 and nothing else; the finish kernel adds them to the mass)
	bool last_nothing_skipped = false;
	lbm::CollParamsD p{};
	// CUDA graphs of GRAPH_STEPS plain steps starting at an even iteration,
	// for the population buffer and inlet profiles they were captured with
	// (two: the two inlet sets of alternating lbm_set_inflow calls)
	struct GraphSlot
	{
		cudaGraphExec_t exec = nullptr;
		const void* f = nullptr;
		const void* inflow[3] = {nullptr, nullptr, nullptr};
	};
	GraphSlot graphs[2];
	int graph_next = 0;	 // slot the next capture replaces
	std::vector<uint8_t> map_host;			 // host copy of the accepted map
	int streaming = LBM_STREAMING_AA;
	void* f_out = nullptr;		// A-B: the write buffer (swapped with g.f after every step)
	unsigned* split_tiles = nullptr;  // split step: fluid-only tiles, then the others
	long long split_n[2] = {0, 0};
	int split_tiles_x = 0;
	// pair step with a map ([0] plain steps, [1] observation steps): rest-site
	// lists, work lists (pair.cuh aa_pair_work_kernel) and the group flags
	unsigned long long* pair_rest[2] = {nullptr, nullptr};
	long long pair_nrest[2] = {0, 0};
	unsigned* pair_work[2] = {nullptr, nullptr};
	long long pair_nwork[2] = {0, 0};
	uint8_t* pair_groups = nullptr;  // PAIR_GROUP_* of every group of PAIR_GROUP sites
	void* stats = nullptr;		// D3Q27_MACRO_Mean fields [9][sites], compute type
	long long stats_count = 0;	// steps accumulated in stats
	lbm::AdjointState* adjoint = nullptr;	 // checkpoints of lbm_adjoint_forward
	lbm::AdeState* ade = nullptr;			 // coupled D3Q7 scalar, or null
	bool distributed_z = false;				 // a slab of a lattice split along z (lbm_set_distributed_z)
	cudaEvent_t halo_ev = nullptr;			 // ordering of halo copies against this lattice's stream
	static constexpr int GRAPH_STEPS = 16;

	long long sites() const
	{
		return (long long) d.X * d.Y * d.Z;
	}
	dim3 block() const
	{
		if (bx > 0)
			return dim3(bx, by, 1);
		const int bxd = d.X >= 128 ? 128 : ((d.X + 31) / 32) * 32;
		return dim3(bxd, 128 / bxd, 1);
	}
	dim3 grid() const
	{
		const dim3 b = block();
		return dim3((d.X + b.x - 1) / b.x, (d.Y + b.y - 1) / b.y, d.Z);
	}
	long long grid_blocks() const
	{
		const dim3 gr = grid();
		return (long long) gr.x * gr.y * gr.z;
	}
	// partial-sum slots any step kernel variant may need: one per block of the
	// persistent tile kernel, one per warp of the direct and A-B kernels
	long long max_step_blocks() const
	{
		const long long tile = (long long) lbm::TILE_MAX_BLOCKS_PER_SM * sms;
		const dim3 b = block();
		const long long direct = grid_blocks() * ((b.x * b.y) / 32);
		// pair step: the two-site grid's warps, or the work list's (4 per item)
		long long pairs = (long long) (((d.X + 1) / 2 + b.x - 1) / b.x) * ((d.Y + b.y - 1) / b.y) * d.Z * ((b.x * b.y) / 32);
		for (long long nw : pair_nwork)
			pairs = pairs > 4 * nw ? pairs : 4 * nw;
		const long long m = tile > direct ? tile : direct;
		return m > pairs ? m : pairs;
	}
	void drop_graph()
	{
		for (GraphSlot& g : graphs) {
			if (g.exec)
				cudaGraphExecDestroy(g.exec);
			g = GraphSlot{};
		}
		graph_next = 0;
	}
};

namespace lbm {
// message of lbm_last_error() for the calling thread (lbm_abi.cu)
int record_error(int code, const char* msg);
}  // namespace lbm
