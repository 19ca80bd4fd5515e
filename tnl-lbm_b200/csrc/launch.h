// Internal launch interface between the C-ABI (lbm_abi.cu) and the kernel
// instantiations, one translation unit per population storage format
// (aa_store_*.cu).  Arguments are type-erased here and converted to the
// storage's compute type inside each unit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lbm {

enum Storage : int
{
	ST_F64 = 0,
	ST_F32 = 1,
	ST_F32S = 2,
	ST_F16S = 3,
	ST_BF16S = 4,
	ST_F16SR = 5,
	ST_BF16SR = 6,
	ST_I16S = 7,
	ST_COUNT = 8
};

// collision-slot constants in double; each unit casts them to its compute type
struct CollParamsD
{
	double nu, fx, fy, fz;
	double w1, w3, w4, w5, A, B;
	double tau;
	int eq;
};

struct Geometry
{
	void* f;		  // population storage (element 0 of the allocation)
	long long sq;	  // slot stride in elements (one row: the slots of a lattice row lie side by side)
	int sy, sz, x0;	  // lattice-row stride, plane stride, interior x offset (elements)
	int X, Y, Z;
};

// initial state: mode 0 uniform (rho0, v0) everywhere; mode 1 device double
// [Z][Y][X] fields for the interior, uniform state in the ghost layer; mode 2
// Taylor-Green vortex of amplitude u0 around rho0 (ghost layer: rho0, 0)
struct InitSpec
{
	int mode;
	int eq;
	const double *rho, *vx, *vy, *vz;
	double rho0, vx0, vy0, vz0;
	double u0;
};

// work list of the pair step on a lattice with a map: items (pair tiles and
// rest chunks, pair.cuh) and the rest-site list the chunks index
struct PairWork
{
	const unsigned* work;
	long long nwork;
	const unsigned long long* rest;	 // row << 32 | x, row = z Y + y
	long long nrest;
};

struct StepLaunch
{
	Geometry g;
	const uint8_t* map;		   // null: periodic kernel
	const void* inflow[3];	   // compute-type [Z][Y] profiles or null
	void* macro;			   // compute-type [4][Z][Y][X] or null
	double* partials;		   // [blocks][NRED] or null
	CollParamsD p;
	int coll, cum_flags;
	bool odd;
	int kernel;		   // KERNEL_DIRECT, KERNEL_TILE, KERNEL_SPLIT or KERNEL_PAIR
	dim3 grid, block;  // direct kernel launch shape
	int* status;	   // device status word (STATUS_* bits)
	long long wait_limit;  // tries per mbarrier wait in the tile kernel's loop; negative: the default
	cudaStream_t stream;
	long long* blocks_out;	// partial-sum slots the launch writes (blocks or warps)
	bool dry_run;			// only resolve launch facts (attributes, grid), launch nothing
	void* f_out;			// A-B step: the output buffer (g.f is the input)
	// split step: tiles [0, split_n[0]) fluid-only, then split_n[1] others
	const unsigned* split_tiles;
	long long split_n[2];
	int split_tiles_x;
	const struct AdeLaunch* ade;  // coupled D3Q7 scalar (ade.cuh), or null
	bool distributed_z;			  // a slab: z neighbours through the ghost layer, no z wrap
	// pair step with a map: group flags, and the work lists of plain and of
	// observation steps (pair.cuh aa_pair_work_kernel)
	const uint8_t* pair_groups;	 // PAIR_GROUP_* per group of PAIR_GROUP sites of a row
	PairWork pair_work, pair_work_out;
	// set by a step whose partial sums leave out the GEO_NOTHING sites (a
	// sums-only step of the pair kernel over the plain work list), or null
	bool* nothing_skipped;
};

// the coupled D3Q7 advection-diffusion scalar of a lattice (ade.cuh)
struct AdeLaunch
{
	void* g;			  // compute-type populations: 7 slot rows per lattice row
	long long sq;		  // their geometry (rows as the flow lattice's, x0 alike)
	int sy, sz;
	const uint8_t* map;	  // ADE site types [Z][Y][X]
	const void* dcoef;	  // compute-type per-site diffusion coefficient, or null
	double D;			  // diffusion coefficient when dcoef is null
	double inflow_phi;
	void* phi;			  // compute-type [Z][Y][X] output of observation steps, or null
	int coll;			  // 0 SRT, 1 MRT, 2 central-moment (CLBM)
	// two-site coupled step (ade_pair.cuh): group flags and work list, or null
	const uint8_t* pair_groups;
	PairWork pair_work;
};

// two-site coupled flow + scalar step for FP32 storage (ade_pair.cuh);
// cudaErrorNotSupported where it does not apply
cudaError_t ade_pair_step_f32(const StepLaunch&);

// step kernel variants: one thread per site with direct loads, or the
// persistent bulk-copy pipeline of aa_tile.cuh
enum : int
{
	KERNEL_DIRECT = 0,
	KERNEL_TILE = 1,
	KERNEL_SPLIT = 3,
	KERNEL_PAIR = 4
};

// two-site step kernels (pair.cuh), one per storage with FP32 arithmetic;
// cudaErrorNotSupported for the collisions they do not cover
using PairStepFn = cudaError_t (*)(const StepLaunch&);
cudaError_t pair_step_f32(const StepLaunch&);
cudaError_t pair_step_f32s(const StepLaunch&);
cudaError_t pair_step_f16s(const StepLaunch&);
cudaError_t pair_step_f16sr(const StepLaunch&);
cudaError_t pair_step_bf16s(const StepLaunch&);
cudaError_t pair_step_bf16sr(const StepLaunch&);
cudaError_t pair_step_i16s(const StepLaunch&);
// upper bound of the tile kernel's grid (blocks per SM x SMs)
constexpr int TILE_MAX_BLOCKS_PER_SM = 8;

// one A-A step of an ensemble of periodic lattices (ensemble.cuh)
struct EnsLaunch
{
	const void* members;	 // device table of the storage's EnsMember entries
	const int* tile_member;	 // member of each tile
	long long ntiles;
	int tpb;		   // sites per tile = threads per block: 128 or 256
	bool pair;		   // two sites per thread (tpb = 256 sites on 128 threads, cumulant, FP32 arithmetic)
	long long grid;	   // blocks; 0 = resident blocks per SM x SMs (persistent)
	double* partials;  // [NRED][ntiles] or null
	int coll, cum_flags;
	bool odd;
	cudaStream_t stream;
	bool dry_run;
	long long* blocks_out;
};

struct StorageOps
{
	// one A-A step
	cudaError_t (*step)(const StepLaunch&);
	// equilibrium on every site incl. the ghost layer
	cudaError_t (*init_eq)(const Geometry&, const InitSpec&, cudaStream_t);
	// convert between storage and a dense buffer [27][nz][ny][nx] of double
	// (dtype 0) or float (dtype 1); ghost = 1 includes the ghost layer
	cudaError_t (*pack)(const Geometry&, void* dense, int dtype, int ghost, cudaStream_t);
	cudaError_t (*unpack)(const Geometry&, const void* dense, int dtype, int ghost, cudaStream_t);
	// one A-B step (ab_kernels.cuh) from L.g.f into L.f_out
	cudaError_t (*ab_step)(const StepLaunch&);
	// ensemble: bytes of one member-table entry, host-side fill of an entry,
	// and the step
	size_t ens_entry_bytes;
	void (*ens_entry)(void* dst, const Geometry&, const CollParamsD&, long long tile0);
	cudaError_t (*ens_step)(const EnsLaunch&);
	// one coupled flow + D3Q7 scalar step (L.ade set); cudaErrorNotSupported
	// for storages whose element is not the compute type
	cudaError_t (*ade_step)(const StepLaunch&);
	int compute_size;  // sizeof the compute type (8 or 4)
	int elem_size;	   // sizeof the storage element
	const char* name;
};

const StorageOps& storage_ops(int storage);

// FP64 reductions shared by all storages (lbm_reduce.cu)
constexpr int NRED_HOST = 6;
// partials are stored as [NRED][nslots]; stage is scratch of
// finish_scratch_doubles() doubles; arrived is a device counter that holds
// zero between launches (one per stream that runs finish_sums); out may be
// device or mapped host memory
long long finish_scratch_doubles();
// mass_offset is added to the summed mass (sites left out of the partials
// that each contribute a known density)
cudaError_t finish_sums(const double* partials, long long nslots, double* stage, unsigned* arrived, double* out,
						cudaStream_t, double mass_offset = 0.0);
// enstrophy-type sum rho * |grad u|^2 with central differences over the macro
// field (compute type given by compute_size), periodic wrap as sim_4.cu:21-54
cudaError_t enstrophy_partials(const void* macro, int compute_size, int X, int Y, int Z, double* partials, long long* nblocks,
							   cudaStream_t);

// running velocity statistics of D3Q27_MACRO_Mean from the macro field of one
// step: stats [9][n] in the compute type (lbm_stats.cu)
cudaError_t stats_update(const void* macro, void* stats, int compute_size, long long n, int counter, cudaStream_t);

}  // namespace lbm
