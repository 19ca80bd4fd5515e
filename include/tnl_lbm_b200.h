/*
 * tnl_lbm_b200.h -- C-ABI of the B200-native D3Q27 A-A hot path.
 *
 * This is the drop-in boundary for TNL-LBM's per-step update: the fused
 * collision + A-A streaming kernel with the COLL / BC / MACRO plugins of
 * LBM_CONFIG (include/lbm3d/defs.h:288-310, include/lbm3d/kernels.h:59-112)
 * and the host-side pieces of the time loop that drive it.  Plain C types
 * only: sizes, host pointers, device pointers as void*.  Every entry point
 * returns an int status (LBM_OK = 0); lbm_last_error() describes the last
 * failure of the calling thread.  A handle owns one lattice on one GPU with
 * its own CUDA stream; calls on one handle are not thread-safe.
 *
 * Population slot order (q = 0..26) is the reference's direction enum
 * (include/lbm3d/defs.h:318-350); map values are the GEO enum of
 * D3Q27_BC_All (include/lbm3d/d3q27/bc.h:17-43).  Arrays exchanged with the
 * host are dense, C order, x fastest:
 *   populations  [27][Z][Y][X]       (LBM_LAYOUT_INTERIOR)
 *                [27][Z+2][Y+2][X+2] (LBM_LAYOUT_GHOST: incl. the ghost layer)
 *   map          [Z][Y][X] uint8
 *   macro        [4][Z][Y][X] double (rho, vx, vy, vz)
 *   inflow       [Z][Y] double per velocity component
 */
#ifndef TNL_LBM_B200_H
#define TNL_LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LBM_API __attribute__((visibility("default")))
#else
#define LBM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbm_lattice* lbm_handle;

/* status codes */
#define LBM_OK 0
#define LBM_ERR_INVALID 1     /* bad argument or handle */
#define LBM_ERR_UNSUPPORTED 2 /* combination not provided (e.g. a site type) */
#define LBM_ERR_CUDA 3        /* CUDA runtime error */
#define LBM_ERR_NONFINITE 4   /* non-finite density detected by a reduction */
#define LBM_ERR_SIZE 5        /* size beyond a documented maximum */

/* population storage in HBM */
#define LBM_STORE_F64 0   /* double f_q */
#define LBM_STORE_F32 1   /* float f_q */
#define LBM_STORE_F32S 2  /* float f_q - w_q (shifted) */
#define LBM_STORE_F16S 3  /* half (f_q - w_q) * 2^k_q, 2^k_q >= 1/w_q; FP32 arithmetic */
#define LBM_STORE_BF16S 4 /* bfloat16 f_q - w_q; FP32 arithmetic */
#define LBM_STORE_F16SR 5  /* as LBM_STORE_F16S, stochastic rounding on store */
#define LBM_STORE_BF16SR 6 /* as LBM_STORE_BF16S, stochastic rounding on store */
#define LBM_STORE_I16S 7   /* int16 round((f_q - w_q) / q_q), q_q a power of two with
                              32767 q_q = 0.42 w_q: fixed point over |f_q - w_q| <= 0.42 w_q
                              (clamped beyond); FP32 arithmetic */

/* collision slot (COLL of LBM_CONFIG) */
#define LBM_COLL_CUM 0 /* D3Q27_CUM, include/lbm3d/d3q27/col_cum.h */
#define LBM_COLL_SRT 1 /* D3Q27_SRT, col_srt.h */
#define LBM_COLL_BGK 2 /* D3Q27_BGK, col_bgk.h */
#define LBM_COLL_MRT 3 /* D3Q27_MRT (MRT-LES), col_mrt.h */
/* ids of user-compiled collisions (lbm_register_collision) */
#define LBM_COLL_PLUGIN_FIRST 16
#define LBM_COLL_PLUGIN_LAST 31

/* cumulant variant bits (USE_GEIER_CUM_2017, USE_GEIER_CUM_ANTIALIAS; defs.h:312-315).
 * Valid sets: 0, ANTIALIAS, 2017|ANTIALIAS. */
#define LBM_CUM_GEIER_2017 1
#define LBM_CUM_ANTIALIAS 2

/* equilibrium (EQ of LBM_CONFIG) */
#define LBM_EQ_SECOND_ORDER 0 /* D3Q27_EQ, eq.h */
#define LBM_EQ_INV_CUM 1      /* D3Q27_EQ_INV_CUM, eq_inv_cum.h */

#define LBM_LAYOUT_INTERIOR 0
#define LBM_LAYOUT_GHOST 1
#define LBM_DTYPE_F64 0
#define LBM_DTYPE_F32 1

/* lbm_step flags: what the last of the requested steps also produces */
#define LBM_STEP_MACRO 1  /* store rho, u (D3Q27_MACRO_Default::outputMacro, macro.h:70-76) */
#define LBM_STEP_SUMS 2   /* FP64 sums of rho, rho*u, rho*|u|^2 and a non-finite count */

typedef struct lbm_desc {
	int32_t X, Y, Z;      /* lattice sites per axis (without the ghost layer) */
	int32_t storage;      /* LBM_STORE_* */
	int32_t collision;    /* LBM_COLL_* */
	int32_t cum_flags;    /* LBM_CUM_* bits, cumulant only */
	int32_t equilibrium;  /* LBM_EQ_*: SRT collision and equilibrium BCs */
	int32_t periodic;     /* 1: every site GEO_PERIODIC and no map is used */
	double viscosity;     /* lattice viscosity nu (LBM_Data::lbmViscosity) */
	double fx, fy, fz;    /* homogeneous body force (NSE_Data::fx..fz, lbm_data.h:65-73) */
	int32_t device;       /* CUDA device ordinal */
	int32_t use_graphs;   /* 1: replay the time loop from captured CUDA graphs */
} lbm_desc;

/* Allocate a lattice (populations incl. a one-site ghost layer, map, macro).
 * Replaces LBM_BLOCK::allocateDeviceData (include/lbm3d/lbm_block.hpp:549-617)
 * together with the LBM_CONFIG composition (defs.h:288-310). */
LBM_API int lbm_create(const lbm_desc* desc, lbm_handle* out);

/* Release everything the handle owns. */
LBM_API int lbm_destroy(lbm_handle h);

/* Message of the last failed call on this thread (never NULL). */
LBM_API const char* lbm_last_error(void);

/* Per-site GEO types, host [Z][Y][X] uint8; required unless desc.periodic.
 * Replaces LBM_BLOCK map setup + copyMapToDevice (lbm_block.hpp, state.hpp:1151-1232).
 * Supported: GEO_FLUID, WALL, INFLOW, INFLOW_LEFT, INFLOW_EQ_LEFT, OUTFLOW_EQ,
 * PERIODIC, NOTHING, SYM_TOP..SYM_FRONT, and with LBM_STREAMING_AB also
 * INFLOW_BB_LEFT, OUTFLOW_RIGHT, OUTFLOW_RIGHT_INTERP.  Returns
 * LBM_ERR_UNSUPPORTED for those three under A-A (their A-A update depends on
 * the order in which sites run) and for the adjoint types. */
LBM_API int lbm_set_map(lbm_handle h, const uint8_t* map);

/* The map last set (by lbm_set_map or lbm_checkpoint_load), host [Z][Y][X];
 * LBM_ERR_INVALID on a periodic lattice or before a map was set.  Replaces
 * copyMapToHost (include/lbm3d/lbm.h:66). */
LBM_API int lbm_get_map(lbm_handle h, uint8_t* map);

/* Inlet velocity profiles, host [Z][Y] doubles; NULL means zero.  The
 * values are copied before the call returns (the caller may reuse its
 * buffers); the upload to the device overlaps the steps already enqueued,
 * and every step enqueued after the call sees the new profiles.
 * Replaces NSE_Data_InflowProfile (include/lbm3d/lbm_data.h:95-133). */
LBM_API int lbm_set_inflow(lbm_handle h, const double* vx, const double* vy, const double* vz);

/* Change the lattice viscosity (State::updateKernelData, state.hpp:1627-1634). */
LBM_API int lbm_set_viscosity(lbm_handle h, double nu);

/* Equilibrium populations on every site incl. the ghost layer.  rho, vx, vy,
 * vz: host [Z][Y][X] fields for the interior, or all NULL for the uniform
 * state (rho0, v0), which also fills the ghost layer.
 * Replaces LBM_BLOCK::setEquilibrium (lbm_block.hpp:248-278) and the
 * setEquilibriumLat initialisers (common.h:127-158, sim_4.cu:126-171). */
LBM_API int lbm_init_equilibrium(lbm_handle h, const double* rho, const double* vx, const double* vy, const double* vz,
                         double rho0, double vx0, double vy0, double vz0);

/* Taylor-Green vortex of sim_NSE/sim_4.cu:145-163 in lattice units:
 * u = u0 sin(kx) cos(ky) cos(kz), v = -u0 (kx/ky) cos(kx) sin(ky) cos(kz), w = 0,
 * rho = rho0 + 3 (u0^2/16) (cos 2kx + cos 2ky)(cos 2kz + 2) with k = 2 pi / N per
 * axis at cell centres (i + 1/2 - N/2); the ghost layer gets (rho0, 0). */
LBM_API int lbm_init_taylor_green(lbm_handle h, double u0, double rho0);

/* Copy populations in / out (dtype LBM_DTYPE_*, layout LBM_LAYOUT_*).
 * Values are f_q in slot order at the current A-A parity (after an odd number
 * of steps the slots hold the streamed, swapped state of streaming_AA.h). */
LBM_API int lbm_set_populations(lbm_handle h, const void* host, int layout, int dtype);
LBM_API int lbm_get_populations(lbm_handle h, void* host, int layout, int dtype);

/* Advance nsteps A-A steps (State::SimUpdate + LBM::updateKernelData,
 * state.hpp:1235-1314, lbm.hpp:307-323).  The even/odd parity follows the
 * handle's iteration counter.  flags (LBM_STEP_*) apply to the last step. */
LBM_API int lbm_step(lbm_handle h, int64_t nsteps, int flags);

/* Iteration counter (LBM::iterations); setting it changes the A-A parity. */
LBM_API int64_t lbm_iteration(lbm_handle h);
LBM_API int lbm_set_iteration(lbm_handle h, int64_t iteration);

/* Macro field of the last step run with LBM_STEP_MACRO, host [4][Z][Y][X]. */
LBM_API int lbm_get_macro(lbm_handle h, double* host);

/* Sums of the last step run with LBM_STEP_SUMS: out[6] = {sum rho, sum rho vx,
 * sum rho vy, sum rho vz, sum rho |u|^2, non-finite count}, accumulated in
 * FP64 (GEO_NOTHING sites count as rho = 1, u = 0).  Returns
 * LBM_ERR_NONFINITE when the count is non-zero (state.hpp:1469-1492).  The
 * last stage of the reduction runs on a stream of the library's own, so the
 * lattice's next step does not wait for it; lbm_get_sums, lbm_get_sums_of
 * and lbm_synchronize wait for it. */
LBM_API int lbm_get_sums(lbm_handle h, double* out);
/* The sums of the observation step (LBM_STEP_SUMS) that ended at `iteration`;
 * the last two observation steps are kept.  Waits for that step alone, not
 * for work enqueued after it, so a caller can enqueue step n+1 before reading
 * the result of step n.  LBM_ERR_INVALID when that step is no longer kept. */
LBM_API int lbm_get_sums_of(lbm_handle h, int64_t iteration, double* out);

/* sum rho |grad u|^2 over the macro field of the last LBM_STEP_MACRO step with
 * periodic central differences (sim_4.cu:21-54, :279-298). */
LBM_API int lbm_enstrophy_sum(lbm_handle h, double* out);

/* Wait for all work of the handle (its stream and its reduction stream). */
LBM_API int lbm_synchronize(lbm_handle h);

/* Thread-block shape of the step kernels; (0,0) restores the default. */
LBM_API int lbm_set_block(lbm_handle h, int bx, int by);
LBM_API int lbm_get_block(lbm_handle h, int* bx, int* by);

/* Time candidate block shapes on the current state (which is restored) and
 * keep the fastest; ntrials steps per candidate.  Replaces the heuristic of
 * get_optimal_block_size (include/lbm3d/block_size_optimizer.h:18-111). */
LBM_API int lbm_autotune(lbm_handle h, int ntrials);

/* Step kernel: LBM_KERNEL_DIRECT (default) is one thread per site with
 * direct coalesced loads and stores; LBM_KERNEL_TILE is a persistent kernel
 * that streams population rows into shared memory with bulk copies.  Both
 * compute the same update, bit for bit. */
#define LBM_KERNEL_DIRECT 0
#define LBM_KERNEL_TILE 1
#define LBM_KERNEL_SPLIT 3 /* lattices with a map: one launch over the tiles of 128
                              x-sites that hold only GEO_FLUID (no map read, no
                              boundary branch), one over the others */
#define LBM_KERNEL_PAIR 4  /* two x-adjacent sites per thread, the collision of both
                              on the packed FP32 (f32x2) instructions; storages with
                              FP32 arithmetic and the built-in collisions (FP64
                              storage runs LBM_KERNEL_DIRECT).  Same update as the
                              direct kernel up to the rounding of the fused
                              multiply-adds. */
LBM_API int lbm_set_kernel(lbm_handle h, int kernel);
LBM_API int lbm_get_kernel(lbm_handle h, int* kernel);

/* Streaming pattern (STREAMING of LBM_CONFIG).  LBM_STREAMING_AA (default):
 * in place, one buffer, streaming_AA.h.  LBM_STREAMING_AB: the pull scheme of
 * streaming_AB.h with a second population buffer, swapped after every step
 * (lbm.hpp:314-322); boundary sites read clamped neighbours as a single
 * block does (kernels.h:48-55), and the map may also hold GEO_INFLOW_BB_LEFT,
 * GEO_OUTFLOW_RIGHT and GEO_OUTFLOW_RIGHT_INTERP.  Switching to A-B copies the
 * current populations into the second buffer; switching back is refused
 * while the map holds one of those three types.  The discrete adjoint
 * (lbm_adjoint_*) runs on A-A lattices only. */
#define LBM_STREAMING_AA 0
#define LBM_STREAMING_AB 1
LBM_API int lbm_set_streaming(lbm_handle h, int streaming);
LBM_API int lbm_get_streaming(lbm_handle h, int* streaming);

/* Running velocity statistics of D3Q27_MACRO_Mean (macro.h:89-180).  While
 * enabled, every step also outputs the macro field and updates, per site, the
 * mean velocity m (moving average) and the co-moments S_ab of the online
 * covariance, Cov(a, b) = S_ab / count.  lbm_set_statistics(h, 1) allocates
 * and zeroes 9 fields of the compute type (count = 0), 0 frees them.
 * lbm_get_statistics: out[9][Z][Y][X] = m_x, m_y, m_z, S_xx, S_yy, S_zz,
 * S_xy, S_xz, S_yz, and the number of accumulated steps. */
LBM_API int lbm_set_statistics(lbm_handle h, int enable);
LBM_API int lbm_get_statistics(lbm_handle h, double* out, int64_t* count);

/* Checkpoint / resume (the reference's State::saveState / loadState through
 * ADIOS2, include/lbm3d/state.hpp:891-1012).  One binary file: the lattice
 * description, the iteration counter (A-A parity), the streaming pattern,
 * the map, the inlet profiles and the population buffer as stored on the
 * device, so a resumed run continues bit for bit.  lbm_checkpoint_load needs
 * a handle created with the same sizes, storage, collision slot, equilibrium,
 * periodicity and body force; it restores the viscosity. */
LBM_API int lbm_checkpoint_save(lbm_handle h, const char* path);
LBM_API int lbm_checkpoint_load(lbm_handle h, const char* path);

/* Device status word: bit LBM_STATUS_TIMEOUT is set when a bounded wait inside
 * a kernel gave up (the kernel then stops early; the step's result is invalid).
 * Waits for the handle's work, returns the word and clears it.  The reference
 * has no status word (CUDA errors throw, TNL_BACKEND_SAFE_CALL in
 * lbm_block.hpp:132); this replaces its terminate flag (state.hpp:1486-1491)
 * for failures inside a step. */
#define LBM_STATUS_TIMEOUT 1
LBM_API int lbm_status(lbm_handle h, int* status);
/* Bound of the tile kernel's (LBM_KERNEL_TILE) per-tile mbarrier waits, in
 * tries; a negative value restores the default (about seconds).  With 0 the
 * waits give up at once while the tile's bulk copies are still in flight:
 * the step stops early, sets LBM_STATUS_TIMEOUT and still waits (with the
 * default bound) for every copy it issued, so tests can drive the timeout
 * path without a fault.  No counterpart in the reference. */
LBM_API int lbm_set_wait_limit(lbm_handle h, int64_t tries);

/* Device view for zero-copy interop (pytnl_lbm): the population base pointer
 * and strides in elements: index(q,x,y,z) = q*sq + (z+1)*sz + (y+1)*sy + x0 + x. */
typedef struct lbm_device_view {
	void* populations;
	int64_t sq;
	int32_t sy, sz, x0;
	int32_t elem_size;
	void* macro;        /* compute type [4][Z][Y][X] */
	int32_t macro_elem_size;
	void* stream;       /* cudaStream_t of the handle */
} lbm_device_view;
LBM_API int lbm_device_view_get(lbm_handle h, lbm_device_view* out);

/* Allocation-free FP64 sums of a macro field, for callers that cannot
 * allocate device memory where they need the result: an application whose
 * own pool allocator owns the device memory and forbids libraries to
 * allocate beside it, or a real-time loop that must not take an
 * allocation's implicit synchronisation.  No counterpart in the reference.
 *   macro   device pointer to a field [4][nsites] (rho, vx, vy, vz) of
 *           LBM_DTYPE_F64 or LBM_DTYPE_F32 values, e.g. a lattice's macro
 *           field from lbm_device_view_get
 *   out     device pointer to 6 doubles: the sums of lbm_get_sums
 *   stream  cudaStream_t (NULL: the default stream); the call is asynchronous
 * The partial sums live in a file-scope device array of
 * LBM_NOALLOC_SCRATCH_DOUBLES doubles (96 KiB per GPU that loads the library,
 * kept until the process exits).  The call allocates nothing.  Its first
 * call on a device resolves the array's device address (cudaGetSymbolAddress)
 * and loads its reduction kernels, so make that first call before any stream
 * capture; the address is kept for the life of the process, so do not call
 * it again after a cudaDeviceReset.  The race is per device: calls on
 * different GPUs may overlap, while calls on one GPU share its array, and
 * calls that overlap there (other streams, other host threads) race and must
 * be serialised.  nsites above LBM_NOALLOC_MAX_SITES returns LBM_ERR_SIZE. */
#define LBM_NOALLOC_MAX_BLOCKS 2048
#define LBM_NOALLOC_SCRATCH_DOUBLES (6 * LBM_NOALLOC_MAX_BLOCKS)
#define LBM_NOALLOC_MAX_SITES ((int64_t) 1 << 40)
LBM_API int lbm_macro_sums_noalloc(const void* macro, int dtype, int64_t nsites, double* out, void* stream);

/* ---- Ensembles of periodic lattices ------------------------------------
 * Many independent periodic lattices of different sizes and viscosities,
 * advanced by one persistent launch per A-A step (captured in CUDA graphs).
 * The reference has no ensemble driver: a TNL-LBM user runs one solver
 * instance (State / LBM_BLOCK, include/lbm3d/state.h, lbm_block.h) per
 * lattice, one after the other.  Each member's update equals, bit for bit,
 * that of a single periodic lattice (lbm_create with periodic = 1) with the
 * same size, viscosity and initial state.  Members share the storage format,
 * collision slot and equilibrium. */
typedef struct lbm_ensemble_desc {
	int32_t count;            /* members, 1 .. LBM_ENSEMBLE_MAX_MEMBERS */
	const int32_t* X;         /* [count] sites per axis of each member (X*Y*Z < 2^31) */
	const int32_t* Y;
	const int32_t* Z;
	const double* viscosity;  /* [count] lattice viscosity of each member */
	int32_t storage, collision, cum_flags, equilibrium; /* as lbm_desc */
	int32_t device;
	int32_t use_graphs;
} lbm_ensemble_desc;
#define LBM_ENSEMBLE_MAX_MEMBERS 65536
typedef struct lbm_ensemble_t* lbm_ensemble;

LBM_API int lbm_ensemble_create(const lbm_ensemble_desc* desc, lbm_ensemble* out);
LBM_API int lbm_ensemble_destroy(lbm_ensemble e);
/* Taylor-Green vortex in every member (each in its own box, as
 * lbm_init_taylor_green), or a uniform equilibrium; iteration reset to 0. */
LBM_API int lbm_ensemble_init_taylor_green(lbm_ensemble e, double u0, double rho0);
LBM_API int lbm_ensemble_init_equilibrium(lbm_ensemble e, double rho0, double vx0, double vy0, double vz0);
/* populations of one member, layouts and dtypes as lbm_set_populations */
LBM_API int lbm_ensemble_set_populations(lbm_ensemble e, int member, const void* host, int layout, int dtype);
LBM_API int lbm_ensemble_get_populations(lbm_ensemble e, int member, void* host, int layout, int dtype);
/* nsteps A-A steps of every member; LBM_STEP_SUMS computes per-member sums
 * in the last step (lbm_ensemble_get_sums). */
LBM_API int lbm_ensemble_step(lbm_ensemble e, int64_t nsteps, int flags);
/* out[count][6]: the sums of lbm_get_sums for each member */
LBM_API int lbm_ensemble_get_sums(lbm_ensemble e, double* out);
LBM_API int64_t lbm_ensemble_iteration(lbm_ensemble e);
/* the ensemble's CUDA stream (cudaStream_t), for events and interop */
LBM_API int lbm_ensemble_get_stream(lbm_ensemble e, void** stream);
LBM_API int lbm_ensemble_synchronize(lbm_ensemble e);
/* Launch shape: sites per tile (= threads per block) 128 or 256, and grid
 * 0 (persistent: resident blocks per SM x SMs), 1 (one block per tile), or
 * 2 (every member runs the single-lattice kernel on one of up to 64 streams,
 * the members being independent branches of the captured graph; steps with
 * LBM_STEP_SUMS use the persistent kernel), or 3 (persistent, two x-adjacent
 * sites per thread on packed FP32 arithmetic; tile_sites 256, an
 * FP32-arithmetic storage and members of even width, else
 * LBM_ERR_UNSUPPORTED). */
LBM_API int lbm_ensemble_set_shape(lbm_ensemble e, int tile_sites, int grid_policy);
LBM_API int lbm_ensemble_get_shape(lbm_ensemble e, int* tile_sites, int* grid_policy);
/* Times every launch shape on the current state (restored afterwards) and
 * keeps the fastest. */
LBM_API int lbm_ensemble_autotune(lbm_ensemble e, int ntrials);

/* ---- Discrete adjoint (SRT collision, per-site body force as the control) --
 * Gradient of an objective on the state after nsteps A-A steps with respect
 * to a per-site body force field F [3][Z][Y][X] and to the initial population
 * array.  The objective is J = sum_i 1/2 [rho_weight (rho_i - rho*_i)^2 +
 * |u_i - u*_i|^2] over sample sites i (site index (z*Y + y)*X + x, distinct
 * fluid sites), with rho and u the moments the next step would compute at
 * the final state and target[i] = {rho*, u*x, u*y, u*z}.  The time loop is
 * differentiated exactly (discrete adjoint), with checkpoints every
 * checkpoint_every steps (<= 0: ceil(sqrt(nsteps))) and recomputation; the
 * force gradient is accumulated in FP64.
 * Requirements: LBM_COLL_SRT with LBM_EQ_SECOND_ORDER, LBM_STORE_F64 or
 * LBM_STORE_F32, site types FLUID, WALL, INFLOW, OUTFLOW_EQ, PERIODIC,
 * NOTHING, SYM_*.  The reference's sim_adjoint (sim_adjoint/sim_adjoint.cu)
 * solves a steady adjoint about a frozen flow with D3Q27_SRT_ADJOINT
 * (col_srt_adjoint.h); the transpose applied here at each site reduces to
 * that adjoint collision at rho = 1 and F = 0.
 * lbm_adjoint_forward starts from the current populations and iteration,
 * advances the lattice by nsteps (force NULL: the descriptor's uniform
 * force) and returns the objective.  lbm_adjoint_backward returns seed * dJ/dF
 * ([3][Z][Y][X] doubles, or NULL) and seed * dJ/d(initial populations)
 * (layout and dtype as lbm_get_populations, or NULL).  force, grad_force and
 * grad_populations may point to host or device memory (unified addressing).
 * The adjoint populations are FP64 whatever the storage: with LBM_STORE_F32
 * the primal runs in FP32 and its transpose is evaluated and accumulated in
 * FP64 at the FP32 primal's values.
 * lbm_adjoint_release frees the checkpoints. */
LBM_API int lbm_adjoint_forward(lbm_handle h, const double* force, int64_t nsteps, int64_t checkpoint_every,
                                const int64_t* samples, int32_t nsamples, const double* target, double rho_weight,
                                double* loss);
LBM_API int lbm_adjoint_backward(lbm_handle h, double seed, double* grad_force, void* grad_populations, int layout,
                                 int dtype);
LBM_API int lbm_adjoint_release(lbm_handle h);

/* Library build information: sm architecture and version string. */
/* Coupled D3Q7 advection-diffusion scalar (State_NSE_ADE with the coupled
 * kernel of include/lbm3d/kernels.h:114-196).  Once enabled, every lbm_step
 * also advances the scalar phi with the flow site's velocity, in the same
 * kernel: the seven scalar populations use the A-A pattern and the flow
 * lattice's neighbour indices.  Collisions (include/lbm3d/d3q7/): SRT, MRT
 * and the central-moment CLBM, omega = 1 / (1/2 + 4 D).  Scalar site types
 * (d3q7/bc.h:17-36, values LBM_ADE_GEO_*): FLUID, WALL, WALL_BODY, SOLID,
 * INFLOW (phi = inflow_phi, ADE_Data_ConstInflow), PERIODIC, NOTHING and
 * SYM_TOP..SYM_FRONT; the outflow and phase-transfer types are refused
 * (their A-A update depends on the order of the sites).  Provided for FP64,
 * FP32 and F32S storage on A-A lattices; the adjoint and checkpoints refuse a
 * lattice with a scalar. */
#define LBM_ADE_SRT 0
#define LBM_ADE_MRT 1
#define LBM_ADE_CLBM 2
#define LBM_ADE_GEO_FLUID 0
#define LBM_ADE_GEO_WALL 1
#define LBM_ADE_GEO_WALL_BODY 2
#define LBM_ADE_GEO_SOLID 3
#define LBM_ADE_GEO_INFLOW 7
#define LBM_ADE_GEO_PERIODIC 9
#define LBM_ADE_GEO_NOTHING 10
#define LBM_ADE_GEO_SYM_TOP 12
#define LBM_ADE_GEO_SYM_BOTTOM 13
#define LBM_ADE_GEO_SYM_LEFT 14
#define LBM_ADE_GEO_SYM_RIGHT 15
#define LBM_ADE_GEO_SYM_BACK 16
#define LBM_ADE_GEO_SYM_FRONT 17

typedef struct lbm_ade_desc
{
	int32_t collision;	/* LBM_ADE_SRT, LBM_ADE_MRT or LBM_ADE_CLBM */
	double diffusion;	/* lattice diffusion coefficient (ADE lbmViscosity) */
	double inflow_phi;	/* phi imposed at LBM_ADE_GEO_INFLOW sites */
} lbm_ade_desc;

/* Allocate the scalar (all sites LBM_ADE_GEO_FLUID, populations zero). */
LBM_API int lbm_ade_enable(lbm_handle h, const lbm_ade_desc* desc);
LBM_API int lbm_ade_disable(lbm_handle h);
/* Scalar site types, host [Z][Y][X]. */
LBM_API int lbm_ade_set_map(lbm_handle h, const uint8_t* map);
/* Per-site diffusion coefficient, host [Z][Y][X] doubles (the
 * diffusion_coefficient_ptr of ADE_Data, lbm_data.h:219-239); NULL returns
 * to the descriptor's constant. */
LBM_API int lbm_ade_set_diffusion(lbm_handle h, const double* field);
/* Equilibrium of phi (host [Z][Y][X] or NULL for uniform_phi) with the given
 * velocity (NULL for zero) on every site; ghost sites take the nearest
 * lattice site's values (setEquilibriumLat, d3q7/common.h:51-61). */
LBM_API int lbm_ade_init_equilibrium(lbm_handle h, const double* phi, const double* vx, const double* vy,
									 const double* vz, double uniform_phi);
/* Scalar populations, host [7][Z(+2)][Y(+2)][X(+2)] in the layouts and
 * dtypes of lbm_set_populations. */
LBM_API int lbm_ade_set_populations(lbm_handle h, const void* host, int layout, int dtype);
LBM_API int lbm_ade_get_populations(lbm_handle h, void* host, int layout, int dtype);
/* phi [Z][Y][X] of the last lbm_step with LBM_STEP_MACRO (outputMacro of
 * D3Q7_MACRO_Default, d3q7/macro.h:33-37). */
LBM_API int lbm_ade_get_phi(lbm_handle h, double* host);

/* Slabs of a lattice split along z (the reference's MPI decomposition,
 * include/lbm3d/lattice_decomposition.h:16-55, lbm.hpp:189-273, on GPUs).
 * A slab is a lattice of the slab's z extent marked distributed along z: its
 * periodic sites do not wrap in z but reach their z neighbours through the
 * ghost layer (kernelInitIndices with distributed.z(), kernels.h:21-37).
 * Under the A-A pattern only odd steps cross a z face, and only the nine
 * slots whose c_z points across it.  Per interface (lower slab L of Zl layers,
 * upper slab U), before every odd step:
 *   U plane -1 <- L plane Zl-1, slots c_z = -1;  L plane Zl <- U plane 0, slots c_z = +1
 * and after it:
 *   L plane Zl-1 <- U plane -1, slots c_z = -1;  U plane 0 <- L plane Zl, slots c_z = +1
 * Planes are indexed in the ghost frame (z = -1 and z = Z are ghost planes).
 * lbm_halo_copy moves the planes between two handles of one process (peer
 * loads between GPUs), ordered after the sender's and before the receiver's
 * later work; lbm_halo_pack / lbm_halo_unpack stage them in a device buffer of
 * lbm_halo_bytes bytes on the handle's stream, for a transport between
 * processes.  A-A only; not with a coupled scalar. */
LBM_API int lbm_set_distributed_z(lbm_handle h, int distributed);
LBM_API int64_t lbm_halo_bytes(lbm_handle h);
LBM_API int lbm_halo_pack(lbm_handle h, int z, int cz, void* dev_buf);
LBM_API int lbm_halo_unpack(lbm_handle h, int z, int cz, const void* dev_buf);
LBM_API int lbm_halo_copy(lbm_handle dst, int dst_z, lbm_handle src, int src_z, int cz);

/* ---- Collision plugins (the open COLL slot of LBM_CONFIG) ---------------
 * The reference composes a user's collision struct into its step kernel at
 * compile time: LBM_CONFIG<..., COLL, ...> (defs.h:288-310) calls
 * COLL::collision(KS) on the D3Q27_KernelStruct of each site (defs.h:256-262,
 * e.g. D3Q27_SRT::collision, d3q27/col_srt.h:7-15).  Here a user compiles a
 * collision struct into a launcher with LBM_COLLISION_PLUGIN
 * (tnl-lbm_b200/csrc/plugin.cuh): the launcher runs this library's fused A-A
 * step (streaming, every boundary type of lbm_set_map, macro and sums
 * outputs) with the user's collision inlined in it, and registers under an
 * id in [LBM_COLL_PLUGIN_FIRST, LBM_COLL_PLUGIN_LAST] that lbm_desc.collision
 * then names.
 *
 * A launcher is called with the library's launch record of one step (an
 * opaque pointer) and the lattice's LBM_STORE_* storage, on the handle's
 * device; it returns a cudaError_t value (0 = success).  Called with
 * step == NULL it only answers whether it was built for `storage` (0, or
 * cudaErrorNotSupported).  abi_version is LBM_PLUGIN_ABI_VERSION as the
 * plugin saw it when compiled; the launch record's layout is that of the
 * same header tree, so a plugin is compiled against the headers of the
 * library it loads into.  Registration is process-wide; a handle keeps the
 * launcher it was created with, so the plugin's code must stay loaded while
 * such a handle lives.  launcher == NULL removes the id.  Plugin lattices run
 * the one-site kernel, or with LBM_KERNEL_PAIR on storages with FP32
 * arithmetic the two-site kernel, with A-A streaming (lbm_set_kernel accepts
 * LBM_KERNEL_DIRECT and LBM_KERNEL_PAIR, lbm_set_streaming only
 * LBM_STREAMING_AA) and take no coupled scalar, adjoint or ensemble. */
#define LBM_PLUGIN_ABI_VERSION 2
typedef int32_t (*lbm_collision_launcher)(const void* step, int32_t storage);
LBM_API int lbm_register_collision(int32_t id, lbm_collision_launcher launcher, int32_t abi_version, const char* name);
/* Name under which `id` was registered (NULL when none). */
LBM_API const char* lbm_collision_name(int32_t id);

LBM_API const char* lbm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* TNL_LBM_B200_H */
