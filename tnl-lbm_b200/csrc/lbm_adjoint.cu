// C-ABI of the discrete adjoint (lbm_adjoint_*, declared in
// include/tnl_lbm_b200.h): gradients of an objective on the state after N
// A-A steps with the SRT collision, with respect to a per-site body force
// field and to the initial populations.
//
// Memory: sqrt(N)-style checkpointing.  The forward pass keeps the population
// array every K steps (ceil(N/K) checkpoints) and the final state.  The
// backward pass walks the segments from the last to the first: it restores
// the segment's checkpoint, recomputes and keeps the K states of the segment,
// and runs the K adjoint steps backwards through them.  Peak memory is
// (ceil(N/K) + K + 2) population arrays; K = sqrt(N) minimises it, and the
// cost is two primal steps and one adjoint step per step.
//
// The reference's adjoint (sim_adjoint/sim_adjoint.cu with D3Q27_SRT_ADJOINT,
// col_srt_adjoint.h) iterates a steady adjoint problem about a frozen primal
// flow; this is the time-dependent discrete adjoint of the same collision,
// whose per-site transpose reduces to the reference's adjoint collision at
// rho = 1 and zero force (adjoint.cuh).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <set>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tnl_lbm_b200.h"
#include "coll_params.cuh"
#include "adjoint.cuh"
#include "lattice.h"

namespace lbm {

struct AdjointState
{
	double* force = nullptr;	 // [3][Z][Y][X]
	std::vector<void*> ckpt;
	void* final_state = nullptr;
	std::vector<void*> seg;
	double* lam = nullptr;	 // FP64, the element strides of the population array
	double* grad = nullptr;	 // [3][Z][Y][X]
	long long* samples = nullptr;
	double* target = nullptr;
	double* loss_terms = nullptr;
	int nsamples = 0;
	double w_rho = 0;
	long long it0 = 0, nsteps = 0, every = 1;
	long long nckpt = 0;	   // checkpoints of this run (ckpt may hold more from earlier runs)
	int nsamples_cap = 0;	   // capacity of samples / target / loss_terms
	double loss = 0;
	bool forward_done = false;
};

void adjoint_free(AdjointState* a)
{
	if (!a)
		return;
	cudaFree(a->force);
	for (void* p : a->ckpt)
		cudaFree(p);
	cudaFree(a->final_state);
	for (void* p : a->seg)
		cudaFree(p);
	cudaFree(a->lam);
	cudaFree(a->grad);
	cudaFree(a->samples);
	cudaFree(a->target);
	cudaFree(a->loss_terms);
	delete a;
}

}  // namespace lbm

namespace {

int afail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int afail(int code, const char* fmt, ...)
{
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	return lbm::record_error(code, buf);
}

#define ADJ_CUDA(call)                                                                                    \
	do {                                                                                                  \
		cudaError_t err_ = (call);                                                                        \
		if (err_ != cudaSuccess)                                                                          \
			return afail(LBM_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_), __FILE__, \
						 __LINE__);                                                                       \
	} while (0)

template <typename S>
lbm::AdjArgs<typename S::T, typename S::R> make_args(lbm_handle h, void* f, void* lam, double* grad)
{
	using R = typename S::R;
	lbm::AdjArgs<typename S::T, R> a{};
	a.f = (typename S::T*) f;
	a.lam = (double*) lam;
	a.sq = h->g.sq;
	a.sy = h->g.sy;
	a.sz = h->g.sz;
	a.x0 = h->g.x0;
	a.X = h->g.X;
	a.Y = h->g.Y;
	a.Z = h->g.Z;
	a.map = h->d.periodic ? nullptr : h->map;
	a.in_vx = (const R*) h->inflow[0];
	a.in_vy = (const R*) h->inflow[1];
	a.in_vz = (const R*) h->inflow[2];
	a.force = h->adjoint->force;
	a.grad = grad;
	a.p = lbm::make_coll_params<R>(h->p);
	return a;
}

dim3 site_grid(lbm_handle h)
{
	return dim3((unsigned) ((h->d.X + 127) / 128), (unsigned) h->d.Y, (unsigned) h->d.Z);
}

template <typename S>
cudaError_t primal_step(lbm_handle h, void* f, long long n)
{
	const auto a = make_args<S>(h, f, nullptr, nullptr);
	if ((h->adjoint->it0 + n) & 1)
		lbm::adj_primal_kernel<S, true><<<site_grid(h), 128, 0, h->stream>>>(a);
	else
		lbm::adj_primal_kernel<S, false><<<site_grid(h), 128, 0, h->stream>>>(a);
	return cudaGetLastError();
}

template <typename S>
cudaError_t adjoint_step(lbm_handle h, void* f, long long n)
{
	auto* st = h->adjoint;
	const auto a = make_args<S>(h, f, st->lam, st->grad);
	if ((st->it0 + n) & 1)
		lbm::adj_step_kernel<S, true><<<site_grid(h), 128, 0, h->stream>>>(a);
	else
		lbm::adj_step_kernel<S, false><<<site_grid(h), 128, 0, h->stream>>>(a);
	return cudaGetLastError();
}

template <typename S>
cudaError_t objective(lbm_handle h, bool with_gradient, double seed)
{
	auto* st = h->adjoint;
	const auto a = make_args<S>(h, st->final_state, with_gradient ? st->lam : nullptr, with_gradient ? st->grad : nullptr);
	const int nb = (st->nsamples + 127) / 128;
	if ((st->it0 + st->nsteps) & 1)
		lbm::adj_objective_kernel<S, true>
			<<<nb, 128, 0, h->stream>>>(a, st->samples, st->target, st->nsamples, st->w_rho, seed, st->loss_terms);
	else
		lbm::adj_objective_kernel<S, false>
			<<<nb, 128, 0, h->stream>>>(a, st->samples, st->target, st->nsamples, st->w_rho, seed, st->loss_terms);
	return cudaGetLastError();
}

template <typename S>
int forward_typed(lbm_handle h)
{
	auto* st = h->adjoint;
	const size_t pb = h->pop_bytes;
	for (long long n = 0; n < st->nsteps; n++) {
		if (n % st->every == 0)
			ADJ_CUDA(cudaMemcpyAsync(st->ckpt[(size_t) (n / st->every)], h->g.f, pb, cudaMemcpyDeviceToDevice, h->stream));
		ADJ_CUDA(primal_step<S>(h, h->g.f, n));
	}
	ADJ_CUDA(cudaMemcpyAsync(st->final_state, h->g.f, pb, cudaMemcpyDeviceToDevice, h->stream));
	ADJ_CUDA(objective<S>(h, false, 0.0));
	std::vector<double> terms(st->nsamples);
	ADJ_CUDA(cudaMemcpyAsync(terms.data(), st->loss_terms, sizeof(double) * st->nsamples, cudaMemcpyDeviceToHost, h->stream));
	ADJ_CUDA(cudaStreamSynchronize(h->stream));
	double loss = 0;
	for (double v : terms)
		loss += v;
	st->loss = loss;
	return LBM_OK;
}

// bytes of the FP64 adjoint array (the population array's element count)
size_t lam_bytes(lbm_handle h)
{
	return h->pop_bytes / (size_t) h->ops->elem_size * sizeof(double);
}

template <typename S>
int backward_typed(lbm_handle h, double seed)
{
	auto* st = h->adjoint;
	ADJ_CUDA(cudaMemsetAsync(st->lam, 0, lam_bytes(h), h->stream));
	ADJ_CUDA(cudaMemsetAsync(st->grad, 0, sizeof(double) * 3 * h->sites(), h->stream));
	ADJ_CUDA(objective<S>(h, true, seed));
	const size_t pb = h->pop_bytes;
	const long long nseg = st->nckpt;
	for (long long s = nseg - 1; s >= 0; s--) {
		const long long n0 = s * st->every;
		const long long n1 = n0 + st->every < st->nsteps ? n0 + st->every : st->nsteps;
		ADJ_CUDA(cudaMemcpyAsync(st->seg[0], st->ckpt[(size_t) s], pb, cudaMemcpyDeviceToDevice, h->stream));
		for (long long i = 1; i < n1 - n0; i++) {
			ADJ_CUDA(cudaMemcpyAsync(st->seg[(size_t) i], st->seg[(size_t) (i - 1)], pb, cudaMemcpyDeviceToDevice, h->stream));
			ADJ_CUDA(primal_step<S>(h, st->seg[(size_t) i], n0 + i - 1));
		}
		for (long long n = n1 - 1; n >= n0; n--)
			ADJ_CUDA(adjoint_step<S>(h, st->seg[(size_t) (n - n0)], n));
	}
	return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_adjoint_forward(lbm_handle h, const double* force, int64_t nsteps, int64_t checkpoint_every, const int64_t* samples,
						int32_t nsamples, const double* target, double rho_weight, double* loss)
{
	if (!h)
		return afail(LBM_ERR_INVALID, "null handle");
	if (cudaSetDevice(h->d.device) != cudaSuccess)
		return afail(LBM_ERR_CUDA, "cudaSetDevice(%d) failed", h->d.device);
	if (h->d.collision != LBM_COLL_SRT || h->d.equilibrium != LBM_EQ_SECOND_ORDER)
		return afail(LBM_ERR_UNSUPPORTED, "the adjoint is provided for the SRT collision with D3Q27_EQ (LBM_EQ_SECOND_ORDER)");
	if (h->ade)
		return afail(LBM_ERR_UNSUPPORTED, "the adjoint does not cover a coupled scalar (lbm_ade_disable first)");
	if (h->streaming != LBM_STREAMING_AA)
		return afail(LBM_ERR_UNSUPPORTED, "the adjoint is provided for the A-A streaming pattern");
	if (h->d.storage != LBM_STORE_F64 && h->d.storage != LBM_STORE_F32)
		return afail(LBM_ERR_UNSUPPORTED, "the adjoint is provided for LBM_STORE_F64 and LBM_STORE_F32");
	if (!h->d.periodic && !h->map_set)
		return afail(LBM_ERR_INVALID, "lbm_set_map must be called before the adjoint of a non-periodic lattice");
	if (nsteps < 1 || nsamples < 1 || !samples || !target || !loss)
		return afail(LBM_ERR_INVALID, "nsteps and nsamples must be positive; samples, target and loss are required");
	if (!(rho_weight >= 0.0) || !std::isfinite(rho_weight))
		return afail(LBM_ERR_INVALID, "rho_weight must be non-negative");
	for (uint8_t g : h->map_host)
		if (g == lbm::GEO_INFLOW_LEFT || g == lbm::GEO_INFLOW_EQ_LEFT)
			return afail(LBM_ERR_UNSUPPORTED, "the adjoint has no transpose of GEO_INFLOW_LEFT / GEO_INFLOW_EQ_LEFT; use GEO_INFLOW");
	const long long nsites = h->sites();
	std::set<long long> seen;
	for (int i = 0; i < nsamples; i++) {
		const long long s = samples[i];
		if (s < 0 || s >= nsites)
			return afail(LBM_ERR_INVALID, "sample %d: site index %lld out of range", i, s);
		if (!seen.insert(s).second)
			return afail(LBM_ERR_INVALID, "sample %d: site %lld listed twice", i, s);
		if (!h->d.periodic && h->map_host[(size_t) s] != lbm::GEO_FLUID && h->map_host[(size_t) s] != lbm::GEO_PERIODIC)
			return afail(LBM_ERR_INVALID, "sample %d: site %lld is not a fluid site", i, s);
	}
	long long every = checkpoint_every;
	if (every <= 0)
		every = (long long) std::ceil(std::sqrt((double) nsteps));
	if (every > nsteps)
		every = nsteps;
	const long long nckpt = (nsteps + every - 1) / every;

	// the buffers of an earlier run are kept and grown only when this run
	// needs more (an optimisation loop reruns forward and backward)
	if (!h->adjoint)
		h->adjoint = new lbm::AdjointState();
	auto* st = h->adjoint;
	st->forward_done = false;
	st->it0 = h->iteration;
	st->nsteps = nsteps;
	st->every = every;
	st->nsamples = nsamples;
	st->w_rho = rho_weight;
	const int cs = h->ops->compute_size;
	auto fail_free = [&](int rc) {
		lbm::adjoint_free(h->adjoint);
		h->adjoint = nullptr;
		return rc;
	};
	// the control: per-site force in FP64, from host or device memory (the
	// uniform force of the descriptor when force is NULL); each step rounds it
	// to the compute type
	const size_t force_bytes = sizeof(double) * 3 * (size_t) nsites;
	std::vector<double> fh;
	if (!force) {
		fh.resize((size_t) 3 * nsites);
		for (long long k = 0; k < 3; k++)
			for (long long i = 0; i < nsites; i++)
				fh[(size_t) (k * nsites + i)] = k == 0 ? h->d.fx : (k == 1 ? h->d.fy : h->d.fz);
	}
	if ((!st->force && cudaMalloc(&st->force, force_bytes) != cudaSuccess)
		|| (!st->final_state && cudaMalloc(&st->final_state, h->pop_bytes) != cudaSuccess))
		return fail_free(afail(LBM_ERR_CUDA, "adjoint buffers: allocation failed"));
	if (nsamples > st->nsamples_cap) {
		cudaFree(st->samples);
		cudaFree(st->target);
		cudaFree(st->loss_terms);
		st->samples = nullptr;
		st->target = nullptr;
		st->loss_terms = nullptr;
		if (cudaMalloc(&st->samples, sizeof(long long) * nsamples) != cudaSuccess
			|| cudaMalloc(&st->target, sizeof(double) * 4 * nsamples) != cudaSuccess
			|| cudaMalloc(&st->loss_terms, sizeof(double) * nsamples) != cudaSuccess)
			return fail_free(afail(LBM_ERR_CUDA, "adjoint buffers: allocation failed"));
		st->nsamples_cap = nsamples;
	}
	while ((long long) st->ckpt.size() < nckpt) {
		void* p = nullptr;
		if (cudaMalloc(&p, h->pop_bytes) != cudaSuccess)
			return fail_free(afail(LBM_ERR_CUDA, "adjoint checkpoints: allocation of %lld x %zu bytes failed", nckpt, h->pop_bytes));
		st->ckpt.push_back(p);
	}
	st->nckpt = nckpt;
	if (cudaMemcpyAsync(st->force, force ? force : fh.data(), force_bytes, cudaMemcpyDefault, h->stream) != cudaSuccess
		|| cudaMemcpyAsync(st->samples, samples, sizeof(long long) * nsamples, cudaMemcpyHostToDevice, h->stream) != cudaSuccess
		|| cudaMemcpyAsync(st->target, target, sizeof(double) * 4 * nsamples, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
		return fail_free(afail(LBM_ERR_CUDA, "adjoint inputs: copy failed"));
	h->drop_graph();
	const int rc = cs == 8 ? forward_typed<lbm::StoreF64>(h) : forward_typed<lbm::StoreF32>(h);
	if (rc)
		return fail_free(rc);
	h->iteration = st->it0 + nsteps;
	h->macro_valid = h->sums_valid = false;
	st->forward_done = true;
	*loss = st->loss;
	return LBM_OK;
}

int lbm_adjoint_backward(lbm_handle h, double seed, double* grad_force, void* grad_populations, int layout, int dtype)
{
	if (!h)
		return afail(LBM_ERR_INVALID, "null handle");
	if (cudaSetDevice(h->d.device) != cudaSuccess)
		return afail(LBM_ERR_CUDA, "cudaSetDevice(%d) failed", h->d.device);
	auto* st = h->adjoint;
	if (!st || !st->forward_done)
		return afail(LBM_ERR_INVALID, "lbm_adjoint_backward needs a preceding lbm_adjoint_forward");
	if (grad_populations && ((layout != 0 && layout != 1) || (dtype != 0 && dtype != 1)))
		return afail(LBM_ERR_INVALID, "bad layout or dtype");
	const size_t pb = h->pop_bytes;
	if (!st->lam && (cudaMalloc(&st->lam, lam_bytes(h)) != cudaSuccess || cudaMalloc(&st->grad, sizeof(double) * 3 * h->sites()) != cudaSuccess))
		return afail(LBM_ERR_CUDA, "adjoint state allocation failed");
	while ((long long) st->seg.size() < st->every) {
		void* p = nullptr;
		if (cudaMalloc(&p, pb) != cudaSuccess)
			return afail(LBM_ERR_CUDA, "adjoint segment buffers: allocation of %lld x %zu bytes failed", st->every, pb);
		st->seg.push_back(p);
	}
	const int rc = h->ops->compute_size == 8 ? backward_typed<lbm::StoreF64>(h, seed) : backward_typed<lbm::StoreF32>(h, seed);
	if (rc)
		return rc;
	if (grad_force)
		ADJ_CUDA(cudaMemcpyAsync(grad_force, st->grad, sizeof(double) * 3 * h->sites(), cudaMemcpyDefault, h->stream));
	if (grad_populations) {
		// the adjoint of the initial population array, in the dense layout of
		// lbm_get_populations (an FP64 array with the population array's
		// element strides, converted by the FP64 storage's pack kernel)
		const int gh = layout == LBM_LAYOUT_GHOST ? 2 : 0;
		const size_t count = (size_t) 27 * (h->d.X + gh) * (h->d.Y + gh) * (h->d.Z + gh);
		const size_t bytes = count * (dtype == 0 ? 8 : 4);
		void* dev = nullptr;
		ADJ_CUDA(cudaMallocAsync(&dev, bytes, h->stream));
		lbm::Geometry g = h->g;
		g.f = st->lam;
		const cudaError_t e = lbm::storage_ops(lbm::ST_F64).pack(g, dev, dtype, layout, h->stream);
		if (e != cudaSuccess) {
			cudaFreeAsync(dev, h->stream);
			return afail(LBM_ERR_CUDA, "pack failed: %s", cudaGetErrorString(e));
		}
		ADJ_CUDA(cudaMemcpyAsync(grad_populations, dev, bytes, cudaMemcpyDefault, h->stream));
		cudaFreeAsync(dev, h->stream);
	}
	ADJ_CUDA(cudaStreamSynchronize(h->stream));
	return LBM_OK;
}

int lbm_adjoint_release(lbm_handle h)
{
	if (!h)
		return afail(LBM_ERR_INVALID, "null handle");
	cudaSetDevice(h->d.device);
	cudaStreamSynchronize(h->stream);
	lbm::adjoint_free(h->adjoint);
	h->adjoint = nullptr;
	return LBM_OK;
}

}  // extern "C"
