// C-ABI of the coupled D3Q7 advection-diffusion scalar (lbm_ade_*, declared in
// include/tnl_lbm_b200.h).  The reference couples a second LBM block set of
// D3Q7 type to the flow (State_NSE_ADE, include/lbm3d/state_NSE_ADE.h, with
// the coupled kernel of include/lbm3d/kernels.h:114-196); here the scalar is
// an extension of one lattice handle: its seven slots, seven slot rows per
// lattice row with the flow lattice's row pitch, are updated by the coupled
// step kernel of ade.cuh inside every lbm_step.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tnl_lbm_b200.h"
#include "ade.cuh"
#include "host_common.h"
#include "lattice.h"

namespace lbm {
int record_error(int code, const char* msg);

void ade_free(AdeState* s)
{
	if (!s)
		return;
	cudaFree(s->launch.g);
	cudaFree((void*) s->launch.map);
	cudaFree((void*) s->launch.dcoef);
	cudaFree(s->phi_buf);
	cudaFree(s->pair_groups);
	cudaFree(s->pair_rest);
	cudaFree(s->pair_work);
	delete s;
}

// Group flags, rest-site list and work list of the two-site coupled step
// (ade_pair.cuh) from the host copies of both maps: a group of PAIR_GROUP
// sites is a pair group when its flow sites are all GEO_FLUID (or all
// GEO_PERIODIC) and its scalar sites all collide without a boundary rewrite
// (ADE_FLUID, ADE_SOLID, ADE_PERIODIC); the other groups' sites are listed
// unless both their flow and scalar types are NOTHING.  Periodic lattices
// (no flow map) get no lists; their coupled step runs one site per thread.
int ade_build_pair(lbm_lattice* h)
{
	AdeState* s = h->ade;
	cudaFree(s->pair_groups);
	cudaFree(s->pair_rest);
	cudaFree(s->pair_work);
	s->pair_groups = nullptr;
	s->pair_rest = nullptr;
	s->pair_work = nullptr;
	s->launch.pair_groups = nullptr;
	s->launch.pair_work = PairWork{nullptr, 0, nullptr, 0};
	s->pair_dirty = false;
	if (h->d.periodic || !h->map_set)
		return 0;
	const int X = h->d.X, Y = h->d.Y, Z = h->d.Z;
	const uint8_t* fm = h->map_host.data();
	const uint8_t* am = s->map_host.data();
	const int gx = (X + PAIR_GROUP - 1) / PAIR_GROUP;
	const int tiles_x = ((X + 1) / 2 + 127) / 128;
	if ((long long) Y * Z * tiles_x >= (long long) PAIR_WORK_REST)
		return 0;
	std::vector<uint8_t> groups((size_t) gx * Y * Z);
	std::vector<unsigned long long> rest;
	for (long long row = 0; row < (long long) Y * Z; row++)
		for (int k = 0; k < gx; k++) {
			const int x0 = k * PAIR_GROUP;
			const uint8_t first = fm[row * X + x0];
			bool same = x0 + PAIR_GROUP <= X && (first == GEO_FLUID || first == GEO_PERIODIC);
			for (int x = x0; same && x < x0 + PAIR_GROUP; x++) {
				const uint8_t ag = am[row * X + x];
				same = fm[row * X + x] == first && (ag == ADE_FLUID || ag == ADE_SOLID || ag == ADE_PERIODIC);
			}
			groups[row * gx + k] = !same ? PAIR_GROUP_REST : (first == GEO_PERIODIC ? PAIR_GROUP_PERIODIC : PAIR_GROUP_FLUID);
			if (!same)
				for (int x = x0; x < x0 + PAIR_GROUP && x < X; x++)
					if (fm[row * X + x] != GEO_NOTHING || am[row * X + x] != ADE_NOTHING)
						rest.push_back((unsigned long long) row << 32 | (unsigned) x);
		}
	const long long nchunks = ((long long) rest.size() + 127) / 128;
	if (nchunks >= (long long) PAIR_WORK_REST)
		return 0;
	std::vector<unsigned> work;
	long long c = 0;
	for (int z = 0; z < Z; z++) {
		// the plane's rest chunks first, as the flow step's work list
		while (c < nchunks && (long long) (rest[(size_t) c * 128] >> 32) / Y <= z)
			work.push_back(PAIR_WORK_REST | (unsigned) c++);
		for (int y = 0; y < Y; y++) {
			const long long row = (long long) z * Y + y;
			for (int t = 0; t < tiles_x; t++) {
				bool any = false;
				for (int g = t * 256 / PAIR_GROUP; !any && g < gx && g < (t + 1) * 256 / PAIR_GROUP; g++)
					any = groups[row * gx + g] != PAIR_GROUP_REST;
				if (any)
					work.push_back((unsigned) (row * tiles_x + t));
			}
		}
	}
	if (work.empty())
		return 0;
	cudaError_t e = cudaMalloc(&s->pair_groups, groups.size());
	if (e == cudaSuccess)
		e = cudaMalloc(&s->pair_rest, (rest.empty() ? 1 : rest.size()) * sizeof(unsigned long long));
	if (e == cudaSuccess)
		e = cudaMalloc(&s->pair_work, work.size() * sizeof(unsigned));
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(s->pair_groups, groups.data(), groups.size(), cudaMemcpyHostToDevice, h->stream);
	if (e == cudaSuccess && !rest.empty())
		e = cudaMemcpyAsync(s->pair_rest, rest.data(), rest.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice,
							h->stream);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(s->pair_work, work.data(), work.size() * sizeof(unsigned), cudaMemcpyHostToDevice, h->stream);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(h->stream);
	if (e != cudaSuccess)
		return record_error(LBM_ERR_CUDA, cudaGetErrorString(e));
	s->launch.pair_groups = s->pair_groups;
	s->launch.pair_work = PairWork{s->pair_work, (long long) work.size(), s->pair_rest, (long long) rest.size()};
	return 0;
}

}  // namespace lbm

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

#define ADE_CUDA(call)                                                                                    \
	do {                                                                                                  \
		cudaError_t err_ = (call);                                                                        \
		if (err_ != cudaSuccess)                                                                          \
			return efail(LBM_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_), __FILE__, \
						 __LINE__);                                                                       \
	} while (0)

int check(lbm_handle h, bool need_ade = true)
{
	if (!h)
		return efail(LBM_ERR_INVALID, "null handle");
	if (cudaSetDevice(h->d.device) != cudaSuccess)
		return efail(LBM_ERR_CUDA, "cudaSetDevice(%d) failed", h->d.device);
	if (need_ade && !h->ade)
		return efail(LBM_ERR_INVALID, "no scalar: call lbm_ade_enable first");
	return LBM_OK;
}

// dense host buffer [7][nz][ny][nx] (ghost layer included when gh = 1) <->
// the scalar's planes in the compute type
template <typename R, typename H, bool TO_DENSE>
__global__ void ade_convert_kernel(lbm::Geometry g, R* __restrict__ planes, H* __restrict__ dense, int gh)
{
	const long long nx = g.X + 2 * gh, ny = g.Y + 2 * gh, nz = g.Z + 2 * gh;
	const long long n = nx * ny * nz;
	const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const long long x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
	// coordinates in the ghost-layer frame (0 = ghost layer)
	const long long xg = x + 1 - gh, yg = y + 1 - gh, zg = z + 1 - gh;
	const long long s = zg * g.sz + yg * g.sy + (g.x0 - 1) + xg;
	for (int q = 0; q < 7; q++) {
		if (TO_DENSE)
			dense[q * n + i] = (H) planes[q * g.sq + s];
		else
			planes[q * g.sq + s] = (R) dense[q * n + i];
	}
}

int convert(lbm_handle h, void* dense_dev, int dtype, int layout, bool to_dense)
{
	const int gh = layout == 1 ? 1 : 0;
	const long long n = (long long) (h->d.X + 2 * gh) * (h->d.Y + 2 * gh) * (h->d.Z + 2 * gh);
	const unsigned nb = (unsigned) ((n + 127) / 128);
	const bool f64 = h->ops->compute_size == 8;
	void* planes = h->ade->launch.g;
	lbm::Geometry g = h->g;	 // the scalar's geometry: the flow's rows, seven slots
	g.sq = h->ade->launch.sq;
	g.sy = h->ade->launch.sy;
	g.sz = h->ade->launch.sz;
#define ADE_CONV(R, H)                                                                                                 \
	do {                                                                                                               \
		if (to_dense)                                                                                                  \
			ade_convert_kernel<R, H, true><<<nb, 128, 0, h->stream>>>(g, (R*) planes, (H*) dense_dev, gh);             \
		else                                                                                                           \
			ade_convert_kernel<R, H, false><<<nb, 128, 0, h->stream>>>(g, (R*) planes, (H*) dense_dev, gh);            \
	} while (0)
	if (f64 && dtype == 0)
		ADE_CONV(double, double);
	else if (f64)
		ADE_CONV(double, float);
	else if (dtype == 0)
		ADE_CONV(float, double);
	else
		ADE_CONV(float, float);
#undef ADE_CONV
	const cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? LBM_OK : efail(LBM_ERR_CUDA, "scalar layout conversion failed: %s", cudaGetErrorString(e));
}

long long dense_count(lbm_handle h, int layout)
{
	const int gh = layout == 1 ? 1 : 0;
	return 7LL * (h->d.X + 2 * gh) * (h->d.Y + 2 * gh) * (h->d.Z + 2 * gh);
}

// D3Q7 equilibrium (d3q7/eq.h:17-54) in FP64 on the host
double feq7(int q, double phi, double vx, double vy, double vz)
{
	static const int c[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
	const double w = q == 0 ? 0.25 : 0.125;
	const double cu = c[q][0] * vx + c[q][1] * vy + c[q][2] * vz;
	return w * phi * (1.0 - 2.0 * (vx * vx + vy * vy + vz * vz) + 4.0 * cu + 8.0 * cu * cu);
}

}  // namespace

extern "C" {

int lbm_ade_enable(lbm_handle h, const lbm_ade_desc* desc)
{
	if (int rc = check(h, false))
		return rc;
	if (!desc)
		return efail(LBM_ERR_INVALID, "null descriptor");
	if (h->ade)
		return efail(LBM_ERR_INVALID, "the scalar is already enabled");
	if (h->ops->elem_size != h->ops->compute_size)
		return efail(LBM_ERR_UNSUPPORTED, "the coupled scalar needs FP64, FP32 or F32S storage (storage %s)", h->ops->name);
	if (h->streaming != LBM_STREAMING_AA)
		return efail(LBM_ERR_UNSUPPORTED, "the coupled scalar runs on A-A lattices only");
	if (h->plugin)
		return efail(LBM_ERR_UNSUPPORTED, "the coupled scalar runs with the built-in collisions only");
	if (h->adjoint)
		return efail(LBM_ERR_UNSUPPORTED, "release the adjoint first (lbm_adjoint_release)");
	if (desc->collision < 0 || desc->collision > 2)
		return efail(LBM_ERR_INVALID, "unknown scalar collision %d", desc->collision);
	if (!(desc->diffusion > 0.0) || !std::isfinite(desc->diffusion) || !std::isfinite(desc->inflow_phi))
		return efail(LBM_ERR_INVALID, "the diffusion coefficient must be positive and finite");
	auto* s = new lbm::AdeState();
	const size_t cs = (size_t) h->ops->compute_size;
	const size_t n = (size_t) h->sites();
	const lbm::Geometry ag = lbm::make_geometry(h->d.X, h->d.Y, h->d.Z, (int) cs, 7);
	s->launch.sq = ag.sq;
	s->launch.sy = ag.sy;
	s->launch.sz = ag.sz;
	const size_t gbytes = lbm::geometry_elems(ag) * cs;
	cudaError_t e = cudaMalloc(&s->launch.g, gbytes);
	uint8_t* map = nullptr;
	if (e == cudaSuccess)
		e = cudaMemsetAsync(s->launch.g, 0, gbytes, h->stream);
	if (e == cudaSuccess)
		e = cudaMalloc(&map, n);
	if (e == cudaSuccess)
		e = cudaMemsetAsync(map, lbm::ADE_FLUID, n, h->stream);
	s->launch.map = map;
	if (e == cudaSuccess)
		e = cudaMalloc(&s->phi_buf, n * cs);
	if (e != cudaSuccess) {
		lbm::ade_free(s);
		return efail(LBM_ERR_CUDA, "scalar allocation failed: %s", cudaGetErrorString(e));
	}
	s->map_host.assign(n, (uint8_t) lbm::ADE_FLUID);
	s->launch.D = desc->diffusion;
	s->launch.inflow_phi = desc->inflow_phi;
	s->launch.coll = desc->collision;
	h->ade = s;
	h->drop_graph();
	return LBM_OK;
}

int lbm_ade_disable(lbm_handle h)
{
	if (int rc = check(h))
		return rc;
	ADE_CUDA(cudaStreamSynchronize(h->stream));
	lbm::ade_free(h->ade);
	h->ade = nullptr;
	h->drop_graph();
	return LBM_OK;
}

int lbm_ade_set_map(lbm_handle h, const uint8_t* map)
{
	if (int rc = check(h))
		return rc;
	if (!map)
		return efail(LBM_ERR_INVALID, "null map");
	const long long n = h->sites();
	for (long long i = 0; i < n; i++)
		if (!lbm::ade_type_supported(map[i]))
			return efail(LBM_ERR_UNSUPPORTED,
						 "scalar site type %d at site %lld is not supported (outflow and phase-transfer types depend on "
						 "the order of the A-A update)",
						 (int) map[i], i);
	h->ade->map_host.assign(map, map + n);
	ADE_CUDA(cudaMemcpyAsync((void*) h->ade->launch.map, h->ade->map_host.data(), (size_t) n, cudaMemcpyHostToDevice,
							 h->stream));
	ADE_CUDA(cudaStreamSynchronize(h->stream));
	h->ade->pair_dirty = true;
	h->drop_graph();
	return LBM_OK;
}

int lbm_ade_set_diffusion(lbm_handle h, const double* field)
{
	if (int rc = check(h))
		return rc;
	const size_t n = (size_t) h->sites();
	const size_t cs = (size_t) h->ops->compute_size;
	if (!field) {
		if (h->ade->launch.dcoef) {
			ADE_CUDA(cudaStreamSynchronize(h->stream));
			cudaFree((void*) h->ade->launch.dcoef);
			h->ade->launch.dcoef = nullptr;
			h->drop_graph();
		}
		return LBM_OK;
	}
	for (size_t i = 0; i < n; i++)
		if (!(field[i] > 0.0) || !std::isfinite(field[i]))
			return efail(LBM_ERR_INVALID, "diffusion coefficient at site %zu must be positive and finite", i);
	std::vector<unsigned char> tmp(n * cs);
	if (cs == 8)
		std::memcpy(tmp.data(), field, n * 8);
	else
		for (size_t i = 0; i < n; i++)
			((float*) tmp.data())[i] = (float) field[i];
	if (!h->ade->launch.dcoef) {
		void* p = nullptr;
		ADE_CUDA(cudaMalloc(&p, n * cs));
		h->ade->launch.dcoef = p;
		h->drop_graph();
	}
	ADE_CUDA(cudaMemcpyAsync((void*) h->ade->launch.dcoef, tmp.data(), n * cs, cudaMemcpyHostToDevice, h->stream));
	ADE_CUDA(cudaStreamSynchronize(h->stream));
	return LBM_OK;
}

int lbm_ade_init_equilibrium(lbm_handle h, const double* phi, const double* vx, const double* vy, const double* vz,
							 double uniform_phi)
{
	if (int rc = check(h))
		return rc;
	const long long X = h->d.X, Y = h->d.Y, Z = h->d.Z;
	const long long nxg = X + 2, nyg = Y + 2, nzg = Z + 2, ng = nxg * nyg * nzg;
	std::vector<double> dense(7 * (size_t) ng);
	auto clampi = [](long long v, long long n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); };
	// ghost sites take the equilibrium of the nearest lattice site
	for (long long zg = 0; zg < nzg; zg++)
		for (long long yg = 0; yg < nyg; yg++)
			for (long long xg = 0; xg < nxg; xg++) {
				const long long x = clampi(xg - 1, X), y = clampi(yg - 1, Y), z = clampi(zg - 1, Z);
				const long long i = (z * Y + y) * X + x;
				const double p = phi ? phi[i] : uniform_phi;
				const double ux = vx ? vx[i] : 0.0, uy = vy ? vy[i] : 0.0, uz = vz ? vz[i] : 0.0;
				const long long d = (zg * nyg + yg) * nxg + xg;
				for (int q = 0; q < 7; q++)
					dense[q * ng + d] = feq7(q, p, ux, uy, uz);
			}
	return lbm_ade_set_populations(h, dense.data(), 1, 0);
}

int lbm_ade_set_populations(lbm_handle h, const void* host, int layout, int dtype)
{
	if (int rc = check(h))
		return rc;
	if (!host || (layout != 0 && layout != 1) || (dtype != 0 && dtype != 1))
		return efail(LBM_ERR_INVALID, "bad arguments");
	const size_t bytes = (size_t) dense_count(h, layout) * (dtype == 0 ? 8 : 4);
	void* dev = nullptr;
	ADE_CUDA(cudaMallocAsync(&dev, bytes, h->stream));
	ADE_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, h->stream));
	const int rc = convert(h, dev, dtype, layout, false);
	cudaFreeAsync(dev, h->stream);
	ADE_CUDA(cudaStreamSynchronize(h->stream));
	return rc;
}

int lbm_ade_get_populations(lbm_handle h, void* host, int layout, int dtype)
{
	if (int rc = check(h))
		return rc;
	if (!host || (layout != 0 && layout != 1) || (dtype != 0 && dtype != 1))
		return efail(LBM_ERR_INVALID, "bad arguments");
	const size_t bytes = (size_t) dense_count(h, layout) * (dtype == 0 ? 8 : 4);
	void* dev = nullptr;
	ADE_CUDA(cudaMallocAsync(&dev, bytes, h->stream));
	int rc = convert(h, dev, dtype, layout, true);
	if (rc == LBM_OK && cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
		rc = efail(LBM_ERR_CUDA, "scalar population copy failed");
	cudaFreeAsync(dev, h->stream);
	ADE_CUDA(cudaStreamSynchronize(h->stream));
	return rc;
}

int lbm_ade_get_phi(lbm_handle h, double* host)
{
	if (int rc = check(h))
		return rc;
	if (!host)
		return efail(LBM_ERR_INVALID, "null output");
	if (!h->macro_valid || !h->ade->phi_valid)
		return efail(LBM_ERR_INVALID, "no scalar field: run lbm_step with LBM_STEP_MACRO first");
	const size_t n = (size_t) h->sites();
	const size_t cs = (size_t) h->ops->compute_size;
	std::vector<unsigned char> tmp(n * cs);
	ADE_CUDA(cudaMemcpyAsync(tmp.data(), h->ade->phi_buf, n * cs, cudaMemcpyDeviceToHost, h->stream));
	ADE_CUDA(cudaStreamSynchronize(h->stream));
	if (cs == 8)
		std::memcpy(host, tmp.data(), n * 8);
	else
		for (size_t i = 0; i < n; i++)
			host[i] = ((const float*) tmp.data())[i];
	return LBM_OK;
}

}  // extern "C"
