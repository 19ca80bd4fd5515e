// C-ABI of checkpoint / resume (lbm_checkpoint_save, lbm_checkpoint_load,
// declared in include/tnl_lbm_b200.h).
//
// The reference writes its state through ADIOS2 (State::saveState /
// loadState, include/lbm3d/state.hpp:891-1012): populations, macro fields,
// the map and the iteration counter.  ADIOS2 is not available here, so a
// checkpoint is one binary file: a fixed header with the lattice description
// and the A-A parity, then the map, the inlet profiles and the population
// buffer exactly as it sits in device memory (storage format and layout
// included), so that a resumed run continues bit for bit.
//
// File layout (little-endian, as written by this host):
//   Header   (struct CheckpointHeader below)
//   map      X*Y*Z bytes                     (when has_map)
//   inflow   Y*Z compute-type values each    (for each bit set in inflow_mask)
//   pops     pop_bytes                       (the current population buffer)
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tnl_lbm_b200.h"
#include "lattice.h"

namespace {

constexpr char MAGIC[8] = {'T', 'N', 'L', 'B', '2', '0', '0', 'C'};
constexpr uint32_t VERSION = 2;  // 2: slot rows interleaved per lattice row

struct CheckpointHeader
{
	char magic[8];
	uint32_t version;
	int32_t X, Y, Z;
	int32_t storage, collision, cum_flags, equilibrium, periodic, streaming;
	int32_t has_map;
	int32_t inflow_mask;  // bit k: inflow component k saved
	int32_t elem_size, compute_size;
	int64_t iteration;
	uint64_t pop_bytes;
	double viscosity, fx, fy, fz;
};

int cfail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int cfail(int code, const char* fmt, ...)
{
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	return lbm::record_error(code, buf);
}

struct File
{
	FILE* f = nullptr;
	~File()
	{
		if (f)
			fclose(f);
	}
};

}  // namespace

extern "C" {

int lbm_checkpoint_save(lbm_handle h, const char* path)
{
	if (!h || !path)
		return cfail(LBM_ERR_INVALID, "null argument");
	if (cudaSetDevice(h->d.device) != cudaSuccess)
		return cfail(LBM_ERR_CUDA, "cudaSetDevice(%d) failed", h->d.device);
	if (h->ade)
		return cfail(LBM_ERR_UNSUPPORTED, "checkpoints do not hold a coupled scalar (lbm_ade_disable first)");
	CheckpointHeader hd{};
	memcpy(hd.magic, MAGIC, sizeof(MAGIC));
	hd.version = VERSION;
	hd.X = h->d.X;
	hd.Y = h->d.Y;
	hd.Z = h->d.Z;
	hd.storage = h->d.storage;
	hd.collision = h->d.collision;
	hd.cum_flags = h->d.cum_flags;
	hd.equilibrium = h->d.equilibrium;
	hd.periodic = h->d.periodic;
	hd.streaming = h->streaming;
	hd.has_map = h->map_set ? 1 : 0;
	hd.elem_size = h->ops->elem_size;
	hd.compute_size = h->ops->compute_size;
	hd.iteration = h->iteration;
	hd.pop_bytes = h->pop_bytes;
	hd.viscosity = h->d.viscosity;
	hd.fx = h->d.fx;
	hd.fy = h->d.fy;
	hd.fz = h->d.fz;
	for (int k = 0; k < 3; k++)
		if (h->inflow[k])
			hd.inflow_mask |= 1 << k;
	const size_t prof = (size_t) h->d.Y * h->d.Z * h->ops->compute_size;
	std::vector<unsigned char> pops(h->pop_bytes);
	std::vector<unsigned char> inflow(3 * prof);
	if (cudaMemcpyAsync(pops.data(), h->g.f, h->pop_bytes, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
		return cfail(LBM_ERR_CUDA, "population read-back failed");
	for (int k = 0; k < 3; k++)
		if (h->inflow[k] && cudaMemcpyAsync(inflow.data() + k * prof, h->inflow[k], prof, cudaMemcpyDeviceToHost, h->stream)
								!= cudaSuccess)
			return cfail(LBM_ERR_CUDA, "inflow read-back failed");
	if (cudaStreamSynchronize(h->stream) != cudaSuccess)
		return cfail(LBM_ERR_CUDA, "stream synchronisation failed");
	File out;
	out.f = fopen(path, "wb");
	if (!out.f)
		return cfail(LBM_ERR_INVALID, "cannot open %s for writing", path);
	bool ok = fwrite(&hd, sizeof(hd), 1, out.f) == 1;
	if (ok && hd.has_map)
		ok = fwrite(h->map_host.data(), 1, h->map_host.size(), out.f) == h->map_host.size();
	for (int k = 0; ok && k < 3; k++)
		if (hd.inflow_mask & (1 << k))
			ok = fwrite(inflow.data() + k * prof, 1, prof, out.f) == prof;
	if (ok)
		ok = fwrite(pops.data(), 1, pops.size(), out.f) == pops.size();
	if (!ok || fflush(out.f) != 0)
		return cfail(LBM_ERR_INVALID, "writing %s failed", path);
	return LBM_OK;
}

int lbm_checkpoint_load(lbm_handle h, const char* path)
{
	if (!h || !path)
		return cfail(LBM_ERR_INVALID, "null argument");
	if (cudaSetDevice(h->d.device) != cudaSuccess)
		return cfail(LBM_ERR_CUDA, "cudaSetDevice(%d) failed", h->d.device);
	if (h->ade)
		return cfail(LBM_ERR_UNSUPPORTED, "checkpoints do not hold a coupled scalar (lbm_ade_disable first)");
	File in;
	in.f = fopen(path, "rb");
	if (!in.f)
		return cfail(LBM_ERR_INVALID, "cannot open %s", path);
	CheckpointHeader hd{};
	if (fread(&hd, sizeof(hd), 1, in.f) != 1 || memcmp(hd.magic, MAGIC, sizeof(MAGIC)) != 0)
		return cfail(LBM_ERR_INVALID, "%s is not a checkpoint of this library", path);
	if (hd.version != VERSION)
		return cfail(LBM_ERR_UNSUPPORTED, "checkpoint version %u, expected %u", hd.version, VERSION);
	if (hd.X != h->d.X || hd.Y != h->d.Y || hd.Z != h->d.Z || hd.storage != h->d.storage || hd.collision != h->d.collision
		|| hd.cum_flags != h->d.cum_flags || hd.equilibrium != h->d.equilibrium || hd.periodic != h->d.periodic
		|| hd.pop_bytes != h->pop_bytes)
		return cfail(LBM_ERR_INVALID,
					 "checkpoint of a %d x %d x %d lattice (storage %d, collision %d/%d, equilibrium %d, periodic %d) does not "
					 "match this handle",
					 hd.X, hd.Y, hd.Z, hd.storage, hd.collision, hd.cum_flags, hd.equilibrium, hd.periodic);
	if (hd.fx != h->d.fx || hd.fy != h->d.fy || hd.fz != h->d.fz)
		return cfail(LBM_ERR_INVALID, "checkpoint body force differs from this handle's");
	const size_t nsites = (size_t) hd.X * hd.Y * hd.Z;
	const size_t nprof = (size_t) hd.Y * hd.Z;
	const size_t cs = (size_t) hd.compute_size;
	std::vector<uint8_t> map;
	if (hd.has_map) {
		map.resize(nsites);
		if (fread(map.data(), 1, nsites, in.f) != nsites)
			return cfail(LBM_ERR_INVALID, "%s is truncated (map)", path);
	}
	std::vector<double> prof[3];
	for (int k = 0; k < 3; k++) {
		if (!(hd.inflow_mask & (1 << k)))
			continue;
		std::vector<unsigned char> raw(nprof * cs);
		if (fread(raw.data(), 1, raw.size(), in.f) != raw.size())
			return cfail(LBM_ERR_INVALID, "%s is truncated (inflow)", path);
		prof[k].resize(nprof);
		for (size_t i = 0; i < nprof; i++)
			prof[k][i] = cs == 8 ? ((const double*) raw.data())[i] : (double) ((const float*) raw.data())[i];
	}
	std::vector<unsigned char> pops(hd.pop_bytes);
	if (fread(pops.data(), 1, pops.size(), in.f) != pops.size())
		return cfail(LBM_ERR_INVALID, "%s is truncated (populations)", path);

	// the A-A/A-B pattern first (the map may hold types only A-B provides)
	if (int rc = lbm_set_streaming(h, hd.streaming))
		return rc;
	if (hd.has_map)
		if (int rc = lbm_set_map(h, map.data()))
			return rc;
	if (hd.inflow_mask)
		if (int rc = lbm_set_inflow(h, prof[0].empty() ? nullptr : prof[0].data(), prof[1].empty() ? nullptr : prof[1].data(),
									prof[2].empty() ? nullptr : prof[2].data()))
			return rc;
	if (hd.viscosity != h->d.viscosity)
		if (int rc = lbm_set_viscosity(h, hd.viscosity))
			return rc;
	if (cudaMemcpyAsync(h->g.f, pops.data(), pops.size(), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
		return cfail(LBM_ERR_CUDA, "population upload failed");
	if (h->streaming == LBM_STREAMING_AB
		&& cudaMemcpyAsync(h->f_out, h->g.f, h->pop_bytes, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
		return cfail(LBM_ERR_CUDA, "second buffer copy failed");
	if (cudaStreamSynchronize(h->stream) != cudaSuccess)
		return cfail(LBM_ERR_CUDA, "stream synchronisation failed");
	h->iteration = hd.iteration;
	h->macro_valid = h->sums_valid = false;
	h->drop_graph();
	return LBM_OK;
}

}  // extern "C"
