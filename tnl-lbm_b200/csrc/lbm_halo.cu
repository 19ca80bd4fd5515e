// Slabs of a lattice split along z, and their halo exchange (lbm_halo_*,
// declared in include/tnl_lbm_b200.h).
//
// The reference decomposes the lattice over MPI ranks and synchronises the
// overlaps of every population array after each step
// (include/lbm3d/lattice_decomposition.h:16-55, lbm.hpp:189-273).  Here a slab
// is a lattice handle marked as distributed along z: its periodic sites do not
// wrap in z (kernelInitIndices with distributed.z(), kernels.h:21-37) but reach
// the ghost layer.  Under the A-A pattern only the odd step reads and writes
// across a z face, and only the nine slots whose direction crosses it:
//
//   before the odd step  upper.ghost(z = -1)[c_z = -1]  <- lower.interior(Z-1)[c_z = -1]
//                        lower.ghost(z = Z)[c_z = +1]   <- upper.interior(0)[c_z = +1]
//   after the odd step   lower.interior(Z-1)[c_z = -1]  <- upper.ghost(z = -1)[c_z = -1]
//                        upper.interior(0)[c_z = +1]    <- lower.ghost(z = Z)[c_z = +1]
//
// (a site at the face reads those slots from the neighbour before the step and
// writes the populations that leave the slab into its ghost layer).  The even
// step is local.  Every plane moved is the whole (y, x) plane of a slot with
// its ghost rows: Y + 2 rows of sq elements, sy apart (the slots of a lattice
// row lie side by side).
//
// lbm_halo_copy moves planes between two slabs of one process with one kernel
// on the receiver's device; between GPUs the kernel reads the sender's memory
// with peer loads over NVLink (plain loads, no bulk-copy multicast).
// lbm_halo_pack / lbm_halo_unpack stage the planes in a device buffer for a
// transport between processes (NCCL send/recv in pytnl_lbm).
#include <cstdarg>
#include <cstdio>

#include <cuda_runtime.h>

#include "../../include/tnl_lbm_b200.h"
#include "d3q27.cuh"
#include "lattice.h"

namespace {

int hfail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int hfail(int code, const char* fmt, ...)
{
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof(buf), fmt, ap);
	va_end(ap);
	return lbm::record_error(code, buf);
}

#define HALO_CUDA(call)                                                                                   \
	do {                                                                                                  \
		cudaError_t err_ = (call);                                                                        \
		if (err_ != cudaSuccess)                                                                          \
			return hfail(LBM_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_), __FILE__, \
						 __LINE__);                                                                       \
	} while (0)

// the nine slots whose z component is cz
struct Slots
{
	int q[9];
};

Slots slots_of(int cz)
{
	Slots s{};
	int n = 0;
	for (int q = 0; q < 27; q++)
		if (lbm::cz(q) == cz)
			s.q[n++] = q;
	return s;
}

// One (y, x) plane of a slot: Y + 2 rows of `row` elements, `pitch` apart.
struct Plane
{
	char* base;		 // element 0 of the allocation
	long long sq;	 // slot stride (0 for a staging buffer: planes back to back)
	long long pitch; // row stride
	long long off;	 // element offset of the plane's first row
	long long sbuf;	 // staging buffer: element stride between the nine planes
};

// dst slot dq[k] plane <- src slot sq_[k] plane, k = 0..8 (blockIdx.y); W is
// an unsigned type of the storage element's width; n = rows * row elements
template <typename W>
__global__ void plane_copy_kernel(Plane dst, Slots dq, Plane src, Slots sq_, long long row, long long n)
{
	const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
	const int k = blockIdx.y;
	if (i >= n)
		return;
	const long long r = i / row, c = i - r * row;
	W* d = reinterpret_cast<W*>(dst.base) + dq.q[k] * dst.sq + k * dst.sbuf + dst.off + r * dst.pitch + c;
	const W* s = reinterpret_cast<const W*>(src.base) + sq_.q[k] * src.sq + k * src.sbuf + src.off + r * src.pitch + c;
	*d = *s;
}

Slots dense_slots()
{
	Slots s{};
	for (int k = 0; k < 9; k++)
		s.q[k] = k;
	return s;
}

int check(lbm_handle h)
{
	if (!h)
		return hfail(LBM_ERR_INVALID, "null handle");
	if (cudaSetDevice(h->d.device) != cudaSuccess)
		return hfail(LBM_ERR_CUDA, "cudaSetDevice(%d) failed", h->d.device);
	return LBM_OK;
}

bool args_ok(lbm_handle h, int z, int cz)
{
	return z >= -1 && z <= h->d.Z && (cz == -1 || cz == 1);
}

// elements of one slot plane: Y + 2 rows of one row pitch
long long plane_elems(lbm_handle h)
{
	return (long long) (h->d.Y + 2) * h->g.sq;
}

// slot plane z (ghost frame -1 .. Z) of a lattice
Plane lattice_plane(lbm_handle h, int z)
{
	return Plane{(char*) h->g.f, h->g.sq, h->g.sy, (long long) (z + 1) * h->g.sz, 0};
}

// the nine planes of a staging buffer, back to back
Plane buffer_planes(lbm_handle h, const void* buf)
{
	return Plane{(char*) buf, 0, h->g.sq, 0, plane_elems(h)};
}

int launch_planes(cudaStream_t st, int elem, const Plane& dst, const Slots& dq, const Plane& src, const Slots& sq_,
				  long long row, long long n)
{
	const dim3 grid((unsigned) ((n + 255) / 256), 9);
	if (elem == 8)
		plane_copy_kernel<unsigned long long><<<grid, 256, 0, st>>>(dst, dq, src, sq_, row, n);
	else if (elem == 4)
		plane_copy_kernel<unsigned><<<grid, 256, 0, st>>>(dst, dq, src, sq_, row, n);
	else
		plane_copy_kernel<unsigned short><<<grid, 256, 0, st>>>(dst, dq, src, sq_, row, n);
	const cudaError_t e = cudaGetLastError();
	return e == cudaSuccess ? LBM_OK : hfail(LBM_ERR_CUDA, "halo copy launch failed: %s", cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int lbm_set_distributed_z(lbm_handle h, int distributed)
{
	if (int rc = check(h))
		return rc;
	if (distributed && h->streaming != LBM_STREAMING_AA)
		return hfail(LBM_ERR_UNSUPPORTED, "slabs are provided for the A-A pattern");
	if (distributed && h->ade)
		return hfail(LBM_ERR_UNSUPPORTED, "slabs do not carry a coupled scalar");
	h->distributed_z = distributed != 0;
	h->drop_graph();
	return LBM_OK;
}

int64_t lbm_halo_bytes(lbm_handle h)
{
	if (!h)
		return -1;
	return (int64_t) 9 * plane_elems(h) * h->ops->elem_size;
}

int lbm_halo_pack(lbm_handle h, int z, int cz, void* dev_buf)
{
	if (int rc = check(h))
		return rc;
	if (!dev_buf || !args_ok(h, z, cz))
		return hfail(LBM_ERR_INVALID, "bad arguments (z %d, cz %d)", z, cz);
	return launch_planes(h->stream, h->ops->elem_size, buffer_planes(h, dev_buf), dense_slots(), lattice_plane(h, z),
						 slots_of(cz), h->g.sq, plane_elems(h));
}

int lbm_halo_unpack(lbm_handle h, int z, int cz, const void* dev_buf)
{
	if (int rc = check(h))
		return rc;
	if (!dev_buf || !args_ok(h, z, cz))
		return hfail(LBM_ERR_INVALID, "bad arguments (z %d, cz %d)", z, cz);
	return launch_planes(h->stream, h->ops->elem_size, lattice_plane(h, z), slots_of(cz), buffer_planes(h, dev_buf),
						 dense_slots(), h->g.sq, plane_elems(h));
}

int lbm_halo_copy(lbm_handle dst, int dst_z, lbm_handle src, int src_z, int cz)
{
	if (int rc = check(src))
		return rc;
	if (!dst || !args_ok(dst, dst_z, cz) || !args_ok(src, src_z, cz))
		return hfail(LBM_ERR_INVALID, "bad arguments (z %d / %d, cz %d)", dst_z, src_z, cz);
	if (dst->g.sq != src->g.sq || dst->d.Y != src->d.Y || dst->ops != src->ops)
		return hfail(LBM_ERR_INVALID, "the two slabs differ in their x-y plane or storage format");
	// the sender's stream has finished what it wrote into the plane
	if (!src->halo_ev)
		HALO_CUDA(cudaEventCreateWithFlags(&src->halo_ev, cudaEventDisableTiming));
	HALO_CUDA(cudaEventRecord(src->halo_ev, src->stream));
	if (int rc = check(dst))
		return rc;
	if (dst->d.device != src->d.device) {
		int can = 0;
		HALO_CUDA(cudaDeviceCanAccessPeer(&can, dst->d.device, src->d.device));
		if (!can)
			return hfail(LBM_ERR_UNSUPPORTED, "device %d cannot read device %d's memory", dst->d.device, src->d.device);
		const cudaError_t e = cudaDeviceEnablePeerAccess(src->d.device, 0);
		if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled)
			return hfail(LBM_ERR_CUDA, "peer access: %s", cudaGetErrorString(e));
		cudaGetLastError();	 // clear cudaErrorPeerAccessAlreadyEnabled
	}
	if (!dst->halo_ev)
		HALO_CUDA(cudaEventCreateWithFlags(&dst->halo_ev, cudaEventDisableTiming));
	HALO_CUDA(cudaStreamWaitEvent(dst->stream, src->halo_ev, 0));
	const Slots sl = slots_of(cz);
	if (int rc = launch_planes(dst->stream, dst->ops->elem_size, lattice_plane(dst, dst_z), sl, lattice_plane(src, src_z), sl,
							   dst->g.sq, plane_elems(dst)))
		return rc;
	// the sender does not overwrite the plane before the copy has read it
	HALO_CUDA(cudaEventRecord(dst->halo_ev, dst->stream));
	if (int rc = check(src))
		return rc;
	HALO_CUDA(cudaStreamWaitEvent(src->stream, dst->halo_ev, 0));
	return LBM_OK;
}

}  // extern "C"
