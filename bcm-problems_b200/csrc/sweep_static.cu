// Allocation-free variant of the Jacobi-sweep triangular solve.
//
// bsg_solve_l_dev / bsg_solve_u_dev in sweep mode (mode 1, nsweeps > 1)
// ping-pong the iterates between the output vector and an n-length work
// vector that they take from the stream-ordered pool on every call.
// bsg_solve_sweep_static runs the same kernels in the same order, with the
// work vector replaced by a fixed device array of this file, so a call
// allocates and frees nothing.  It exists for callers that apply the
// preconditioner where device allocation is not available to them: a
// process whose memory budget is fixed up front, or a host loop that must
// not take the allocator's locks or grow the pool between iterations.
//
// Limits and rules:
//   * at most BSG_SWEEP_STATIC_ROWS rows (2^21, a 16 MiB array of doubles);
//     larger factors are rejected with BSG_ERR_ARG;
//   * the first call on a device looks up the array's address with
//     cudaGetSymbolAddress (which can load this module); make that first call
//     before any stream capture;
//   * the address is kept for the life of the process: a cudaDeviceReset (or
//     any reset of the device's primary context) unloads the module and
//     leaves the kept address stale, so after such a reset this entry point
//     must not be called again until the process restarts;
//   * the array is shared by every call on the device: calls that overlap in
//     time (other threads, other streams) race on it and give wrong results;
//     keep the calls on one stream, one after another;
//   * nothing in the array has to start at zero: every sweep writes all n
//     entries before the next sweep reads them.
#include "bsg_internal.cuh"
#include <cstdio>
#include <mutex>

#define BSG_SWEEP_STATIC_ROWS (1 << 21)
#define BSG_SWEEP_STATIC_DEVICES 64

static __device__ __align__(256) double g_sweep_scratch[BSG_SWEEP_STATIC_ROWS];

static double *g_sweep_scratch_ptr[BSG_SWEEP_STATIC_DEVICES];
static std::mutex g_sweep_scratch_mu;

// Address of the scratch array on `device` (looked up once per device, with
// that device current).
static int sweep_scratch(int device, double **out) {
	if (device < 0 || device >= BSG_SWEEP_STATIC_DEVICES)
		return bsg_set_error(BSG_ERR_UNSUPPORTED, "bsg_solve_sweep_static: device index too large");
	std::lock_guard<std::mutex> lock(g_sweep_scratch_mu);
	if (!g_sweep_scratch_ptr[device]) {
		int prev = -1;
		BSG_CUDA(cudaGetDevice(&prev));
		if (prev != device) BSG_CUDA(cudaSetDevice(device));
		void *p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_sweep_scratch);
		if (prev != device) cudaSetDevice(prev);
		if (e != cudaSuccess) return bsg_set_cuda_error(e, "cudaGetSymbolAddress(g_sweep_scratch)", __FILE__, __LINE__);
		g_sweep_scratch_ptr[device] = static_cast<double *>(p);
	}
	*out = g_sweep_scratch_ptr[device];
	return BSG_OK;
}

extern "C" int bsg_solve_sweep_static(bsg_ctx *c, const bsg_fct *f, int lower, int nsweeps, const double *x,
                                      double *y) {
	if (!c || !f || !x || !y || x == y) return bsg_set_error(BSG_ERR_ARG, "bsg_solve_sweep_static: bad argument");
	if (f->d_bia) return bsg_set_error(BSG_ERR_UNSUPPORTED, "bsg_solve_sweep_static: block factor");
	if (f->n > BSG_SWEEP_STATIC_ROWS) {
		char msg[160];
		std::snprintf(msg, sizeof msg, "bsg_solve_sweep_static: %d rows exceed the static scratch of %d rows", f->n,
		              BSG_SWEEP_STATIC_ROWS);
		return bsg_set_error(BSG_ERR_ARG, msg);
	}
	double *work = nullptr;
	int rc = sweep_scratch(c->device, &work);
	if (rc) return rc;
	// a failed launch has already recorded its own cause (bsg_last_error)
	return bsg_trisolve_launch(c, f, lower ? 1 : 0, 1, nsweeps, x, y, work);
}
