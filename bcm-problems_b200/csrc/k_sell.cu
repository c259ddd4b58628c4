// SELL-8 storage and kernels for the bandwidth-bound products of the path:
// the SpMV of a point matrix and the Jacobi sweeps of the triangular solves.
//
// Layout.  Rows are cut into slices of C = 8 consecutive rows; slice s has
// width w_s = the longest row in it, and its entries are stored column-major
// in [off_s, off_s + 8 w_s): entry k of row 8 s + l at off_s + 8 k + l.
// Short rows are padded with (column = the row itself, value 0).
//
// Why: a warp serves 4 consecutive slices, an 8-lane group one slice, lane l
// its row.  Every column / value load of a group is one 32 B sector (FP32,
// int32) or two (FP64), and the 8 gathers of the input vector for entry k hit
// the columns of 8 neighbouring rows -- for stencil-like matrices and their
// incomplete factors, consecutive addresses.  Slices of 8 rather than 32 rows
// keep the padding small when row lengths vary (threshold factors), while the
// DRAM sector stays fully used.  Each lane keeps 8 entries in flight
// (unrolled), enough bytes per SM to run at the HBM roofline: per entry 4 B
// column + 4 B (FP32) or 8 B (FP64) value.
#include "bsg_internal.cuh"
#include <cub/device/device_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#define SELL_C 8

namespace {

__global__ void k_sell_width(int n, const int *rp, int skip, const int *perm, long long *width) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int slice = t / SELL_C;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int r = t < n ? (perm ? perm[t] : t) : n; // one thread per row slot
	int len = r < n ? rp[r + 1] - rp[r] - skip : 0;
	if (len < 0) len = 0;
#pragma unroll
	for (int o = SELL_C / 2; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, o, SELL_C));
	if ((t % SELL_C) == 0 && slice < nsl) width[slice] = (long long)SELL_C * len;
}

template <typename VT>
__global__ void k_sell_fill(int n, const int *rp, const int *ci, const double *v, int skip, const int *perm,
                            const long long *off, int *scol, VT *sval) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int slice = t / SELL_C, l = t % SELL_C;
	if (slice >= nsl) return;
	const int r = t < n ? (perm ? perm[t] : t) : n;
	const long long base = off[slice];
	const int w = (int)((off[slice + 1] - base) / SELL_C);
	const int b = r < n ? rp[r] + skip : 0;
	const int len = r < n ? rp[r + 1] - b : 0;
	for (int k = 0; k < w; k++) {
		const long long p = base + (long long)SELL_C * k + l;
		if (k < len) {
			scol[p] = ci[b + k];
			sval[p] = (VT)v[b + k];
		} else {
			scol[p] = r < n ? r : 0;
			sval[p] = (VT)0;
		}
	}
}

// y = A x (OUT 0) or y = (x - N yin) * dinv (OUT 1); IN 1 forms
// yin[c] = x[c] * dinv[c] on the fly (the first two Jacobi iterates in one
// pass).
template <typename VT, int IN, int OUT>
__global__ void __launch_bounds__(256) k_sell_apply(int n, const int *__restrict__ perm,
                                                    const long long *__restrict__ off,
                                                    const int *__restrict__ scol, const VT *__restrict__ sval,
                                                    const double *__restrict__ xin, const double *__restrict__ dinv_in,
                                                    const double *__restrict__ xrhs,
                                                    const double *__restrict__ dinv_out, double *__restrict__ y) {
	constexpr int SPW = 32 / SELL_C; // slices per warp
	const int lane = threadIdx.x & 31;
	const int grp = lane / SELL_C, l = lane % SELL_C;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int s0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * SPW; s0 < nsl; s0 += nwarps * SPW) {
		const int slice = s0 + grp;
		if (slice >= nsl) continue;
		const long long base = __ldg(off + slice);
		const int w = (int)((__ldg(off + slice + 1) - base) / SELL_C);
		const int *cp = scol + base + l;
		const VT *vp = sval + base + l;
		double sum = 0.0;
		int k = 0;
		for (; k + 8 <= w; k += 8) {
			int c[8];
			double a[8], xv[8];
#pragma unroll
			for (int u = 0; u < 8; u++) {
				c[u] = __ldcs(cp + SELL_C * (k + u));
				a[u] = (double)__ldcs(vp + SELL_C * (k + u));
			}
#pragma unroll
			for (int u = 0; u < 8; u++) {
				xv[u] = __ldg(xin + c[u]);
				if (IN == 1) xv[u] *= __ldg(dinv_in + c[u]);
			}
#pragma unroll
			for (int u = 0; u < 8; u++) sum = fma(a[u], xv[u], sum);
		}
		for (; k < w; k++) {
			const int c = __ldcs(cp + SELL_C * k);
			const double a = (double)__ldcs(vp + SELL_C * k);
			double xv = __ldg(xin + c);
			if (IN == 1) xv *= __ldg(dinv_in + c);
			sum = fma(a, xv, sum);
		}
		const int t = slice * SELL_C + l;
		if (t < n) {
			const int r = perm ? __ldg(perm + t) : t;
			if (OUT == 0) y[r] = sum;
			else y[r] = (xrhs[r] - sum) * dinv_out[r];
		}
	}
}

// One Jacobi pass of an FP32 factor with FP32 iterates: out = (rhs - N x32)
// * dinv, written as FP64 (the last pass, OUT64 1) or as the FP32 iterate the
// next pass gathers (OUT64 0).  Gathering 4-byte iterates halves the
// sector traffic of the gathers; the products and sums stay FP64.
template <int OUT64>
__global__ void __launch_bounds__(256) k_sell_sweep32(int n, const int *__restrict__ perm,
                                                      const long long *__restrict__ off,
                                                      const int *__restrict__ scol, const float *__restrict__ sval,
                                                      const float *__restrict__ x32, const double *__restrict__ rhs,
                                                      const double *__restrict__ dinv, double *__restrict__ y,
                                                      float *__restrict__ y32) {
	constexpr int SPW = 32 / SELL_C;
	const int lane = threadIdx.x & 31;
	const int grp = lane / SELL_C, l = lane % SELL_C;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int s0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * SPW; s0 < nsl; s0 += nwarps * SPW) {
		const int slice = s0 + grp;
		if (slice >= nsl) continue;
		const long long base = __ldg(off + slice);
		const int w = (int)((__ldg(off + slice + 1) - base) / SELL_C);
		const int *cp = scol + base + l;
		const float *vp = sval + base + l;
		double sum = 0.0;
		int k = 0;
		for (; k + 8 <= w; k += 8) {
			int c[8];
			float a[8], xv[8];
#pragma unroll
			for (int u = 0; u < 8; u++) {
				c[u] = __ldcs(cp + SELL_C * (k + u));
				a[u] = __ldcs(vp + SELL_C * (k + u));
			}
#pragma unroll
			for (int u = 0; u < 8; u++) xv[u] = __ldg(x32 + c[u]);
#pragma unroll
			for (int u = 0; u < 8; u++) sum = fma((double)a[u], (double)xv[u], sum);
		}
		for (; k < w; k++) {
			const int c = __ldcs(cp + SELL_C * k);
			sum = fma((double)__ldcs(vp + SELL_C * k), (double)__ldg(x32 + c), sum);
		}
		const int t = slice * SELL_C + l;
		if (t < n) {
			const int r = perm ? __ldg(perm + t) : t;
			const double v = (rhs[r] - sum) * dinv[r];
			if (OUT64) y[r] = v;
			else y32[r] = (float)v;
		}
	}
}

// x32 = x * dinv rounded to FP32 (the first Jacobi iterate)
__global__ void k_scale32(int n, const double *x, const double *dinv, float *x32) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		x32[i] = (float)(x[i] * dinv[i]);
}

inline int nb(long long n, int t) { return n > 0 ? (int)((n + t - 1) / t) : 1; }

} // namespace

// Build SELL-8 of a CSR matrix (device arrays); skip = 1 drops the first
// entry of every row (the diagonal of a factor row).  Values are stored as VT.
__global__ void k_len_keys(int n, const int *rp, int skip, int sigma, unsigned long long *keys, int *vals) {
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= n) return;
	int len = rp[r + 1] - rp[r] - skip;
	if (len < 0) len = 0;
	if (len > 0xfffff) len = 0xfffff;
	// window ascending, then longer rows first, then row index (stable)
	keys[r] = ((unsigned long long)(r / sigma) << 20) | (unsigned long long)(0xfffff - len);
	vals[r] = r;
}

template <typename VT>
int bsg_sell_build_t(bsg_ctx *c, int n, const int *rp, const int *ci, const double *v, int skip, bsg_sell *out,
                     int sigma) {
	cudaStream_t s = c->stream;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	out->perm = nullptr;
	if (sigma > 0 && n > 0) {
		// SELL-C-sigma: rows sorted by length inside windows of sigma rows
		unsigned long long *keys, *k2;
		int *vals;
		BSG_CUDA(cudaMallocAsync(&keys, sizeof(unsigned long long) * n, s));
		BSG_CUDA(cudaMallocAsync(&k2, sizeof(unsigned long long) * n, s));
		BSG_CUDA(cudaMallocAsync(&vals, sizeof(int) * n, s));
		BSG_CUDA(cudaMallocAsync(&out->perm, sizeof(int) * n, s));
		BSG_COUNT(1);
		k_len_keys<<<nb(n, 256), 256, 0, s>>>(n, rp, skip, sigma, keys, vals);
		size_t t2 = 0;
		int end_bit = 20;
		while ((1ull << (end_bit - 20)) <= (unsigned long long)(n / sigma + 1)) end_bit++;
		BSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t2, keys, k2, vals, out->perm, n, 0, end_bit, s));
		void *d_t2;
		BSG_CUDA(cudaMallocAsync(&d_t2, t2 > 0 ? t2 : 1, s));
		BSG_CUDA(cub::DeviceRadixSort::SortPairs(d_t2, t2, keys, k2, vals, out->perm, n, 0, end_bit, s));
		cudaFreeAsync(keys, s); cudaFreeAsync(k2, s); cudaFreeAsync(vals, s); cudaFreeAsync(d_t2, s);
	}
	long long *width;
	BSG_CUDA(cudaMallocAsync(&width, sizeof(long long) * (nsl + 1), s));
	BSG_CUDA(cudaMallocAsync(&out->off, sizeof(long long) * (nsl + 1), s));
	BSG_CUDA(cudaMemsetAsync(width + nsl, 0, sizeof(long long), s));
	BSG_COUNT(2);
	k_sell_width<<<nb((long long)nsl * SELL_C, 256), 256, 0, s>>>(n, rp, skip, out->perm, width);
	// off = exclusive scan of the slice sizes
	size_t tmp = 0;
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, width, out->off, nsl + 1, s));
	void *d_tmp;
	BSG_CUDA(cudaMallocAsync(&d_tmp, tmp > 0 ? tmp : 1, s));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, width, out->off, nsl + 1, s));
	long long total = 0;
	BSG_CUDA(cudaMemcpyAsync(&total, out->off + nsl, sizeof(long long), cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	out->n = n;
	out->entries = total;
	BSG_CUDA(cudaMallocAsync(&out->col, sizeof(int) * (total > 0 ? total : 1), s));
	BSG_CUDA(cudaMallocAsync(&out->val, sizeof(VT) * (total > 0 ? total : 1), s));
	out->fp32 = sizeof(VT) == 4;
	k_sell_fill<VT><<<nb((long long)nsl * SELL_C, 256), 256, 0, s>>>(n, rp, ci, v, skip, out->perm, out->off,
	                                                                out->col, (VT *)out->val);
	BSG_CUDA(cudaGetLastError());
	BSG_CUDA(cudaFreeAsync(width, s));
	BSG_CUDA(cudaFreeAsync(d_tmp, s));
	return BSG_OK;
}

int bsg_sell_build(bsg_ctx *c, int n, const int *rp, const int *ci, const double *v, int skip, int fp32,
                   bsg_sell *out, int sigma) {
	return fp32 ? bsg_sell_build_t<float>(c, n, rp, ci, v, skip, out, sigma)
	            : bsg_sell_build_t<double>(c, n, rp, ci, v, skip, out, sigma);
}

void bsg_sell_free(bsg_sell *m, cudaStream_t s) {
	if (m->perm) cudaFreeAsync(m->perm, s);
	m->perm = nullptr;
	if (m->off) cudaFreeAsync(m->off, s);
	if (m->col) cudaFreeAsync(m->col, s);
	if (m->val) cudaFreeAsync(m->val, s);
	m->off = nullptr;
	m->col = nullptr;
	m->val = nullptr;
}

static int sell_grid(int n) {
	int warps = (n + 31) / 32;
	int blocks = (warps + 7) / 8;
	int cap = BSG_SMS * 8;
	return blocks < 1 ? 1 : (blocks < cap ? blocks : cap);
}

// y = A x
int bsg_sell_spmv(cudaStream_t s, const bsg_sell *m, const double *x, double *y) {
	BSG_COUNT(1);
	if (m->fp32)
		k_sell_apply<float, 0, 0><<<sell_grid(m->n), 256, 0, s>>>(m->n, m->perm, m->off, m->col, (const float *)m->val, x,
		                                                          nullptr, nullptr, nullptr, y);
	else
		k_sell_apply<double, 0, 0><<<sell_grid(m->n), 256, 0, s>>>(m->n, m->perm, m->off, m->col, (const double *)m->val, x,
		                                                           nullptr, nullptr, nullptr, y);
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}

// One Jacobi pass yout = (x - N yin) * dinv; scaled_in: yin = x * dinv.
int bsg_sell_sweep(cudaStream_t s, const bsg_sell *m, const double *x, const double *dinv, const double *yin,
                   int scaled_in, double *yout) {
	BSG_COUNT(1);
	const int g = sell_grid(m->n);
	if (m->fp32) {
		const float *v = (const float *)m->val;
		if (scaled_in) k_sell_apply<float, 1, 1><<<g, 256, 0, s>>>(m->n, m->perm, m->off, m->col, v, x, dinv, x, dinv, yout);
		else k_sell_apply<float, 0, 1><<<g, 256, 0, s>>>(m->n, m->perm, m->off, m->col, v, yin, nullptr, x, dinv, yout);
	} else {
		const double *v = (const double *)m->val;
		if (scaled_in) k_sell_apply<double, 1, 1><<<g, 256, 0, s>>>(m->n, m->perm, m->off, m->col, v, x, dinv, x, dinv, yout);
		else k_sell_apply<double, 0, 1><<<g, 256, 0, s>>>(m->n, m->perm, m->off, m->col, v, yin, nullptr, x, dinv, yout);
	}
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}

// Jacobi sweeps of an FP32 factor with FP32 iterates: nsweeps >= 2 iterates
// in total (the first, D^-1 x, formed by k_scale32), the last written to
// yout in FP64.  work32 holds 2 n floats (the ping-pong iterates).
int bsg_sell_sweeps32(cudaStream_t s, const bsg_sell *m, const double *x, const double *dinv, int nsweeps,
                      float *work32, double *yout) {
	if (!m->fp32 || nsweeps < 2) return BSG_ERR_ARG;
	const int n = m->n, g = sell_grid(n);
	const float *v = (const float *)m->val;
	float *a = work32, *b = work32 + n;
	BSG_COUNT(nsweeps);
	k_scale32<<<nb(n, 256) < BSG_SMS * 16 ? nb(n, 256) : BSG_SMS * 16, 256, 0, s>>>(n, x, dinv, b);
	for (int pass = 0; pass < nsweeps - 1; pass++) {
		const bool last = pass == nsweeps - 2;
		if (last) k_sell_sweep32<1><<<g, 256, 0, s>>>(n, m->perm, m->off, m->col, v, b, x, dinv, yout, nullptr);
		else k_sell_sweep32<0><<<g, 256, 0, s>>>(n, m->perm, m->off, m->col, v, b, x, dinv, nullptr, a);
		float *t = a; a = b; b = t;
	}
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}

// One full FP32-iterate pass (timing of the sweep kernel alone).
int bsg_sell_sweep32_pass(cudaStream_t s, const bsg_sell *m, const double *x, const double *dinv, const float *x32,
                          double *yout) {
	BSG_COUNT(1);
	k_sell_sweep32<1><<<sell_grid(m->n), 256, 0, s>>>(m->n, m->perm, m->off, m->col, (const float *)m->val, x32, x, dinv,
	                                                  yout, nullptr);
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}

// Stored entries (with padding) of a SELL matrix: the bytes a product reads.
long long bsg_sell_entries(const bsg_sell *m) { return m->entries; }
