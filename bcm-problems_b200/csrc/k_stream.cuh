// Row-chunk streaming for short-row CSR products (SpMV y = A x and the
// Jacobi sweeps of the triangular solves, y = D^{-1}(x - N y_in)).
//
// A warp owns 32 consecutive rows.  Their entries are one contiguous stretch
// [rp[r0], rp[r0 + 32]) of the column / value arrays; the warp streams that
// stretch with every lane issuing up to 8 independent column loads, 8 value
// loads and then 8 gathers of the input vector before it waits, writes the
// products to a shared buffer, and finally lane l sums row r0 + l from the
// buffer.  Compared with a sub-warp per row this keeps ~8x more bytes in
// flight per SM, which is what an HBM-bound product with 7-30 entries per row
// needs to approach the bandwidth roofline.
#pragma once
#include "bsg_internal.cuh"

#define STREAM_ROWS 32
#define STREAM_CAP 256 // products buffered per warp per pass (8 per lane)
#define STREAM_UNROLL 8

// How the input vector entry for column c is formed.
enum StreamIn { IN_VEC = 0, IN_SCALED = 1 }; // y_in[c]  or  x[c] * dinv[c]
// What the row sum becomes.
enum StreamOut { OUT_SUM = 0, OUT_SWEEP = 1 }; // y = s  or  y = (x - s) * dinv

template <typename VT, int IN, int OUT>
__device__ __forceinline__ void stream_rows(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                            const VT *__restrict__ v, int skip, const double *__restrict__ xin,
                                            const double *__restrict__ dinv_in, const double *__restrict__ xrhs,
                                            const double *__restrict__ dinv_out, double *__restrict__ y,
                                            double *prod /* shared, STREAM_CAP */) {
	const int lane = threadIdx.x & 31;
	const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int r0 = warp * STREAM_ROWS; r0 < n; r0 += nwarps * STREAM_ROWS) {
		const int row = r0 + lane;
		const int rlast = min(r0 + STREAM_ROWS, n);
		const int b = (row < n) ? __ldg(rp + row) : 0;
		const int e = (row < n) ? __ldg(rp + row + 1) : 0;
		const int s0 = __shfl_sync(0xffffffffu, b, 0);
		const int s1 = __shfl_sync(0xffffffffu, e, rlast - r0 - 1);
		double sum = 0.0;
		for (int base = s0; base < s1; base += STREAM_CAP) {
			const int cnt = min(STREAM_CAP, s1 - base);
			for (int k0 = 0; k0 < cnt; k0 += 32 * STREAM_UNROLL) {
				int c[STREAM_UNROLL];
				double a[STREAM_UNROLL], xv[STREAM_UNROLL];
#pragma unroll
				for (int u = 0; u < STREAM_UNROLL; u++) {
					const int k = k0 + u * 32 + lane;
					c[u] = 0;
					a[u] = 0.0;
					if (k < cnt) {
						c[u] = __ldcs(ci + base + k);
						a[u] = (double)__ldcs(v + base + k);
					}
				}
#pragma unroll
				for (int u = 0; u < STREAM_UNROLL; u++) {
					if (IN == IN_VEC) xv[u] = __ldg(xin + c[u]);
					else xv[u] = __ldg(xin + c[u]) * __ldg(dinv_in + c[u]);
				}
#pragma unroll
				for (int u = 0; u < STREAM_UNROLL; u++) {
					const int k = k0 + u * 32 + lane;
					if (k < cnt) prod[k] = a[u] * xv[u];
				}
			}
			__syncwarp();
			if (row < n) {
				const int lo = max(b + skip, base), hi = min(e, base + cnt);
				for (int k = lo; k < hi; k++) sum += prod[k - base];
			}
			__syncwarp();
		}
		if (row < n) {
			if (OUT == OUT_SUM) y[row] = sum;
			else y[row] = (xrhs[row] - sum) * dinv_out[row];
		}
	}
}
