// Sparse matrix-vector products of the solver path, FP64 (the reference's
// CSMatrixR::MvmA Bslib/mvm.cpp:2489 and CSMatrixRS::MvmA :2530; the
// symmetric MvmASymm forms :2637/:3008 run as gather products over the
// expanded matrix).
//
// HBM roofline: one pass over the matrix (8 B value + 4 B column per point
// entry, 72 B + 4 B per 3x3 block), the row pointers, and x/y once each.
//   * point CSR: a sub-warp of G lanes per row (G chosen from the mean row
//     length); consecutive rows of a warp read one contiguous stretch of
//     ja/a, so the stream loads are fully coalesced; x is gathered through
//     the read-only path and stays in L2 (<= 16.8 MB at n = 2.1M).
//   * 3x3 block CSR: one warp per block row walks the row's contiguous
//     9*nblocks values element by element (coalesced), accumulating the three
//     output rows, then three warp reductions.
//   * multi-RHS: the same sweeps carry K right-hand sides so the matrix is
//     read once for all of them.
#include "bsg_internal.cuh"
#include "k_stream.cuh"

namespace {

// Point CSR, one right-hand side: row-chunk streaming (k_stream.cuh).
__global__ void __launch_bounds__(256) k_spmv_stream(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                                     const double *__restrict__ a, const double *__restrict__ x,
                                                     double *__restrict__ y) {
	__shared__ double prod[8][STREAM_CAP];
	stream_rows<double, IN_VEC, OUT_SUM>(n, ia, ja, a, 0, x, nullptr, nullptr, nullptr, y, prod[threadIdx.x >> 5]);
}

__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ int ld_stream(const int *p) { return __ldcs(p); }

template <int G>
__global__ void __launch_bounds__(256) k_spmv_csr(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                                  const double *__restrict__ a, const double *__restrict__ x,
                                                  double *__restrict__ y) {
	const int lane32 = threadIdx.x & 31;
	const int lane = lane32 & (G - 1);
	const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	constexpr int RPW = 32 / G;
	for (int r0 = warp * RPW; r0 < n; r0 += nwarps * RPW) {
		int row = r0 + lane32 / G;
		double s = 0.0;
		if (row < n) {
			int b = ia[row], e = ia[row + 1];
			for (int k = b + lane; k < e; k += G) s = fma(ld_stream(a + k), __ldg(x + ld_stream(ja + k)), s);
		}
		s = group_sum<G>(s);
		if (row < n && lane == 0) y[row] = s;
	}
}

// Multi-RHS point SpMM: Y[:,r] = A X[:,r], r < K (K <= 8), vectors at stride ld.
template <int G, int K>
__global__ void __launch_bounds__(256) k_spmm_csr(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                                  const double *__restrict__ a, const double *__restrict__ X,
                                                  double *__restrict__ Y, long long ld) {
	const int lane32 = threadIdx.x & 31;
	const int lane = lane32 & (G - 1);
	const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	constexpr int RPW = 32 / G;
	for (int r0 = warp * RPW; r0 < n; r0 += nwarps * RPW) {
		int row = r0 + lane32 / G;
		double s[K];
#pragma unroll
		for (int r = 0; r < K; r++) s[r] = 0.0;
		if (row < n) {
			int b = ia[row], e = ia[row + 1];
			for (int k = b + lane; k < e; k += G) {
				double v = ld_stream(a + k);
				int c = ld_stream(ja + k);
#pragma unroll
				for (int r = 0; r < K; r++) s[r] = fma(v, __ldg(X + r * ld + c), s[r]);
			}
		}
#pragma unroll
		for (int r = 0; r < K; r++) s[r] = group_sum<G>(s[r]);
		if (row < n && lane == 0) {
#pragma unroll
			for (int r = 0; r < K; r++) Y[r * ld + row] = s[r];
		}
	}
}

// 3x3 block rows, device blocks row-major (element (r,c) at 9*blk + 3*r + c).
template <int K>
__global__ void __launch_bounds__(256) k_spmv_bsr3(int nb, const int *__restrict__ ia, const int *__restrict__ ja,
                                                   const double *__restrict__ a, const double *__restrict__ X,
                                                   double *__restrict__ Y, long long ld) {
	const int lane = threadIdx.x & 31;
	const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int br = warp; br < nb; br += nwarps) {
		const int b = ia[br], e = ia[br + 1];
		const int nv = (e - b) * 9;
		const double *av = a + (size_t)b * 9;
		double s0[K], s1[K], s2[K];
#pragma unroll
		for (int r = 0; r < K; r++) s0[r] = s1[r] = s2[r] = 0.0;
		for (int t = lane; t < nv; t += 32) {
			int blk = t / 9;
			int w = t - 9 * blk;
			int rr = w / 3;
			int cc = w - 3 * rr;
			double v = ld_stream(av + t);
			int col = 3 * __ldg(ja + b + blk) + cc;
#pragma unroll
			for (int r = 0; r < K; r++) {
				double p = v * __ldg(X + r * ld + col);
				s0[r] += rr == 0 ? p : 0.0;
				s1[r] += rr == 1 ? p : 0.0;
				s2[r] += rr == 2 ? p : 0.0;
			}
		}
#pragma unroll
		for (int r = 0; r < K; r++) {
			double t0 = warp_sum(s0[r]), t1 = warp_sum(s1[r]), t2 = warp_sum(s2[r]);
			if (lane == 0) {
				Y[r * ld + 3 * br + 0] = t0;
				Y[r * ld + 3 * br + 1] = t1;
				Y[r * ld + 3 * br + 2] = t2;
			}
		}
	}
}

int grid_for(int warps_needed) {
	int blocks = (warps_needed + 7) / 8;           // 8 warps per 256-thread block
	int cap = BSG_SMS * 8;                          // 8 resident blocks per SM
	return blocks < cap ? (blocks > 0 ? blocks : 1) : cap;
}

} // namespace

int bsg_choose_group(double mean_row) {
	if (mean_row <= 5.0) return 4;
	if (mean_row <= 12.0) return 8;
	if (mean_row <= 24.0) return 16;
	return 32;
}

int bsg_spmm_launch(const bsg_mat *m, int nrhs, const double *X, double *Y, long long ld, cudaStream_t s) {
	if (m->bs == 3) {
		int g = grid_for(m->n);
		for (int r0 = 0; r0 < nrhs;) {
			BSG_COUNT(1);
			int k = nrhs - r0;
			const double *Xr = X + r0 * ld;
			double *Yr = Y + r0 * ld;
			if (k >= 4) { k_spmv_bsr3<4><<<g, 256, 0, s>>>(m->n, m->d_ia, m->d_ja, m->d_a, Xr, Yr, ld); r0 += 4; }
			else if (k >= 2) { k_spmv_bsr3<2><<<g, 256, 0, s>>>(m->n, m->d_ia, m->d_ja, m->d_a, Xr, Yr, ld); r0 += 2; }
			else { k_spmv_bsr3<1><<<g, 256, 0, s>>>(m->n, m->d_ia, m->d_ja, m->d_a, Xr, Yr, ld); r0 += 1; }
		}
		return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
	}
	if (m->bs != 1) return BSG_ERR_UNSUPPORTED;
	if (nrhs == 1) {
		if (m->sell.off) return bsg_sell_spmv(s, &m->sell, X, Y);
		BSG_COUNT(1);
		int warps = (m->n + STREAM_ROWS - 1) / STREAM_ROWS;
		k_spmv_stream<<<grid_for(warps), 256, 0, s>>>(m->n, m->d_ia, m->d_ja, m->d_a, X, Y);
		return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
	}
	const int G = m->group;
	const int rows_per_warp = 32 / G;
	int g = grid_for((m->n + rows_per_warp - 1) / rows_per_warp);
	for (int r0 = 0; r0 < nrhs;) {
		BSG_COUNT(1);
		int k = nrhs - r0;
		const double *Xr = X + r0 * ld;
		double *Yr = Y + r0 * ld;
#define BSG_SPMM_CASE(GG)                                                                                   \
	if (G == GG) {                                                                                          \
		if (k == 1) { k_spmv_csr<GG><<<g, 256, 0, s>>>(m->n, m->d_ia, m->d_ja, m->d_a, Xr, Yr); r0 += 1; }   \
		else if (k < 4) { k_spmm_csr<GG, 2><<<g, 256, 0, s>>>(m->n, m->d_ia, m->d_ja, m->d_a, Xr, Yr, ld); r0 += 2; } \
		else { k_spmm_csr<GG, 4><<<g, 256, 0, s>>>(m->n, m->d_ia, m->d_ja, m->d_a, Xr, Yr, ld); r0 += 4; } \
		continue;                                                                                           \
	}
		BSG_SPMM_CASE(4)
		BSG_SPMM_CASE(8)
		BSG_SPMM_CASE(16)
		BSG_SPMM_CASE(32)
#undef BSG_SPMM_CASE
		return BSG_ERR_ARG;
	}
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}

int bsg_spmv_launch(const bsg_mat *m, const double *x, double *y, cudaStream_t s) {
	return bsg_spmm_launch(m, 1, x, y, (long long)m->n * m->bs, s);
}
