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
//   * 3x3 block CSR: one warp per block row; 27 lanes at fixed (block, row,
//     column) positions read the row's values 27 at a time (coalesced), then
//     two shuffle rounds give the three output rows.
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
// A warp takes a block row.  Lanes 0..26 hold fixed positions lane = 9 t + 3 r
// + c (block t of three, row r, column c) and step through the row three
// blocks at a time, so each step reads 27 contiguous values and gathers three
// 24-byte pieces of x; U steps' loads are issued before their products.  The
// sums over c and then over t are two shuffle rounds, and lanes 0, 3, 6 hold
// the three output rows.  nr <= K vectors at stride ld share each value load;
// each vector's sums are formed in the same order whatever K is.
template <int K>
__global__ void __launch_bounds__(256, K > 4 ? 4 : (K > 2 ? 5 : 8)) k_spmv_bsr3(int nb, int nr, const int *__restrict__ ia,
                                                   const int *__restrict__ ja, const double *__restrict__ a,
                                                   const double *__restrict__ X, double *__restrict__ Y,
                                                   long long ld) {
	const int lane = threadIdx.x & 31;
	const int t = lane / 9, w = lane - 9 * (lane / 9), c = w % 3;
	const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	constexpr int U = 4;
	for (int br = warp; br < nb; br += nwarps) {
		const int b = __ldg(ia + br), e = lane < 27 ? __ldg(ia + br + 1) : b;
		double s[K];
#pragma unroll
		for (int q = 0; q < K; q++) s[q] = 0.0;
		int j = b + t;
		for (; j + 3 * (U - 1) < e; j += 3 * U) {
			double v[U];
			int J[U];
#pragma unroll
			for (int u = 0; u < U; u++) {
				v[u] = ld_stream(a + 9LL * (j + 3 * u) + w);
				J[u] = __ldg(ja + j + 3 * u);
			}
#pragma unroll
			for (int u = 0; u < U; u++)
#pragma unroll
				for (int q = 0; q < K; q++)
					if (q < nr) s[q] = fma(v[u], __ldg(X + q * ld + 3LL * J[u] + c), s[q]);
		}
		for (; j < e; j += 3) {
			const double v = ld_stream(a + 9LL * j + w);
			const long long J = 3LL * __ldg(ja + j) + c;
#pragma unroll
			for (int q = 0; q < K; q++)
				if (q < nr) s[q] = fma(v, __ldg(X + q * ld + J), s[q]);
		}
#pragma unroll
		for (int q = 0; q < K; q++) {
			if (q >= nr) break;
			double v = s[q] + __shfl_down_sync(0xffffffffu, s[q], 1);
			v += __shfl_down_sync(0xffffffffu, s[q], 2);
			double u = v + __shfl_down_sync(0xffffffffu, v, 9);
			u += __shfl_down_sync(0xffffffffu, v, 18);
			if (lane < 9 && c == 0) Y[q * ld + 3LL * br + w / 3] = u;
		}
	}
}

template <int K>
int bsr3_grid(int nb) {
	static int cap = 0;
	if (!cap) {
		int per_sm = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmv_bsr3<K>, 256, 0);
		cap = (per_sm > 0 ? per_sm : 1) * BSG_SMS;
	}
	const int g = (nb + 7) / 8; // a warp per block row, 8 warps a block
	return g < 1 ? 1 : (g < cap ? g : cap);
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
		for (int r0 = 0; r0 < nrhs; r0 += 8) {
			BSG_COUNT(1);
			const int k = nrhs - r0 < 8 ? nrhs - r0 : 8;
			const double *Xr = X + r0 * ld;
			double *Yr = Y + r0 * ld;
			if (k == 1) k_spmv_bsr3<1><<<bsr3_grid<1>(m->n), 256, 0, s>>>(m->n, k, m->d_ia, m->d_ja, m->d_a, Xr, Yr, ld);
			else if (k == 2) k_spmv_bsr3<2><<<bsr3_grid<2>(m->n), 256, 0, s>>>(m->n, k, m->d_ia, m->d_ja, m->d_a, Xr, Yr, ld);
			else if (k <= 4) k_spmv_bsr3<4><<<bsr3_grid<4>(m->n), 256, 0, s>>>(m->n, k, m->d_ia, m->d_ja, m->d_a, Xr, Yr, ld);
			else k_spmv_bsr3<8><<<bsr3_grid<8>(m->n), 256, 0, s>>>(m->n, k, m->d_ia, m->d_ja, m->d_a, Xr, Yr, ld);
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
