// Triangular solves with an IC2 / ILU2 factor (CSMatrixR::SolveL,
// Bslib/mvm.cpp:3042 -- L by columns, inverse pivot first; SolveU, :3343 --
// U by rows, inverse pivot first).
//
// The column-stored L is turned into rows (gather form) once per factor, so
// both solves read their factor rows contiguously:
//   forward  y_i = dinv_l[i] * (x_i - sum_{k<i} L(i,k) y_k)
//   backward y_i = dinv_u[i] * (x_i - sum_{k>i} U(i,k) y_k)
//
// mode 0 -- exact, sync-free: a warp solves one row; warps claim rows in
//   dependency order (ascending for L, descending for U) from an atomic
//   counter, and each lane waits on the entry it needs.  "Solved" is encoded
//   in the value itself: y is pre-filled with a NaN bit pattern no arithmetic
//   produces, and a 64-bit store publishes the result in one transaction.
//   Every wait is bounded by globaltimer (BSG_ERR_TIMEOUT).
// mode 1 -- Jacobi sweeps: y <- D^{-1}(x - N y) repeated nsweeps times from
//   y = D^{-1} x; every sweep is a fully parallel pass over the factor (HBM
//   bound: 4 B value (FP32) or 8 B (FP64) + 4 B column per entry).  It applies
//   a fixed polynomial in the factor, so it is a valid flexible (FGMRES)
//   preconditioner and, applied symmetrically, a valid PCG preconditioner.
#include "bsg_internal.cuh"
#include "k_stream.cuh"

#ifndef SELL_SIGMA
#define SELL_SIGMA 128 // rows per length-sorting window of the factor's sliced copies
#endif

namespace {

// One Jacobi sweep y_out = D^{-1}(x - N y_in) by row-chunk streaming; with
// IN == IN_SCALED the input is the first iterate D^{-1} x, formed on the fly
// (the first two sweeps in one pass).
template <typename VT, int IN>
__global__ void __launch_bounds__(256) k_trsv_sweep(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                                    const VT *__restrict__ v, int skip,
                                                    const double *__restrict__ dinv, const double *__restrict__ x,
                                                    const double *__restrict__ yin, double *__restrict__ yout) {
	__shared__ double prod[8][STREAM_CAP];
	stream_rows<VT, IN, OUT_SWEEP>(n, rp, ci, v, skip, IN == IN_VEC ? yin : x, dinv, x, dinv, yout,
	                               prod[threadIdx.x >> 5]);
}

__global__ void k_scale_vec(int n, const double *x, const double *d, double *y) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i] * d[i];
}

// Rows are claimed in the order of `perm` (ascending forward-solve level;
// read backwards for U), a topological order of both dependency graphs that
// keeps the rows in flight on the current wavefront.
template <typename VT>
__global__ void __launch_bounds__(256) k_trsv_syncfree(int n, int lower, const int *__restrict__ perm,
                                                       const int *__restrict__ rp, const int *__restrict__ ci,
                                                       const VT *__restrict__ v, int skip_first,
                                                       const double *__restrict__ dinv, const double *__restrict__ x,
                                                       double *y, unsigned *claim, bsg_devstat *st) {
	const int lane = threadIdx.x & 31;
	for (;;) {
		int t = 0;
		if (lane == 0) t = (int)atomicAdd(claim, 1u);
		t = __shfl_sync(0xffffffffu, t, 0);
		if (t >= n) return;
		const int row = perm[lower ? t : n - 1 - t];
		const int b = rp[row] + skip_first, e = rp[row + 1];
		double s = 0.0;
		for (int k = b + lane; k < e; k += 32) {
			const int c = ci[k];
			unsigned long long raw = ld_volatile_u64(y + c);
			if (raw == BSG_PENDING) {
				unsigned long long t0 = globaltimer_ns();
				for (unsigned it = 1;; it++) {
					__nanosleep(32);
					raw = ld_volatile_u64(y + c);
					if (raw != BSG_PENDING) break;
					if ((it & 127) == 0) {
						if (*(volatile int *)&st->code != 0) { raw = 0; break; }
						if (globaltimer_ns() - t0 > BSG_SPIN_LIMIT_NS) {
							devstat_fail(st, BSG_ERR_TIMEOUT, row);
							raw = 0;
							break;
						}
					}
				}
			}
			s = fma((double)v[k], __longlong_as_double((long long)raw), s);
		}
		s = warp_sum(s);
		if (lane == 0) st_volatile_f64(y + row, (x[row] - s) * dinv[row]);
	}
}

template <int G, typename VT>
__global__ void __launch_bounds__(256) k_trsv_jacobi(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                                     const VT *__restrict__ v, int skip_first,
                                                     const double *__restrict__ dinv, const double *__restrict__ x,
                                                     const double *__restrict__ yin, double *__restrict__ yout) {
	const int lane32 = threadIdx.x & 31;
	const int lane = lane32 & (G - 1);
	const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	constexpr int RPW = 32 / G;
	for (int r0 = warp * RPW; r0 < n; r0 += nwarps * RPW) {
		int row = r0 + lane32 / G;
		double s = 0.0;
		if (row < n && yin) {
			int b = rp[row] + skip_first, e = rp[row + 1];
			for (int k = b + lane; k < e; k += G) s = fma((double)__ldcs(v + k), __ldg(yin + __ldcs(ci + k)), s);
		}
		s = group_sum<G>(s);
		if (row < n && lane == 0) yout[row] = (x[row] - s) * dinv[row];
	}
}

__global__ void k_fill_u64(long long n, unsigned long long *p, unsigned long long v) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		p[i] = v;
}

__global__ void k_diag_inv(int n, const int *iu, const double *l, const double *u, double *dl, double *du) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) {
		dl[i] = l[iu[i]];
		du[i] = u[iu[i]];
	}
}

__global__ void k_permute(int nk, const int *perm, const double *src, double *dst) {
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < nk) dst[k] = src[perm[k]];
}

__global__ void k_to_f32(long long nk, const double *src, float *dst) {
	for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nk; k += (long long)gridDim.x * blockDim.x)
		dst[k] = (float)src[k];
}

inline int nb(long long n, int t) { return n > 0 ? (int)((n + t - 1) / t) : 1; }

} // namespace

int bsg_strict_transpose(bsg_ctx *c, int n, const int *ia, const int *ja, int nnz, int **it_o, int **jt_o,
                         int **perm_o, int *nnz_o);
int bsg_choose_group(double mean_row);

// Build the gather forms of a freshly compacted factor.
int bsg_fct_finish(bsg_ctx *c, bsg_fct *f) {
	cudaStream_t s = c->stream;
	const int n = f->n;
	BSG_CUDA(cudaMallocAsync(&f->d_dinv_l, sizeof(double) * n, s));
	BSG_CUDA(cudaMallocAsync(&f->d_dinv_u, sizeof(double) * n, s));
	BSG_COUNT(2); // diagonal inverse + value permutation
	k_diag_inv<<<nb(n, 256), 256, 0, s>>>(n, f->d_iu, f->d_l, f->d_u, f->d_dinv_l, f->d_dinv_u);
	int *perm = nullptr, nk = 0;
	int rc = bsg_strict_transpose(c, n, f->d_iu, f->d_ju, f->nnz, &f->d_lr_i, &f->d_lr_j, &perm, &nk);
	if (rc) return rc;
	f->nnz_strict = nk;
	BSG_CUDA(cudaMallocAsync(&f->d_lr_v, sizeof(double) * (nk > 0 ? nk : 1), s));
	k_permute<<<nb(nk, 256), 256, 0, s>>>(nk, perm, f->d_l, f->d_lr_v);
	BSG_CUDA(cudaFreeAsync(perm, s));
	// strict U rows are the factor rows minus their first (diagonal) entry
	f->d_ur_i = f->d_iu;
	f->d_ur_j = f->d_ju;
	f->d_ur_v = f->d_u;
	// factor rows vary in length from row to row (thresholds): sort them by
	// length inside windows of SELL_SIGMA rows so the slices need little padding
	rc = bsg_sell_build(c, n, f->d_lr_i, f->d_lr_j, f->d_lr_v, 0, 0, &f->sl, SELL_SIGMA);
	if (!rc) rc = bsg_sell_build(c, n, f->d_iu, f->d_ju, f->d_u, 1, 0, &f->su, SELL_SIGMA);
	if (rc) return rc;
	BSG_CUDA(cudaGetLastError());
	BSG_CUDA(cudaStreamSynchronize(s));
	return BSG_OK;
}

int bsg_fct_make_fp32(bsg_fct *f) {
	if (f->fp32) return BSG_OK;
	cudaStream_t s = f->ctx->stream;
	if (f->has_t && f->kind == 1) { // the transposed forms are rebuilt in FP32 on next use
		bsg_sell_free(&f->slt, s);
		bsg_sell_free(&f->sut, s);
		if (f->d_utr_v) cudaFreeAsync(f->d_utr_v, s);
		f->d_utr_v = nullptr;
		f->has_t = 0;
	}
	BSG_CUDA(cudaMallocAsync(&f->d_ur_f, sizeof(float) * (f->nnz > 0 ? f->nnz : 1), s));
	BSG_CUDA(cudaMallocAsync(&f->d_lr_f, sizeof(float) * (f->nnz_strict > 0 ? f->nnz_strict : 1), s));
	BSG_COUNT(2);
	k_to_f32<<<BSG_SMS * 4, 256, 0, s>>>(f->nnz, f->d_u, f->d_ur_f);
	k_to_f32<<<BSG_SMS * 4, 256, 0, s>>>(f->nnz_strict, f->d_lr_v, f->d_lr_f);
	BSG_CUDA(cudaGetLastError());
	// the sweeps read the SELL copies: rebuild them with FP32 values
	bsg_sell_free(&f->sl, s);
	bsg_sell_free(&f->su, s);
	int rc = bsg_sell_build(f->ctx, f->n, f->d_lr_i, f->d_lr_j, f->d_lr_v, 0, 1, &f->sl, SELL_SIGMA, 1);
	if (!rc) rc = bsg_sell_build(f->ctx, f->n, f->d_iu, f->d_ju, f->d_u, 1, 1, &f->su, SELL_SIGMA, 1);
	if (rc) return rc;
	f->fp32 = 1;
	return BSG_OK;
}

int bsg_fill_launch(cudaStream_t s, long long n, double *x, double v);

// One full Jacobi sweep y_out = D^{-1}(x - N y_in) (reads the whole factor);
// used to time the sweep kernel on its own.
int bsg_trisolve_sweep_launch(bsg_ctx *c, const bsg_fct *f, int lower, const double *x, const double *yin,
                              double *yout) {
	if (f->d_bia) return bsg_set_error(BSG_ERR_UNSUPPORTED, "single sweep timing of a block factor");
	const double *dinv = lower ? f->d_dinv_l : f->d_dinv_u;
	if (f->fp32) // the FP32-iterate pass of the mixed path; yin's bytes serve as its FP32 input
		return bsg_sell_sweep32_pass(c->stream, lower ? &f->sl : &f->su, x, dinv, reinterpret_cast<const float *>(yin),
		                             yout);
	return bsg_sell_sweep(c->stream, lower ? &f->sl : &f->su, x, dinv, yin, 0, yout);
}

namespace {
// A triangular operand: its rows (strict part, `skip` leading diagonal
// entries), FP64 / FP32 values, inverse pivots and sliced copy.
struct TriOp {
	int lower;
	const int *rp, *ci;
	int skip;
	const double *vd;
	const float *vf;
	const double *dinv;
	const bsg_sell *sell;
};

int trisolve_impl(bsg_ctx *c, const bsg_fct *f, const TriOp &t, int mode, int nsweeps, const double *x, double *y,
                  double *work) {
	cudaStream_t s = c->stream;
	const int n = f->n;
	const bool use32 = f->fp32 != 0;
	if (mode == 0) {
		BSG_COUNT(2); // fill + solve
		k_fill_u64<<<BSG_SMS * 4, 256, 0, s>>>(n, (unsigned long long *)y, BSG_PENDING);
		unsigned *claim = c->d_counters + 1;
		BSG_CUDA(cudaMemsetAsync(claim, 0, sizeof(unsigned), s));
		int grid = BSG_SMS * 8;
		int need = (n + 7) / 8;
		if (grid > need) grid = need > 0 ? need : 1;
		if (use32)
			k_trsv_syncfree<float><<<grid, 256, 0, s>>>(n, t.lower, f->d_perm, t.rp, t.ci, t.vf, t.skip, t.dinv, x, y, claim,
			                                           c->d_stat);
		else
			k_trsv_syncfree<double><<<grid, 256, 0, s>>>(n, t.lower, f->d_perm, t.rp, t.ci, t.vd, t.skip, t.dinv, x, y,
			                                            claim, c->d_stat);
		return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
	}
	if (nsweeps < 1) nsweeps = 1;
	if (nsweeps > 2 && !work) return BSG_ERR_ARG;
	if (nsweeps == 1) { // the first iterate only: y = D^{-1} x
		BSG_COUNT(1);
		k_scale_vec<<<BSG_SMS * 8, 256, 0, s>>>(n, x, t.dinv, y);
		return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
	}
	if (use32) {
		// FP32 factor: FP32 iterates, ping-ponged in work (2 n floats)
		if (!work) return BSG_ERR_ARG;
		return bsg_sell_sweeps32(s, t.sell, x, t.dinv, nsweeps, reinterpret_cast<float *>(work), y);
	}
	// nsweeps - 1 passes (the first two iterates share one), ping-pong so
	// that the last pass lands in y
	const int passes = nsweeps - 1;
	double *bufs[2] = {y, work};
	int cur = (passes + 1) % 2;
	const double *yin = nullptr;
	for (int p = 0; p < passes; p++) {
		double *out = bufs[cur];
		int rc = bsg_sell_sweep(s, t.sell, x, t.dinv, yin, p == 0, out);
		if (rc) return rc;
		yin = out;
		cur ^= 1;
	}
	return BSG_OK;
}
} // namespace

// Solve with L (lower != 0) or U.  x and y must not alias.  `work` (n
// doubles) is needed for mode 1 with nsweeps > 2, and with nsweeps > 1 for an
// FP32 factor, whose sweeps keep their intermediate iterates in FP32 there.
int bsg_trisolve_launch(bsg_ctx *c, const bsg_fct *f, int lower, int mode, int nsweeps, const double *x, double *y,
                        double *work) {
	if (f->d_bia) return bsg_btrisolve_launch(c, f, lower, mode, nsweeps, x, y, work);
	TriOp t;
	t.lower = lower ? 1 : 0;
	t.rp = lower ? f->d_lr_i : f->d_ur_i;
	t.ci = lower ? f->d_lr_j : f->d_ur_j;
	t.skip = lower ? 0 : 1;
	t.vd = lower ? f->d_lr_v : f->d_ur_v;
	t.vf = lower ? f->d_lr_f : f->d_ur_f;
	t.dinv = lower ? f->d_dinv_l : f->d_dinv_u;
	t.sell = lower ? &f->sl : &f->su;
	return trisolve_impl(c, f, t, mode, nsweeps, x, y, work);
}

// nr solves with one factor, vectors at stride n; work holds n nr doubles
// (needed for sweeps).  Sweeps read the untiled sliced copy once per 8
// vectors and give every vector the bits of a single solve (the tiled FP32
// sweeps sum in the same order); exact solves run one vector at a time.
int bsg_trisolve_multi(bsg_ctx *c, const bsg_fct *f, int lower, int mode, int nsweeps, int nr, const double *x,
                       double *y, double *work) {
	if (f->d_bia) return bsg_btrisolve_multi(c, f, lower, mode, nsweeps, nr, x, y, work);
	const int n = f->n;
	if (nr > 1 && mode != 0 && nsweeps >= 2) {
		if (!work) return bsg_set_error(BSG_ERR_ARG, "sweeps of several vectors: work vector missing");
		const bsg_sell *sl = lower ? &f->sl : &f->su;
		const double *dinv = lower ? f->d_dinv_l : f->d_dinv_u;
		if (f->fp32) return bsg_sell_sweeps32_multi(c->stream, sl, nr, x, dinv, nsweeps, reinterpret_cast<float *>(work), y);
		// FP64: nsweeps - 1 passes, ping-pong so that the last lands in y
		const int passes = nsweeps - 1;
		double *bufs[2] = {y, work};
		int cur = (passes + 1) % 2;
		const double *yin = nullptr;
		for (int p = 0; p < passes; p++) {
			int rc = bsg_sell_sweep_multi(c->stream, sl, nr, x, dinv, yin, p == 0, bufs[cur]);
			if (rc) return rc;
			yin = bufs[cur];
			cur ^= 1;
		}
		return BSG_OK;
	}
	for (int q = 0; q < nr; q++) {
		const size_t o = (size_t)q * n;
		int rc = bsg_trisolve_launch(c, f, lower, mode, nsweeps, x + o, y + o, work ? work + o : nullptr);
		if (rc) return rc;
	}
	return BSG_OK;
}

// The transposed forms of an ILU2 factor: U^T rows are the L-row pattern
// with U's values (the transposition that built the L rows, applied to U),
// L^T rows are U's own pattern with L's values.  IC2 factors need none
// (U^T = L, L^T = U).
static int fct_build_transposes(bsg_ctx *c, bsg_fct *f) {
	if (f->has_t || f->kind == 0) { f->has_t = 1; return BSG_OK; }
	cudaStream_t s = c->stream;
	const int n = f->n;
	int *perm = nullptr, nk = 0, *ti = nullptr, *tj = nullptr;
	int rc = bsg_strict_transpose(c, n, f->d_iu, f->d_ju, f->nnz, &ti, &tj, &perm, &nk);
	if (rc) return rc;
	cudaFreeAsync(ti, s);
	cudaFreeAsync(tj, s);
	BSG_CUDA(cudaMallocAsync(&f->d_utr_v, sizeof(double) * (nk > 0 ? nk : 1), s));
	BSG_COUNT(1);
	k_permute<<<nb(nk, 256), 256, 0, s>>>(nk, perm, f->d_u, f->d_utr_v);
	BSG_CUDA(cudaFreeAsync(perm, s));
	const int fp32 = f->fp32 ? 1 : 0;
	if (fp32) {
		BSG_CUDA(cudaMallocAsync(&f->d_utr_f, sizeof(float) * (nk > 0 ? nk : 1), s));
		BSG_CUDA(cudaMallocAsync(&f->d_l_f, sizeof(float) * (f->nnz > 0 ? f->nnz : 1), s));
		BSG_COUNT(2);
		k_to_f32<<<BSG_SMS * 4, 256, 0, s>>>(nk, f->d_utr_v, f->d_utr_f);
		k_to_f32<<<BSG_SMS * 4, 256, 0, s>>>(f->nnz, f->d_l, f->d_l_f);
	}
	rc = bsg_sell_build(c, n, f->d_lr_i, f->d_lr_j, f->d_utr_v, 0, fp32, &f->slt, SELL_SIGMA, fp32);
	if (!rc) rc = bsg_sell_build(c, n, f->d_iu, f->d_ju, f->d_l, 1, fp32, &f->sut, SELL_SIGMA, fp32);
	if (rc) return rc;
	BSG_CUDA(cudaGetLastError());
	f->has_t = 1;
	return BSG_OK;
}

int bsg_trisolve_t_launch(bsg_ctx *c, bsg_fct *f, int which, int mode, int nsweeps, const double *x, double *y,
                          double *work) {
	if (f->kind == 0) return bsg_trisolve_launch(c, f, which == 0 ? 1 : 0, mode, nsweeps, x, y, work);
	if (f->d_bia) return bsg_set_error(BSG_ERR_UNSUPPORTED, "transposed solves of a block factor");
	int rc = fct_build_transposes(c, f);
	if (rc) return rc;
	TriOp t;
	if (which == 0) { // U^T: lower, L-row pattern, U's values, U's inverse pivots
		t.lower = 1; t.rp = f->d_lr_i; t.ci = f->d_lr_j; t.skip = 0;
		t.vd = f->d_utr_v; t.vf = f->d_utr_f; t.dinv = f->d_dinv_u; t.sell = &f->slt;
	} else {          // L^T: upper, U's pattern, L's values, L's inverse pivots
		t.lower = 0; t.rp = f->d_iu; t.ci = f->d_ju; t.skip = 1;
		t.vd = f->d_l; t.vf = f->d_l_f; t.dinv = f->d_dinv_l; t.sell = &f->sut;
	}
	return trisolve_impl(c, f, t, mode, nsweeps, x, y, work);
}

// this unit's copy of the spin-wait bound (bsg_set_spin_limit_ns)
int bsg_spin_limit_set_trsv(unsigned long long ns) {
	return bsg_spin_limit_set_here(ns) == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}
