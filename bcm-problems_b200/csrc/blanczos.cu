// Block Lanczos of the reference's CSMatrixRS driver: CSVector::
// BlockLanczosCentral / BlockLanczosRight / BlockLanczosLeft
// (Bslib/lanczos.cpp:2467 / :932 / :1719), which CSVector::Solver(CSMatrixRS&)
// runs for ittype 2 / 3 / 4 (Bslib/solvers.cpp:1798-1800).
//
// The method is a block Golub-Kahan bidiagonalisation of the preconditioned
// matrix M with block Givens rotations -- block LSQR -- on nrhs right-hand
// sides at once:
//   central  M = L^{-1} A U^{-1},   start L^{-1} r0,   x = x0 + U^{-1} y
//   right    M = A U^{-1} L^{-1},   start r0,          x = x0 + U^{-1} L^{-1} y
//   left     M = U^{-1} L^{-1} A,   start U^{-1} L^{-1} r0, x = x0 + y
// Recurrences (blocks of nrhs columns; QR = thin QR, R upper):
//   U1 B1 = c;  V1 R1 = M^T U1, alpha1 = R1^T;  W = V1, phibar = B1, rhobar = alpha1
//   each step: U' beta = M V - U alpha;   V' R = M^T U' - V beta^T, alpha = R^T
//              block Givens Q^T [rhobar; beta] = [rho; 0],
//              Q^T [0; alpha] = [theta; rhobar'],  Q^T [phibar; 0] = [phi; phibar']
//              Y += W rho^{-1} phi;  W = V' - W rho^{-1} theta
// and the stop test of the reference: every `ichk` steps the true residual
// of each right-hand side, ||r_j|| < eps ||r0_j|| for all j (the right
// variant also accepts ||M^T r_j|| < eps ||M^T r0_j||).
//
// On the GPU: the block products (A for all columns in one SpMM, A^T, the
// factor's forward / backward and transposed solves), the thin QR as
// classical Gram-Schmidt run twice column by column (multi-dot + update
// kernels), and the nrhs x nrhs block updates in one kernel.  The small
// dense algebra (the 2 nrhs x nrhs Householder QR of the block Givens step,
// triangular solves with rho) runs on the host in FP64.  The reference takes
// rho^{-1} from an SVD; rho is upper triangular, so a back substitution gives
// the same inverse.
#include "bsg_internal.cuh"
#include <cmath>
#include <vector>

int bsg_spmm_launch(const bsg_mat *m, int nrhs, const double *X, double *Y, long long ld, cudaStream_t s);
int bsg_dots_launch(bsg_ctx *c, int q, int n, const double *x0, const double *y0, const double *x1,
                    const double *y1, const double *x2, const double *y2, double *d_out);
int bsg_mdot_launch(bsg_ctx *c, int n, const double *V, long long ld, int k, const double *w, double *d_out);
int bsg_gemv_sub_launch(bsg_ctx *c, int n, const double *V, long long ld, int k, const double *h, double *w);
int bsg_scale_by_launch(bsg_ctx *c, int n, const double *x, double *y, const double *num, const double *den,
                        int sqrt_den);
int bsg_residual_launch(bsg_ctx *c, int n, const double *b, double *r);
int bsg_mvm_t_launch(bsg_ctx *c, bsg_mat *m, const double *x, double *y);

#define BL_MAXRHS 16

namespace {

struct Buf {
	double *p = nullptr;
	cudaStream_t s = nullptr;
	~Buf() { if (p) cudaFreeAsync(p, s); }
};

// Yout[:, j] = beta Yin[:, j] + alpha sum_l W[:, l] C[l][j]  (k <= BL_MAXRHS
// columns of length n, leading dimension n; C row-major k x k on the device).
// Yout may be Yin, not W.
__global__ void k_blk_update(int n, int k, const double *__restrict__ W, const double *__restrict__ C, double alpha,
                             double beta, const double *Yin, double *Yout) {
	__shared__ double sc[BL_MAXRHS * BL_MAXRHS];
	for (int t = threadIdx.x; t < k * k; t += blockDim.x) sc[t] = C[t];
	__syncthreads();
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		double w[BL_MAXRHS];
#pragma unroll
		for (int l = 0; l < BL_MAXRHS; l++)
			if (l < k) w[l] = W[(size_t)l * n + i];
		for (int j = 0; j < k; j++) {
			double acc = 0.0;
#pragma unroll
			for (int l = 0; l < BL_MAXRHS; l++)
				if (l < k) acc = fma(w[l], sc[l * k + j], acc);
			const double y0 = beta != 0.0 ? beta * Yin[(size_t)j * n + i] : 0.0;
			Yout[(size_t)j * n + i] = fma(alpha, acc, y0);
		}
	}
}

int ew_grid(long long n) {
	long long b = (n + 255) / 256;
	long long cap = (long long)BSG_SMS * 8;
	return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

// Small dense helpers (row-major).
using Mat = std::vector<double>;

// Householder QR of the r x c matrix G (r >= c): G = Q [R; 0], Q r x r
// orthogonal (returned), R c x c upper triangular (returned in R).
void house_qr(int r, int c, Mat G, Mat &Q, Mat &R) {
	Q.assign((size_t)r * r, 0.0);
	for (int i = 0; i < r; i++) Q[(size_t)i * r + i] = 1.0;
	std::vector<double> v(r);
	for (int j = 0; j < c; j++) {
		double nrm = 0.0;
		for (int i = j; i < r; i++) nrm += G[(size_t)i * c + j] * G[(size_t)i * c + j];
		nrm = std::sqrt(nrm);
		if (nrm == 0.0) continue;
		const double x0 = G[(size_t)j * c + j];
		const double a = x0 >= 0.0 ? -nrm : nrm;
		for (int i = 0; i < r; i++) v[i] = i < j ? 0.0 : G[(size_t)i * c + j];
		v[j] -= a;
		double vv = 0.0;
		for (int i = j; i < r; i++) vv += v[i] * v[i];
		if (vv == 0.0) continue;
		// G <- H G on columns j.., Q <- Q H
		for (int q = j; q < c; q++) {
			double d = 0.0;
			for (int i = j; i < r; i++) d += v[i] * G[(size_t)i * c + q];
			d = 2.0 * d / vv;
			for (int i = j; i < r; i++) G[(size_t)i * c + q] -= d * v[i];
		}
		for (int i = 0; i < r; i++) {
			double d = 0.0;
			for (int q = j; q < r; q++) d += Q[(size_t)i * r + q] * v[q];
			d = 2.0 * d / vv;
			for (int q = j; q < r; q++) Q[(size_t)i * r + q] -= d * v[q];
		}
	}
	R.assign((size_t)c * c, 0.0);
	for (int i = 0; i < c; i++)
		for (int j = i; j < c; j++) R[(size_t)i * c + j] = G[(size_t)i * c + j];
}

// X = R^{-1} B for R k x k upper triangular (a zero pivot gives a zero row:
// the pseudo-inverse on a direction that carries nothing).
Mat upper_solve(int k, const Mat &R, const Mat &B) {
	Mat X((size_t)k * k, 0.0);
	for (int j = 0; j < k; j++)
		for (int i = k - 1; i >= 0; i--) {
			double s = B[(size_t)i * k + j];
			for (int q = i + 1; q < k; q++) s -= R[(size_t)i * k + q] * X[(size_t)q * k + j];
			const double d = R[(size_t)i * k + i];
			X[(size_t)i * k + j] = d != 0.0 ? s / d : 0.0;
		}
	return X;
}

Mat transpose(int k, const Mat &A) {
	Mat T((size_t)k * k);
	for (int i = 0; i < k; i++)
		for (int j = 0; j < k; j++) T[(size_t)j * k + i] = A[(size_t)i * k + j];
	return T;
}

struct Ctx {
	bsg_ctx *c;
	bsg_mat *m;
	bsg_fct *f;
	const bsg_param *p;
	int n, k, variant;
	double *t1, *t2, *work; // n-vectors
	double *dsm;            // device k x k scratch
	double *dh;             // device scratch of 2k values
};

// Y[:, j] = op(X[:, j]) for each column; op on n-vectors.
template <class F>
int columns(const Ctx &x, const double *X, double *Y, F op) {
	for (int j = 0; j < x.k; j++) {
		int rc = op(X + (size_t)j * x.n, Y + (size_t)j * x.n);
		if (rc) return rc;
	}
	return BSG_OK;
}

int lsolve(const Ctx &x, const double *a, double *b) {
	return bsg_trisolve_launch(x.c, x.f, 1, x.p->trisolve, x.p->nsweeps, a, b, x.work);
}
int usolve(const Ctx &x, const double *a, double *b) {
	return bsg_trisolve_launch(x.c, x.f, 0, x.p->trisolve, x.p->nsweeps, a, b, x.work);
}
int ltsolve(const Ctx &x, const double *a, double *b) { // L^{-T}
	return bsg_trisolve_t_launch(x.c, x.f, 1, x.p->trisolve, x.p->nsweeps, a, b, x.work);
}
int utsolve(const Ctx &x, const double *a, double *b) { // U^{-T}
	return bsg_trisolve_t_launch(x.c, x.f, 0, x.p->trisolve, x.p->nsweeps, a, b, x.work);
}
int amul(const Ctx &x, const double *a, double *b) { return bsg_spmm_launch(x.m, 1, a, b, x.n, x.c->stream); }
int atmul(const Ctx &x, const double *a, double *b) { return bsg_mvm_t_launch(x.c, x.m, a, b); }

// y = M v, one column (variant 2 central, 3 right, 4 left)
int apply_m(const Ctx &x, const double *v, double *y) {
	int rc;
	switch (x.variant) {
	case 2: // L^{-1} A U^{-1}
		rc = usolve(x, v, x.t1);
		if (!rc) rc = amul(x, x.t1, x.t2);
		if (!rc) rc = lsolve(x, x.t2, y);
		return rc;
	case 3: // A U^{-1} L^{-1}
		rc = lsolve(x, v, x.t1);
		if (!rc) rc = usolve(x, x.t1, x.t2);
		if (!rc) rc = amul(x, x.t2, y);
		return rc;
	default: // U^{-1} L^{-1} A
		rc = amul(x, v, x.t1);
		if (!rc) rc = lsolve(x, x.t1, x.t2);
		if (!rc) rc = usolve(x, x.t2, y);
		return rc;
	}
}

// y = M^T u, one column
int apply_mt(const Ctx &x, const double *u, double *y) {
	int rc;
	switch (x.variant) {
	case 2: // U^{-T} A^T L^{-T}
		rc = ltsolve(x, u, x.t1);
		if (!rc) rc = atmul(x, x.t1, x.t2);
		if (!rc) rc = utsolve(x, x.t2, y);
		return rc;
	case 3: // L^{-T} U^{-T} A^T
		rc = atmul(x, u, x.t1);
		if (!rc) rc = utsolve(x, x.t1, x.t2);
		if (!rc) rc = ltsolve(x, x.t2, y);
		return rc;
	default: // A^T L^{-T} U^{-T}
		rc = utsolve(x, u, x.t1);
		if (!rc) rc = ltsolve(x, x.t1, x.t2);
		if (!rc) rc = atmul(x, x.t2, y);
		return rc;
	}
}

// x = x0 + P y (P: U^{-1}, U^{-1} L^{-1}, or I), one column
int apply_back(const Ctx &x, const double *y, double *out) {
	switch (x.variant) {
	case 2:
		return usolve(x, y, out);
	case 3: {
		int rc = lsolve(x, y, x.t1);
		return rc ? rc : usolve(x, x.t1, out);
	}
	default:
		BSG_CUDA(cudaMemcpyAsync(out, y, sizeof(double) * x.n, cudaMemcpyDeviceToDevice, x.c->stream));
		return BSG_OK;
	}
}

// Thin QR of the n x k block X in place (X <- Q), R (k x k, row-major) to
// the host: classical Gram-Schmidt run twice per column.
int block_qr(const Ctx &x, double *X, Mat &R) {
	const int n = x.n, k = x.k;
	R.assign((size_t)k * k, 0.0);
	cudaStream_t s = x.c->stream;
	std::vector<double> h(2 * k + 1);
	for (int j = 0; j < k; j++) {
		double *xj = X + (size_t)j * n;
		int rc = BSG_OK;
		if (j > 0) {
			rc = bsg_mdot_launch(x.c, n, X, n, j, xj, x.dh);
			if (!rc) rc = bsg_gemv_sub_launch(x.c, n, X, n, j, x.dh, xj);
			if (!rc) rc = bsg_mdot_launch(x.c, n, X, n, j, xj, x.dh + k);
			if (!rc) rc = bsg_gemv_sub_launch(x.c, n, X, n, j, x.dh + k, xj);
		}
		if (!rc) rc = bsg_dots_launch(x.c, 1, n, xj, xj, nullptr, nullptr, nullptr, nullptr, x.dh + 2 * k);
		if (!rc) rc = bsg_scale_by_launch(x.c, n, xj, xj, nullptr, x.dh + 2 * k, 1);
		if (rc) return rc;
		BSG_CUDA(cudaMemcpyAsync(h.data(), x.dh, sizeof(double) * (2 * k + 1), cudaMemcpyDeviceToHost, s));
		BSG_CUDA(cudaStreamSynchronize(s));
		for (int i = 0; i < j; i++) R[(size_t)i * k + j] = h[i] + h[k + i];
		R[(size_t)j * k + j] = h[2 * k] > 0.0 ? std::sqrt(h[2 * k]) : 0.0;
	}
	return BSG_OK;
}

// Yout = beta Yin + alpha W C (C k x k row-major, host)
int blk_update(const Ctx &x, const double *W, const Mat &C, double alpha, double beta, const double *Yin, double *Yout) {
	BSG_CUDA(cudaMemcpyAsync(x.dsm, C.data(), sizeof(double) * x.k * x.k, cudaMemcpyHostToDevice, x.c->stream));
	BSG_COUNT(1);
	k_blk_update<<<ew_grid(x.n), 256, 0, x.c->stream>>>(x.n, x.k, W, x.dsm, alpha, beta, Yin, Yout);
	BSG_CUDA(cudaGetLastError());
	// C lives in host memory the caller may change: finish the copy first
	BSG_CUDA(cudaStreamSynchronize(x.c->stream));
	return BSG_OK;
}

// per-column 2-norms of an n x k block (host)
int col_norms(const Ctx &x, const double *X, std::vector<double> &out) {
	out.assign(x.k, 0.0);
	for (int j = 0; j < x.k; j++) {
		int rc = bsg_dots_launch(x.c, 1, x.n, X + (size_t)j * x.n, X + (size_t)j * x.n, nullptr, nullptr, nullptr,
		                         nullptr, x.dh + j);
		if (rc) return rc;
	}
	std::vector<double> h(x.k);
	BSG_CUDA(cudaMemcpyAsync(h.data(), x.dh, sizeof(double) * x.k, cudaMemcpyDeviceToHost, x.c->stream));
	BSG_CUDA(cudaStreamSynchronize(x.c->stream));
	for (int j = 0; j < x.k; j++) out[j] = std::sqrt(h[j]);
	return BSG_OK;
}

} // namespace

namespace {
__global__ void k_add(long long n, const double *a, const double *b, double *out) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		out[i] = a[i] + b[i];
}
} // namespace

extern "C" int bsg_block_lanczos_dev(bsg_ctx *c, const bsg_mat *mc, const bsg_fct *fc, int ittype, int nrhs,
                                     const double *d_B, double *d_X, bsg_param *p, double *res) {
	if (!c || !mc || !fc || !d_B || !d_X || !p || nrhs < 1)
		return bsg_set_error(BSG_ERR_ARG, "bsg_block_lanczos_dev: bad argument");
	if (ittype < 2 || ittype > 4)
		return bsg_set_error(BSG_ERR_ARG, "bsg_block_lanczos_dev: ittype must be 2 (central), 3 (right) or 4 (left)");
	if (nrhs > BL_MAXRHS) return bsg_set_error(BSG_ERR_UNSUPPORTED, "bsg_block_lanczos_dev: more than 16 right-hand sides");
	bsg_mat *m = const_cast<bsg_mat *>(mc); // transposed copies are cached on the objects
	bsg_fct *f = const_cast<bsg_fct *>(fc);
	if (m->bs != 1 || f->d_bia)
		return bsg_set_error(BSG_ERR_UNSUPPORTED, "bsg_block_lanczos_dev: point matrices and point factors only");
	const int n = m->n, k = nrhs;
	const long long nk = (long long)n * k;
	cudaStream_t s = c->stream;
	Buf bR, bU, bV, bW, bY, bQ, bT, bS, b1, b2, bw, bsm, bh;
	for (Buf *b : {&bR, &bU, &bV, &bW, &bY, &bQ, &bT, &bS, &b1, &b2, &bw, &bsm, &bh}) b->s = s;
	for (Buf *b : {&bR, &bU, &bV, &bW, &bY, &bQ, &bT, &bS})
		if (cudaMallocAsync(&b->p, sizeof(double) * (nk ? nk : 1), s) != cudaSuccess)
			return bsg_set_error(BSG_ERR_NOMEM, "block Lanczos vectors");
	for (Buf *b : {&b1, &b2, &bw})
		if (cudaMallocAsync(&b->p, sizeof(double) * (n ? n : 1), s) != cudaSuccess)
			return bsg_set_error(BSG_ERR_NOMEM, "block Lanczos vectors");
	BSG_CUDA(cudaMallocAsync(&bsm.p, sizeof(double) * BL_MAXRHS * BL_MAXRHS, s));
	BSG_CUDA(cudaMallocAsync(&bh.p, sizeof(double) * (2 * BL_MAXRHS + 1), s));
	BSG_CUDA(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), s));
	Ctx x{c, m, f, p, n, k, ittype, b1.p, b2.p, bw.p, bsm.p, bh.p};
	cudaEventRecord(c->ev0, s);
	auto mt_cols = [&](const double *in, double *out) {
		return columns(x, in, out, [&](const double *a, double *b) { return apply_mt(x, a, b); });
	};
	// residual block of X0 + P Y (Y == nullptr: of X0) into bR, the point in bQ
	auto residual = [&](const double *Y, std::vector<double> &rn, std::vector<double> *mtn) {
		int r2 = BSG_OK;
		const double *X = d_X;
		if (Y) {
			r2 = columns(x, Y, bQ.p, [&](const double *a, double *b) { return apply_back(x, a, b); });
			if (r2) return r2;
			BSG_COUNT(1);
			k_add<<<ew_grid(nk), 256, 0, s>>>(nk, d_X, bQ.p, bQ.p);
			X = bQ.p;
		}
		r2 = bsg_spmm_launch(m, k, X, bR.p, n, s);
		if (!r2) r2 = bsg_residual_launch(c, (int)nk, d_B, bR.p);
		if (!r2) r2 = col_norms(x, bR.p, rn);
		if (!r2 && mtn) {
			r2 = mt_cols(bR.p, bS.p);
			if (!r2) r2 = col_norms(x, bS.p, *mtn);
		}
		return r2;
	};
	std::vector<double> r0n, mt0n, rn, mtn;
	int rc = residual(nullptr, r0n, ittype == 3 ? &mt0n : nullptr);
	// the start block: central L^{-1} r0, right r0, left U^{-1} L^{-1} r0
	if (!rc) {
		if (ittype == 2) {
			rc = columns(x, bR.p, bU.p, [&](const double *a, double *b) { return lsolve(x, a, b); });
		} else if (ittype == 3) {
			if (cudaMemcpyAsync(bU.p, bR.p, sizeof(double) * nk, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
				rc = bsg_set_error(BSG_ERR_CUDA, "block Lanczos copy");
		} else {
			rc = columns(x, bR.p, bU.p, [&](const double *a, double *b) {
				int r2 = lsolve(x, a, x.t2);
				return r2 ? r2 : usolve(x, x.t2, b);
			});
		}
	}
	if (rc) return rc;
	Mat beta, alpha, R, rhobar, phibar, Q, rho;
	if ((rc = block_qr(x, bU.p, beta))) return rc;
	if ((rc = mt_cols(bU.p, bV.p))) return rc;
	if ((rc = block_qr(x, bV.p, R))) return rc;
	alpha = transpose(k, R);
	BSG_CUDA(cudaMemcpyAsync(bW.p, bV.p, sizeof(double) * nk, cudaMemcpyDeviceToDevice, s));
	BSG_CUDA(cudaMemsetAsync(bY.p, 0, sizeof(double) * nk, s));
	phibar = beta;
	rhobar = alpha;
	const int ichk = p->ichk > 0 ? p->ichk : 1;
	auto done = [&]() {
		for (int j = 0; j < k; j++) {
			const bool ok = rn[j] < p->eps * r0n[j] || (ittype == 3 && mtn[j] < p->eps * mt0n[j]) || r0n[j] == 0.0;
			if (!ok) return false;
		}
		return true;
	};
	int it;
	bool converged = false;
	for (it = 1; it <= p->niter; it++) {
		// U' beta = M V - U alpha
		if ((rc = columns(x, bV.p, bQ.p, [&](const double *a, double *b) { return apply_m(x, a, b); }))) break;
		if ((rc = blk_update(x, bU.p, alpha, -1.0, 1.0, bQ.p, bQ.p))) break;
		if ((rc = block_qr(x, bQ.p, beta))) break;
		std::swap(bU.p, bQ.p);
		// V' R = M^T U' - V beta^T, alpha = R^T
		if ((rc = mt_cols(bU.p, bT.p))) break;
		if ((rc = blk_update(x, bV.p, transpose(k, beta), -1.0, 1.0, bT.p, bT.p))) break;
		if ((rc = block_qr(x, bT.p, R))) break;
		const Mat alpha_new = transpose(k, R);
		// block Givens: Q^T [rhobar; beta] = [rho; 0]
		Mat G((size_t)2 * k * k);
		for (int i = 0; i < k; i++)
			for (int j = 0; j < k; j++) {
				G[(size_t)i * k + j] = rhobar[(size_t)i * k + j];
				G[(size_t)(k + i) * k + j] = beta[(size_t)i * k + j];
			}
		house_qr(2 * k, k, G, Q, rho);
		// [theta; rhobar'] = Q^T [0; alpha'],  [phi; phibar'] = Q^T [phibar; 0]
		Mat theta((size_t)k * k), phi((size_t)k * k), rb((size_t)k * k), pb((size_t)k * k);
		for (int i = 0; i < 2 * k; i++)
			for (int j = 0; j < k; j++) {
				double t = 0.0, f2 = 0.0;
				for (int q = 0; q < k; q++) {
					t += Q[(size_t)(k + q) * 2 * k + i] * alpha_new[(size_t)q * k + j];
					f2 += Q[(size_t)q * 2 * k + i] * phibar[(size_t)q * k + j];
				}
				if (i < k) {
					theta[(size_t)i * k + j] = t;
					phi[(size_t)i * k + j] = f2;
				} else {
					rb[(size_t)(i - k) * k + j] = t;
					pb[(size_t)(i - k) * k + j] = f2;
				}
			}
		alpha = alpha_new;
		rhobar = rb;
		phibar = pb;
		// Y += W rho^{-1} phi;  W = V' - W rho^{-1} theta;  V = V'
		const Mat c1 = upper_solve(k, rho, phi), c2 = upper_solve(k, rho, theta);
		if ((rc = blk_update(x, bW.p, c1, 1.0, 1.0, bY.p, bY.p))) break;
		if ((rc = blk_update(x, bW.p, c2, -1.0, 1.0, bT.p, bQ.p))) break;
		std::swap(bV.p, bT.p);
		std::swap(bW.p, bQ.p);
		if ((rc = bsg_check_devstat(c))) break;
		// the reference's test every ichk steps: the true residual of x
		if (it % ichk == 0) {
			if ((rc = residual(bY.p, rn, ittype == 3 ? &mtn : nullptr))) break;
			if (done()) {
				converged = true;
				break;
			}
		}
	}
	if (rc) return rc;
	cudaEventRecord(c->ev1, s);
	// x = X0 + P Y
	if ((rc = residual(bY.p, rn, nullptr))) return rc;
	BSG_CUDA(cudaMemcpyAsync(d_X, bQ.p, sizeof(double) * nk, cudaMemcpyDeviceToDevice, s));
	if (!converged) converged = done();
	std::vector<double> bn;
	if ((rc = col_norms(x, d_B, bn))) return rc;
	double worst = 0.0;
	for (int j = 0; j < k; j++) {
		const double r = bn[j] > 0.0 ? rn[j] / bn[j] : rn[j];
		if (res) res[j] = r;
		worst = r > worst ? r : worst;
	}
	float ms = 0;
	cudaEventElapsedTime(&ms, c->ev0, c->ev1);
	p->timeitr = ms * 1e-3;
	p->nitperf = it > p->niter ? p->niter : it;
	p->resfin = worst;
	if ((rc = bsg_check_devstat(c))) return rc;
	if (!converged) return bsg_set_error(BSG_ERR_NOCONV, "iteration limit reached");
	return BSG_OK;
}
