// Krylov loops of the solver path on the device: PCG (CSVector::Cg,
// Bslib/cg.cpp:31-350) and right-preconditioned GMRES(m) / FGMRES(m) (the
// restarted FP64 counterpart of CSVector::BlockGMRES, Bslib/gmres.cpp:337).
//
// Vectors and inner products are FP64; the preconditioner may apply FP32
// factor values (the product is still formed in FP64), so the FP64 outer
// loop acts as iterative refinement around the FP32 factor.  Scalars live in
// device memory and are consumed by the next kernel, so a PCG iteration has
// exactly one host synchronisation (the convergence test the reference makes
// every iteration).  GMRES orthogonalises with classical Gram-Schmidt run
// twice (one multi-dot and one update per pass instead of j+1 dependent dots),
// then applies the Givens recurrence of Bslib/gmres.cpp:30-101 on the host.
#include "bsg_internal.cuh"
#include <vector>
#include <cmath>
#include <chrono>

int bsg_spmm_launch(const bsg_mat *m, int nrhs, const double *X, double *Y, long long ld, cudaStream_t s);
int bsg_dots_launch(bsg_ctx *c, int q, int n, const double *x0, const double *y0, const double *x1,
                    const double *y1, const double *x2, const double *y2, double *d_out);
int bsg_mdot_launch(bsg_ctx *c, int n, const double *V, long long ld, int k, const double *w, double *d_out);
int bsg_gemv_sub_launch(bsg_ctx *c, int n, const double *V, long long ld, int k, const double *h, double *w);
int bsg_gemv_add_launch(bsg_ctx *c, int n, const double *V, long long ld, int k, const double *y, double *x);
int bsg_scale_by_launch(bsg_ctx *c, int n, const double *x, double *y, const double *num, const double *den,
                        int sqrt_den);
int bsg_residual_launch(bsg_ctx *c, int n, const double *b, double *r);
int bsg_maxabs_launch(bsg_ctx *c, int n, const double *x, double *d_out);
int bsg_fill_launch(cudaStream_t s, long long n, double *x, double v);
int bsg_unet_apply(void *net, bsg_ctx *c, const double *r, double *z, double *work);
extern "C" int bsg_unet_set_matrix(bsg_unet *u, const bsg_mat *m);

// device scalar slots used by PCG
enum { S_ENRSQ = 0, S_GAMMA = 1, S_GAMOLD = 2, S_PAP = 3, S_BREAK = 4, S_ERR = 5, S_TMP = 8 };

namespace {

__global__ void k_pcg_p(int n, const double *z, double *p, const double *d_s, int first) {
	const double beta = first ? 0.0 : d_s[S_GAMMA] / d_s[S_GAMOLD];
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = p[i] * beta + z[i];
}

__global__ void k_pcg_xr(int n, const double *p, const double *q, double *r, double *x, double *d_s) {
	const double alpha = d_s[S_GAMMA] / d_s[S_PAP];
	if (alpha < 0.0) { // not positive definite: keep x, r (Bslib/cg.cpp:266-278)
		if (blockIdx.x == 0 && threadIdx.x == 0) d_s[S_BREAK] = 1.0;
		return;
	}
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		r[i] = fma(-alpha, q[i], r[i]);
		x[i] = fma(alpha, p[i], x[i]);
	}
}

__global__ void k_copy_scalar(double *d_s, int dst, int src) { d_s[dst] = d_s[src]; }

inline int ew_grid(long long n) {
	long long b = (n + 255) / 256;
	long long cap = (long long)BSG_SMS * 8;
	return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

double now_s() {
	using namespace std::chrono;
	return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Buf {
	double *p = nullptr;
	cudaStream_t s = nullptr;
	~Buf() { if (p) cudaFreeAsync(p, s); }
};

} // namespace

int bsg_precond_apply(bsg_ctx *c, const bsg_fct *f, const bsg_param *p, const double *r, double *z, double *tmp,
                      double *work) {
	int mode = p->trisolve;
	int rc = bsg_trisolve_launch(c, f, 1, mode, p->nsweeps, r, tmp, work);
	if (rc) return rc;
	return bsg_trisolve_launch(c, f, 0, mode, p->nsweeps, tmp, z, work);
}

// bsg_precond_apply for nr vectors at stride n (tmp, work: n nr doubles)
int bsg_precond_apply_multi(bsg_ctx *c, const bsg_fct *f, const bsg_param *p, int nr, const double *r, double *z,
                            double *tmp, double *work) {
	int rc = bsg_trisolve_multi(c, f, 1, p->trisolve, p->nsweeps, nr, r, tmp, work);
	if (rc) return rc;
	return bsg_trisolve_multi(c, f, 0, p->trisolve, p->nsweeps, nr, tmp, z, work);
}

int bsg_check_devstat(bsg_ctx *c);

// FP64 true residual ||b - A x|| / ||b|| (one host sync).
int bsg_true_residual(bsg_ctx *c, const bsg_mat *m, const double *b, const double *x, double *r, double *out) {
	const int N = m->n * m->bs;
	int rc = bsg_spmm_launch(m, 1, x, r, N, c->stream);
	if (rc) return rc;
	rc = bsg_residual_launch(c, N, b, r);
	if (rc) return rc;
	rc = bsg_dots_launch(c, 2, N, r, r, b, b, nullptr, nullptr, c->d_scalars + S_TMP);
	if (rc) return rc;
	BSG_CUDA(cudaMemcpyAsync(c->h_pinned, c->d_scalars + S_TMP, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
	BSG_CUDA(cudaStreamSynchronize(c->stream));
	double rr = c->h_pinned[0], bb = c->h_pinned[1];
	*out = bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
	return BSG_OK;
}

extern "C" int bsg_pcg_dev(bsg_ctx *c, const bsg_mat *m, const bsg_fct *f, const double *d_b, double *d_x,
                           bsg_param *p) {
	if (!c || !m || !f || !d_b || !d_x || !p) return bsg_set_error(BSG_ERR_ARG, "bsg_pcg_dev: null argument");
	if (p->ittype < 0 || p->ittype > 2) return bsg_set_error(BSG_ERR_UNSUPPORTED, "PCG: ittype must be 0, 1 or 2");
	const int N = m->n * m->bs;
	cudaStream_t s = c->stream;
	Buf r, q, z, pp, t, w;
	r.s = q.s = z.s = pp.s = t.s = w.s = s;
	BSG_CUDA(cudaMallocAsync(&r.p, sizeof(double) * N, s));
	BSG_CUDA(cudaMallocAsync(&q.p, sizeof(double) * N, s));
	BSG_CUDA(cudaMallocAsync(&z.p, sizeof(double) * N, s));
	BSG_CUDA(cudaMallocAsync(&pp.p, sizeof(double) * N, s));
	BSG_CUDA(cudaMallocAsync(&t.p, sizeof(double) * N, s));
	BSG_CUDA(cudaMallocAsync(&w.p, sizeof(double) * N, s));
	BSG_CUDA(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), s));
	BSG_CUDA(cudaMemsetAsync(c->d_scalars, 0, 16 * sizeof(double), s));
	BSG_CUDA(cudaMemsetAsync(pp.p, 0, sizeof(double) * N, s));
	double t0 = now_s();
	cudaEventRecord(c->ev0, s);
	// r = b - A x
	int rc = bsg_spmm_launch(m, 1, d_x, r.p, N, s);
	if (!rc) rc = bsg_residual_launch(c, N, d_b, r.p);
	if (rc) return rc;
	double enrsq0 = 0.0, enrsq = 0.0, errmin = 0.0;
	const bool maxnorm = p->ittype == 2;
	int k, nit = 0, status = BSG_OK, replacements = 0;
	const int g = ew_grid(N);
	for (k = 1; k < p->niter; k++) {
		rc = bsg_precond_apply(c, f, p, r.p, z.p, t.p, w.p);
		if (rc) return rc;
		rc = bsg_dots_launch(c, 2, N, r.p, r.p, r.p, z.p, nullptr, nullptr, c->d_scalars + S_ENRSQ);
		// ittype 2: weighted max-norm of the recursive residual, unit weights
		// (Bslib/cg.cpp:195-198, the weights of AbstractSymmSolver are 1)
		if (!rc && maxnorm) rc = bsg_maxabs_launch(c, N, r.p, c->d_scalars + S_ERR);
		if (rc) return rc;
		BSG_CUDA(cudaMemcpyAsync(c->h_pinned, c->d_scalars, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
		BSG_CUDA(cudaStreamSynchronize(s));
		rc = bsg_check_devstat(c);
		if (rc) return rc;
		enrsq = c->h_pinned[S_ENRSQ];
		if (k == 1) enrsq0 = enrsq;
		errmin = c->h_pinned[S_ERR];
		nit = k;
		if (c->h_pinned[S_BREAK] != 0.0) { status = BSG_ERR_BREAKDOWN; break; }
		// stop rules of Bslib/cg.cpp:239-241: 0 relative and 1 absolute on
		// ||r||^2, 2 on max |r_i| <= |eps|
		const double goal = maxnorm ? std::fabs(p->eps) : (p->ittype == 0 ? p->eps * p->eps * enrsq0 : p->eps * p->eps);
		if ((maxnorm ? errmin : enrsq) <= goal) {
			if (!p->true_residual || replacements >= 5) break;
			// the recursive residual says converged: confirm with the FP64
			// true residual in the same norm; if it drifted (FP32
			// preconditioner), continue from the true residual
			rc = bsg_spmm_launch(m, 1, d_x, t.p, N, s);
			if (!rc) rc = bsg_residual_launch(c, N, d_b, t.p);
			if (!rc) rc = maxnorm ? bsg_maxabs_launch(c, N, t.p, c->d_scalars + S_TMP)
			                      : bsg_dots_launch(c, 1, N, t.p, t.p, nullptr, nullptr, nullptr, nullptr, c->d_scalars + S_TMP);
			if (rc) return rc;
			BSG_CUDA(cudaMemcpyAsync(c->h_pinned + 8, c->d_scalars + S_TMP, sizeof(double), cudaMemcpyDeviceToHost, s));
			BSG_CUDA(cudaStreamSynchronize(s));
			if (c->h_pinned[8] <= goal) break;
			replacements++;
			BSG_CUDA(cudaMemcpyAsync(r.p, t.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
			rc = bsg_precond_apply(c, f, p, r.p, z.p, t.p, w.p);
			if (!rc) rc = bsg_dots_launch(c, 2, N, r.p, r.p, r.p, z.p, nullptr, nullptr, c->d_scalars + S_ENRSQ);
			if (rc) return rc;
		}
		BSG_COUNT(3); // k_pcg_p, k_pcg_xr, k_copy_scalar
		k_pcg_p<<<g, 256, 0, s>>>(N, z.p, pp.p, c->d_scalars, k == 1);
		rc = bsg_spmm_launch(m, 1, pp.p, q.p, N, s);
		if (rc) return rc;
		rc = bsg_dots_launch(c, 1, N, pp.p, q.p, nullptr, nullptr, nullptr, nullptr, c->d_scalars + S_PAP);
		if (rc) return rc;
		k_pcg_xr<<<g, 256, 0, s>>>(N, pp.p, q.p, r.p, d_x, c->d_scalars);
		k_copy_scalar<<<1, 1, 0, s>>>(c->d_scalars, S_GAMOLD, S_GAMMA);
		BSG_CUDA(cudaGetLastError());
	}
	if (k >= p->niter) status = BSG_ERR_NOCONV;
	cudaEventRecord(c->ev1, s);
	double res = 0;
	rc = bsg_true_residual(c, m, d_b, d_x, r.p, &res);
	if (rc) return rc;
	float ms = 0;
	cudaEventElapsedTime(&ms, c->ev0, c->ev1);
	p->timeitr = ms * 1e-3;
	p->nitperf = nit;
	p->resfin = res;
	p->resrec = maxnorm ? errmin : (enrsq0 > 0 ? std::sqrt(enrsq / enrsq0) : 0.0);
	(void)t0;
	if (status == BSG_ERR_BREAKDOWN) return bsg_set_error(status, " Matrix is not positive definite");
	if (status == BSG_ERR_NOCONV) return bsg_set_error(status, "iteration limit reached");
	return BSG_OK;
}

// GMRES(m) / FGMRES(m), right preconditioned: A M^{-1} u = b, x = M^{-1} u.
// With a fixed preconditioner the two coincide; FGMRES stores the
// preconditioned directions Z so the preconditioner may change per step
// (the learned stage).
extern "C" int bsg_gmres_dev(bsg_ctx *c, const bsg_mat *m, const bsg_fct *f, const double *d_b, double *d_x,
                             bsg_param *p) {
	if (!c || !m || !f || !d_b || !d_x || !p) return bsg_set_error(BSG_ERR_ARG, "bsg_gmres_dev: null argument");
	const int N = m->n * m->bs;
	const int M = p->restart > 0 ? p->restart : 50;
	cudaStream_t s = c->stream;
	Buf V, Z, w, t, wk, hbuf;
	V.s = Z.s = w.s = t.s = wk.s = hbuf.s = s;
	const long long ld = N;
	if (cudaMallocAsync(&V.p, sizeof(double) * ld * (M + 1), s) != cudaSuccess ||
	    cudaMallocAsync(&Z.p, sizeof(double) * ld * M, s) != cudaSuccess)
		return bsg_set_error(BSG_ERR_NOMEM, "GMRES basis");
	BSG_CUDA(cudaMallocAsync(&w.p, sizeof(double) * N, s));
	BSG_CUDA(cudaMallocAsync(&t.p, sizeof(double) * N, s));
	BSG_CUDA(cudaMallocAsync(&wk.p, sizeof(double) * N, s));
	BSG_CUDA(cudaMallocAsync(&hbuf.p, sizeof(double) * 2 * (M + 2), s));
	BSG_CUDA(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), s));
	cudaEventRecord(c->ev0, s);
	std::vector<double> H((size_t)(M + 1) * M, 0.0), cs(M), sn(M), g(M + 1), y(M), h(M + 2), h2(M + 2);
	double bnorm = 0, beta = 0;
	{
		int rc = bsg_dots_launch(c, 1, N, d_b, d_b, nullptr, nullptr, nullptr, nullptr, c->d_scalars + S_TMP);
		if (rc) return rc;
		BSG_CUDA(cudaMemcpyAsync(c->h_pinned, c->d_scalars + S_TMP, sizeof(double), cudaMemcpyDeviceToHost, s));
		BSG_CUDA(cudaStreamSynchronize(s));
		bnorm = std::sqrt(c->h_pinned[0]);
	}
	const double target = (p->sttype == 0) ? p->eps : p->eps * bnorm;
	const bool flexible = p->krylov == 2;
	if (flexible && p->learned) {
		// the learned stage works on this operator (its diagonal is an input)
		int rc = bsg_unet_set_matrix(static_cast<bsg_unet *>(p->learned), m);
		if (rc) return rc;
	}
	int it = 0, status = BSG_OK;
	double est = 0;
	bool converged = false;
	while (it < p->niter) {
		// r = b - A x into V0
		int rc = bsg_spmm_launch(m, 1, d_x, V.p, ld, s);
		if (!rc) rc = bsg_residual_launch(c, N, d_b, V.p);
		if (!rc) rc = bsg_dots_launch(c, 1, N, V.p, V.p, nullptr, nullptr, nullptr, nullptr, c->d_scalars + S_TMP);
		if (rc) return rc;
		BSG_CUDA(cudaMemcpyAsync(c->h_pinned, c->d_scalars + S_TMP, sizeof(double), cudaMemcpyDeviceToHost, s));
		BSG_CUDA(cudaStreamSynchronize(s));
		beta = std::sqrt(c->h_pinned[0]);
		est = beta;
		if (beta <= target) { converged = true; break; }
		rc = bsg_scale_by_launch(c, N, V.p, V.p, nullptr, c->d_scalars + S_TMP, 1);
		if (rc) return rc;
		std::fill(g.begin(), g.end(), 0.0);
		g[0] = beta;
		int j;
		for (j = 0; j < M && it < p->niter; j++) {
			double *vj = V.p + (size_t)j * ld, *zj = Z.p + (size_t)(flexible ? j : j) * ld, *vn = V.p + (size_t)(j + 1) * ld;
			rc = bsg_precond_apply(c, f, p, vj, zj, t.p, wk.p);
			if (!rc && flexible && p->learned) rc = bsg_unet_apply(p->learned, c, vj, zj, t.p);
			if (!rc) rc = bsg_spmm_launch(m, 1, zj, vn, ld, s);
			if (rc) return rc;
			// CGS2: two passes of h = V^T w, w -= V h
			double *dh = hbuf.p, *dh2 = hbuf.p + (M + 2);
			rc = bsg_mdot_launch(c, N, V.p, ld, j + 1, vn, dh);
			if (!rc) rc = bsg_gemv_sub_launch(c, N, V.p, ld, j + 1, dh, vn);
			if (!rc) rc = bsg_mdot_launch(c, N, V.p, ld, j + 1, vn, dh2);
			if (!rc) rc = bsg_gemv_sub_launch(c, N, V.p, ld, j + 1, dh2, vn);
			if (!rc) rc = bsg_dots_launch(c, 1, N, vn, vn, nullptr, nullptr, nullptr, nullptr, c->d_scalars + S_TMP);
			if (rc) return rc;
			BSG_CUDA(cudaMemcpyAsync(h.data(), dh, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s));
			BSG_CUDA(cudaMemcpyAsync(h2.data(), dh2, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s));
			BSG_CUDA(cudaMemcpyAsync(c->h_pinned, c->d_scalars + S_TMP, sizeof(double), cudaMemcpyDeviceToHost, s));
			rc = bsg_scale_by_launch(c, N, vn, vn, nullptr, c->d_scalars + S_TMP, 1);
			if (rc) return rc;
			BSG_CUDA(cudaStreamSynchronize(s));
			rc = bsg_check_devstat(c);
			if (rc) return rc;
			double hn = std::sqrt(c->h_pinned[0]);
			for (int k = 0; k <= j; k++) H[(size_t)k * M + j] = h[k] + h2[k];
			H[(size_t)(j + 1) * M + j] = hn;
			for (int k = 0; k < j; k++) {
				double a0 = H[(size_t)k * M + j], a1 = H[(size_t)(k + 1) * M + j];
				H[(size_t)k * M + j] = cs[k] * a0 + sn[k] * a1;
				H[(size_t)(k + 1) * M + j] = -sn[k] * a0 + cs[k] * a1;
			}
			double a0 = H[(size_t)j * M + j], a1 = hn;
			double rr = std::hypot(a0, a1);
			cs[j] = rr > 0 ? a0 / rr : 1.0;
			sn[j] = rr > 0 ? a1 / rr : 0.0;
			H[(size_t)j * M + j] = rr;
			H[(size_t)(j + 1) * M + j] = 0.0;
			g[j + 1] = -sn[j] * g[j];
			g[j] = cs[j] * g[j];
			it++;
			est = std::fabs(g[j + 1]);
			if (est <= target || hn == 0.0) { j++; break; }
		}
		// y = R^{-1} g, x += Z y
		for (int k = j - 1; k >= 0; k--) {
			double sum = g[k];
			for (int q = k + 1; q < j; q++) sum -= H[(size_t)k * M + q] * y[q];
			y[k] = sum / H[(size_t)k * M + k];
		}
		BSG_CUDA(cudaMemcpyAsync(hbuf.p, y.data(), sizeof(double) * j, cudaMemcpyHostToDevice, s));
		rc = bsg_gemv_add_launch(c, N, Z.p, ld, j, hbuf.p, d_x);
		if (rc) return rc;
		BSG_CUDA(cudaStreamSynchronize(s));
	}
	if (!converged) {
		// the final restart's check may have left the loop on the iteration limit
		double res = 0;
		int rc = bsg_true_residual(c, m, d_b, d_x, w.p, &res);
		if (rc) return rc;
		if (res * (p->sttype == 0 ? 1.0 : bnorm) <= target) converged = true;
	}
	cudaEventRecord(c->ev1, s);
	double res = 0;
	int rc = bsg_true_residual(c, m, d_b, d_x, w.p, &res);
	if (rc) return rc;
	float ms = 0;
	cudaEventElapsedTime(&ms, c->ev0, c->ev1);
	p->timeitr = ms * 1e-3;
	p->nitperf = it;
	p->resfin = res;
	p->resrec = bnorm > 0 ? est / bnorm : est;
	if (!converged) status = BSG_ERR_NOCONV;
	if (status) return bsg_set_error(status, "iteration limit reached");
	return BSG_OK;
}
