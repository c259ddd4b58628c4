// Preconditioned two-sided Lanczos on the device: CSVector::Lanczos
// (Bslib/lanczos.cpp:34-370), the reference's solver for nonsymmetric
// systems (CSVector::Solver, Bslib/solvers.cpp:1339-1500).
//
// The recurrence is the reference's: per iteration a product with A and the
// preconditioner M^{-1} = U^{-1} L^{-1}, the scalars gamma / ro, three-term
// updates of the solution and of the direction delta, the true residual
// b - A x with its 2-norm and max-norm, then the transposed products
// M^{-T} = L^{-T} U^{-T} and A^T that update the shadow direction Delta.
// The returned solution is the iterate of least max-norm residual.  All
// vectors and scalars are FP64; the scalars live on the device (no host round
// trip between kernels); the host reads the norms once per iteration, where
// the reference tests for convergence.  A^T is a sliced copy of the device
// transpose (built on first use; A itself for symmetric input); the
// transposed solves use the factor's transposed forms (k_trsv.cu).
#include "bsg_internal.cuh"
#include <cmath>

int bsg_spmm_launch(const bsg_mat *m, int nrhs, const double *X, double *Y, long long ld, cudaStream_t s);
int bsg_dots_launch(bsg_ctx *c, int q, int n, const double *x0, const double *y0, const double *x1,
                    const double *y1, const double *x2, const double *y2, double *d_out);
int bsg_residual_launch(bsg_ctx *c, int n, const double *b, double *r);
int bsg_precond_apply(bsg_ctx *c, const bsg_fct *f, const bsg_param *p, const double *r, double *z, double *tmp,
                      double *work);
int bsg_transpose_full(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, int nnz, int **ta_o,
                       int **tja_o, double **tv_o);
int bsg_true_residual(bsg_ctx *c, const bsg_mat *m, const double *b, const double *x, double *r, double *out);

namespace {

// device scalar slots (after the ones PCG / GMRES use)
enum { L_DD = 16, L_DT, L_G, L_DDPREV, L_RO, L_ROG, L_UNRO, L_DD1, L_RR, L_EMAX };

// gamma = (delta . Delta) / (M^{-1} A delta . Delta); ro (Bslib/lanczos.cpp:148-159)
__global__ void k_lz_scal(double *s, int k) {
	const double g1 = s[L_G], dd1 = s[L_DDPREV], dd = s[L_DD];
	const double g = dd / s[L_DT];
	double ro = s[L_RO];
	if (k > 1) ro = 1.0 / (1.0 - (g / g1) * (dd / dd1) / ro);
	s[L_G] = g;
	s[L_RO] = ro;
	s[L_ROG] = ro * g;
	s[L_UNRO] = 1.0 - ro;
	s[L_DD1] = dd1;
	s[L_DDPREV] = dd;
}

// v <- (v ro + v1 (1 - ro)) + sgn w ro gamma, v1 <- old v
template <int SGN>
__global__ void k_lz_three(int n, const double *s, double *v, double *v1, const double *w) {
	const double ro = s[L_RO], un = s[L_UNRO], rog = s[L_ROG];
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const double t = v[i];
		const double p = t * ro + v1[i] * un;
		v[i] = SGN > 0 ? p + w[i] * rog : p - w[i] * rog;
		v1[i] = t;
	}
}

// r . r and max |r_i| (block partials, then one ordered final pass)
#define LZ_BLOCKS 256
__global__ void k_lz_norm_part(int n, const double *r, double *part) {
	__shared__ double sa[8], sm[8];
	double a = 0.0, mx = 0.0;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		a = fma(r[i], r[i], a);
		const double v = fabs(r[i]);
		mx = (v > mx || v != v) ? v : mx; // a NaN entry makes the max NaN (never "better")
	}
	a = warp_sum(a);
	for (int o = 16; o > 0; o >>= 1) {
		const double v = __shfl_xor_sync(0xffffffffu, mx, o);
		mx = (v > mx || v != v) ? v : mx;
	}
	if ((threadIdx.x & 31) == 0) { sa[threadIdx.x >> 5] = a; sm[threadIdx.x >> 5] = mx; }
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0, m = 0.0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) { t += sa[w]; m = (sm[w] > m || sm[w] != sm[w]) ? sm[w] : m; }
		part[blockIdx.x] = t;
		part[LZ_BLOCKS + blockIdx.x] = m;
	}
}
__global__ void k_lz_norm_final(const double *part, double *s) {
	if (threadIdx.x == 0) {
		double t = 0.0, m = 0.0;
		for (int b = 0; b < LZ_BLOCKS; b++) {
			const double v = part[LZ_BLOCKS + b];
			t += part[b];
			m = (v > m || v != v) ? v : m;
		}
		s[L_RR] = t;
		s[L_EMAX] = m;
	}
}

struct Buf {
	double *p = nullptr;
	cudaStream_t s = nullptr;
	~Buf() { if (p) cudaFreeAsync(p, s); }
};

inline int ew(long long n) {
	long long b = (n + 255) / 256;
	return (int)(b < BSG_SMS * 8 ? (b > 0 ? b : 1) : BSG_SMS * 8);
}

// y = A^T x
int mvm_t(bsg_ctx *c, bsg_mat *m, const double *x, double *y) {
	if (m->symm) return bsg_spmm_launch(m, 1, x, y, m->n, c->stream);
	if (!m->sellT.off) {
		int *ta, *tj;
		double *tv;
		int rc = bsg_transpose_full(c, m->n, m->d_ia, m->d_ja, m->d_a, m->nnz, &ta, &tj, &tv);
		if (!rc) rc = bsg_sell_build(c, m->n, ta, tj, tv, 0, 0, &m->sellT, 0);
		cudaFreeAsync(ta, c->stream);
		cudaFreeAsync(tj, c->stream);
		cudaFreeAsync(tv, c->stream);
		if (rc) return rc;
	}
	return bsg_sell_spmv(c->stream, &m->sellT, x, y);
}

} // namespace

// y = A^T x for a point matrix (the SELL copy of A^T is built on first use).
int bsg_mvm_t_launch(bsg_ctx *c, bsg_mat *m, const double *x, double *y) { return mvm_t(c, m, x, y); }

extern "C" int bsg_lanczos_dev(bsg_ctx *c, const bsg_mat *mc, const bsg_fct *fc, const double *d_b, double *d_x,
                               bsg_param *p) {
	if (!c || !mc || !fc || !d_b || !d_x || !p) return bsg_set_error(BSG_ERR_ARG, "bsg_lanczos_dev: null argument");
	bsg_mat *m = const_cast<bsg_mat *>(mc); // the transposed copies are cached on the objects
	bsg_fct *f = const_cast<bsg_fct *>(fc);
	if (m->bs != 1) return bsg_set_error(BSG_ERR_UNSUPPORTED, "bsg_lanczos_dev: point matrices only");
	const int n = m->n;
	cudaStream_t s = c->stream;
	Buf r, good, sol1, D, D1, d, d1, img, pv, t, w, part;
	Buf *all[] = {&r, &good, &sol1, &D, &D1, &d, &d1, &img, &pv, &t, &w};
	for (Buf *b : all) {
		b->s = s;
		if (cudaMallocAsync(&b->p, sizeof(double) * n, s) != cudaSuccess) return bsg_set_error(BSG_ERR_NOMEM, "Lanczos vectors");
	}
	part.s = s;
	BSG_CUDA(cudaMallocAsync(&part.p, sizeof(double) * 2 * LZ_BLOCKS, s));
	BSG_CUDA(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), s));
	BSG_CUDA(cudaMemsetAsync(c->d_scalars + L_DD, 0, 10 * sizeof(double), s));
	{
		const double one = 1.0;
		BSG_CUDA(cudaMemcpyAsync(c->d_scalars + L_RO, &one, sizeof(double), cudaMemcpyHostToDevice, s));
	}
	BSG_CUDA(cudaMemsetAsync(sol1.p, 0, sizeof(double) * n, s));
	BSG_CUDA(cudaMemsetAsync(d1.p, 0, sizeof(double) * n, s));
	BSG_CUDA(cudaMemsetAsync(D1.p, 0, sizeof(double) * n, s));
	cudaEventRecord(c->ev0, s);
	double *sc = c->d_scalars;
	const int g = ew(n);
	auto norms = [&](const double *v) {
		BSG_COUNT(2);
		k_lz_norm_part<<<LZ_BLOCKS, 256, 0, s>>>(n, v, part.p);
		k_lz_norm_final<<<1, 32, 0, s>>>(part.p, sc);
	};
	// r = b - A x, its norms; good = x; Delta = r; delta = M^{-1} r
	int rc = bsg_spmm_launch(m, 1, d_x, r.p, n, s);
	if (!rc) rc = bsg_residual_launch(c, n, d_b, r.p);
	if (rc) return bsg_set_error(rc, "Lanczos start");
	norms(r.p);
	BSG_CUDA(cudaMemcpyAsync(good.p, d_x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
	BSG_CUDA(cudaMemcpyAsync(D.p, r.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
	if ((rc = bsg_precond_apply(c, f, p, r.p, d.p, t.p, w.p))) return bsg_set_error(rc, "Lanczos preconditioner");
	BSG_CUDA(cudaMemcpyAsync(c->h_pinned, sc + L_RR, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	const double resini = std::sqrt(c->h_pinned[0]);
	double errmin = c->h_pinned[1], resi = resini;
	int k;
	int status = BSG_OK;
	for (k = 1; k < p->niter; k++) {
		// img = M^{-1} A delta; (delta . Delta, img . Delta); scalars
		if ((rc = bsg_spmm_launch(m, 1, d.p, r.p, n, s))) break;
		if ((rc = bsg_precond_apply(c, f, p, r.p, img.p, t.p, w.p))) break;
		if ((rc = bsg_dots_launch(c, 2, n, d.p, D.p, img.p, D.p, nullptr, nullptr, sc + L_DD))) break;
		BSG_COUNT(2);
		k_lz_scal<<<1, 1, 0, s>>>(sc, k);
		// x <- (x ro + x1 (1 - ro)) + delta ro gamma
		k_lz_three<1><<<g, 256, 0, s>>>(n, sc, d_x, sol1.p, d.p);
		// true residual and its norms
		if ((rc = bsg_spmm_launch(m, 1, d_x, r.p, n, s))) break;
		if ((rc = bsg_residual_launch(c, n, d_b, r.p))) break;
		norms(r.p);
		BSG_CUDA(cudaMemcpyAsync(c->h_pinned, sc + L_DD, 10 * sizeof(double), cudaMemcpyDeviceToHost, s));
		BSG_CUDA(cudaStreamSynchronize(s));
		const double *h = c->h_pinned; // h[j] = sc[L_DD + j]
		resi = std::sqrt(h[L_RR - L_DD]);
		const double errloc = h[L_EMAX - L_DD];
		if (errloc < errmin) {
			BSG_CUDA(cudaMemcpyAsync(good.p, d_x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
			errmin = errloc;
		}
		const double dd = h[L_DDPREV - L_DD], dd1 = h[L_DD1 - L_DD];
		const bool brk = std::fabs(dd) < 1.e-100 && std::fabs(dd1) < 1.e-100;
		if ((p->sttype == 2 && errmin <= p->eps) || (p->sttype == 0 && resi <= p->eps) ||
		    (p->sttype == 1 && resi <= p->eps * resini) || brk)
			break;
		// delta <- (delta ro + delta1 (1 - ro)) - img ro gamma
		BSG_COUNT(1);
		k_lz_three<-1><<<g, 256, 0, s>>>(n, sc, d.p, d1.p, img.p);
		// img = A^T L^{-T} U^{-T} Delta
		if ((rc = bsg_trisolve_t_launch(c, f, 0, p->trisolve, p->nsweeps, D.p, pv.p, w.p))) break;
		if ((rc = bsg_trisolve_t_launch(c, f, 1, p->trisolve, p->nsweeps, pv.p, r.p, w.p))) break;
		if ((rc = mvm_t(c, m, r.p, img.p))) break;
		// Delta <- (Delta ro + Delta1 (1 - ro)) - img ro gamma
		BSG_COUNT(1);
		k_lz_three<-1><<<g, 256, 0, s>>>(n, sc, D.p, D1.p, img.p);
		BSG_CUDA(cudaGetLastError());
	}
	if (rc) return bsg_set_error(rc, "Lanczos iteration failed");
	if (k >= p->niter) status = BSG_ERR_NOCONV;
	cudaEventRecord(c->ev1, s);
	// the iterate of least max-norm residual is the answer
	BSG_CUDA(cudaMemcpyAsync(d_x, good.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
	if ((rc = bsg_check_devstat(c))) return rc;
	double res = 0;
	if ((rc = bsg_true_residual(c, m, d_b, d_x, r.p, &res))) return rc;
	float ms = 0;
	cudaEventElapsedTime(&ms, c->ev0, c->ev1);
	p->timeitr = ms * 1e-3;
	p->nitperf = k;
	p->resfin = res;
	p->resrec = errmin;
	if (status) return bsg_set_error(status, "iteration limit reached");
	return BSG_OK;
}
