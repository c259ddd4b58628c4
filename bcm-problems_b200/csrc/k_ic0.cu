// Incomplete Cholesky without fill, IC(0): the reference's CSMatrixR::Ich
// (Bslib/ich2r.cpp:1821-1895), the factorisation CSVector::SolveSymm
// (CSMatrixR&) runs for fcttyp = 1 (Bslib/solvers.cpp:4698-4707).
//
// The reference works on the rows of A^T (the lower triangle by rows, columns
// ascending, diagonal last).  For row i and each off-diagonal column k in
// ascending order it forms
//     l_ik = (a_ik - sum_m l_km l_im) * d_k,   d_k = 1 / sqrt(pivot_k),
// the sum running over the columns m < k that rows i and k share, in
// ascending m, each term a product then a subtraction (two roundings); then
//     pivot_i = a_ii - sum_k l_ik^2  (ascending k),  clamped below at 1e-20,
//     d_i = 1 / sqrt(pivot_i),
// and transposes back: U by rows with d_i in the diagonal slot.  The pattern
// is A's.
//
// On the GPU every row is one warp's work, rows claimed in ascending order
// (a topological order: a row needs only smaller rows); lane 0 runs the
// row's merge loops in the reference's order with the same roundings
// (__dmul_rn / __dsub_rn: no fused multiply-add), so the factor is the
// reference's bit for bit.  A row waits for the rows it needs through a
// per-row done flag (acquire / release), each wait bounded by the spin-wait
// limit.  The row's depth in the dependency graph is recorded for the level
// schedule of the triangular solves.
#include "bsg_internal.cuh"
#include <cub/device/device_radix_sort.cuh>

int bsg_strict_transpose(bsg_ctx *c, int n, const int *ia, const int *ja, int nnz, int **it_o, int **jt_o,
                         int **perm_o, int *nnz_o);
int bsg_fct_finish(bsg_ctx *c, bsg_fct *f);

namespace {

inline int nb(long long n, int t) { return n > 0 ? (int)((n + t - 1) / t) : 1; }

// Wait (lane 0) until row k is done; false on the spin limit or another
// failure.
__device__ bool wait_done(const int *done, int k, bsg_devstat *st) {
	if (ld_acquire(done + k)) return true;
	const unsigned long long t0 = globaltimer_ns();
	for (unsigned it = 1;; it++) {
		__nanosleep(32);
		if (ld_acquire(done + k)) return true;
		if ((it & 127) == 0) {
			if (*(volatile int *)&st->code != 0) return false;
			if (globaltimer_ns() - t0 > BSG_SPIN_LIMIT_NS) {
				devstat_fail(st, BSG_ERR_TIMEOUT, k);
				return false;
			}
		}
	}
}

// it / jt: strict lower rows (row i: the columns k < i with A(k, i) stored,
// ascending); lpos[t]: position of A(jt[t], i) in the upper arrays; iu: upper
// row starts (the diagonal first); a: upper values.  Out: lv[t] = l_ik for
// the lower entries, dinv[i], lev[i].
__global__ void k_ic0_rows(int n, const int *__restrict__ it, const int *__restrict__ jt, const int *__restrict__ lpos,
                           const int *__restrict__ iu, const double *__restrict__ a, double *lv, double *dinv,
                           int *lev, int *done, unsigned *claim, bsg_devstat *st) {
	const int lane = threadIdx.x & 31;
	for (;;) {
		int i = 0;
		if (lane == 0) i = (int)atomicAdd(claim, 1u);
		i = __shfl_sync(0xffffffffu, i, 0);
		if (i >= n) return;
		if (lane == 0) {
			bool ok = true;
			int depth = 0;
			const int i1 = it[i], i2 = it[i + 1];
			for (int j = i1; j < i2 && ok; j++) {
				const int k = jt[j];
				if (!wait_done(done, k, st)) { ok = false; break; }
				depth = max(depth, __ldcg(lev + k) + 1);
				double r = a[lpos[j]];
				int ik = it[k], ik2 = it[k + 1], q = i1;
				while (ik < ik2 && q < j) {
					const int ck = jt[ik], cq = jt[q];
					if (ck < cq) {
						ik++;
					} else if (ck > cq) {
						q++;
					} else {
						r = __dsub_rn(r, __dmul_rn(__ldcg(lv + ik), lv[q]));
						q++;
						ik++;
					}
				}
				lv[j] = __dmul_rn(r, __ldcg(dinv + k));
			}
			if (ok) {
				double r = a[iu[i]];
				for (int j = i1; j < i2; j++) r = __dsub_rn(r, __dmul_rn(lv[j], lv[j]));
				if (r < 1.0e-20) r = 1.0e-20;
				dinv[i] = 1.0 / sqrt(r);
				lev[i] = depth;
			} else {
				// a failed wait: publish something so no other row waits on
				// this one past the status check
				dinv[i] = 0.0;
				lev[i] = depth;
			}
			__threadfence();
			st_release(done + i, 1);
		}
		__syncwarp();
	}
}

// U by rows on A's upper pattern: the inverse pivot in the diagonal slot,
// u(k, i) = l_ik elsewhere
__global__ void k_ic0_scatter_diag(int n, const int *iu, const double *dinv, double *u) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) u[iu[i]] = dinv[i];
}
__global__ void k_ic0_scatter_off(int nk, const int *lpos, const double *lv, double *u) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < nk) u[lpos[t]] = lv[t];
}
__global__ void k_ic0_level_keys(int n, const int *lev, unsigned long long *keys, int *vals) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	keys[i] = ((unsigned long long)(unsigned)lev[i] << 32) | (unsigned)i;
	vals[i] = i;
}

struct Dev {
	void *p = nullptr;
	cudaStream_t s = nullptr;
	~Dev() { if (p) cudaFreeAsync(p, s); }
};

} // namespace

// IC(0) of a symmetric point matrix created from its upper triangle.
int bsg_ic0_run(bsg_ctx *c, bsg_mat *m, bsg_fct **out) {
	if (m->bs != 1 || !m->symm)
		return bsg_set_error(BSG_ERR_UNSUPPORTED, "IC(0): a symmetric point matrix (upper-triangle input) is needed");
	const int n = m->n, nnz = m->nnz_up;
	cudaStream_t s = c->stream;
	int *it = nullptr, *jt = nullptr, *lpos = nullptr, nk = 0;
	cudaEventRecord(c->ev0, s);
	int rc = bsg_strict_transpose(c, n, m->d_iu, m->d_ju, nnz, &it, &jt, &lpos, &nk);
	if (rc) return rc;
	Dev dit, djt, dlp, dlv, ddinv, dlev, ddone, dclaim, dkeys, dk2, dvals, dtmp;
	for (Dev *d : {&dit, &djt, &dlp, &dlv, &ddinv, &dlev, &ddone, &dclaim, &dkeys, &dk2, &dvals, &dtmp}) d->s = s;
	dit.p = it;
	djt.p = jt;
	dlp.p = lpos;
	BSG_CUDA(cudaMallocAsync(&dlv.p, sizeof(double) * (nk > 0 ? nk : 1), s));
	BSG_CUDA(cudaMallocAsync(&ddinv.p, sizeof(double) * (n > 0 ? n : 1), s));
	BSG_CUDA(cudaMallocAsync(&dlev.p, sizeof(int) * (n > 0 ? n : 1), s));
	BSG_CUDA(cudaMallocAsync(&ddone.p, sizeof(int) * (n > 0 ? n : 1), s));
	BSG_CUDA(cudaMallocAsync(&dclaim.p, sizeof(unsigned), s));
	BSG_CUDA(cudaMemsetAsync(ddone.p, 0, sizeof(int) * (n > 0 ? n : 1), s));
	BSG_CUDA(cudaMemsetAsync(dclaim.p, 0, sizeof(unsigned), s));
	BSG_CUDA(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), s));
	BSG_COUNT(1);
	k_ic0_rows<<<BSG_SMS * 8, 256, 0, s>>>(n, it, jt, lpos, m->d_iu, m->d_al, (double *)dlv.p, (double *)ddinv.p,
	                                       (int *)dlev.p, (int *)ddone.p, (unsigned *)dclaim.p, c->d_stat);
	BSG_CUDA(cudaGetLastError());
	rc = bsg_check_devstat(c);
	if (rc) return rc;
	bsg_fct *f = new (std::nothrow) bsg_fct();
	if (!f) return bsg_set_error(BSG_ERR_NOMEM, "IC(0) factor");
	f->ctx = c;
	f->n = n;
	f->bs = 1;
	f->kind = 0;
	f->nnz = nnz;
	f->density = 1.0;
	f->density2 = 0.0;
	rc = BSG_OK;
	if (cudaMallocAsync(&f->d_iu, sizeof(int) * (n + 1), s) != cudaSuccess ||
	    cudaMallocAsync(&f->d_ju, sizeof(int) * (nnz > 0 ? nnz : 1), s) != cudaSuccess ||
	    cudaMallocAsync(&f->d_u, sizeof(double) * (nnz > 0 ? nnz : 1), s) != cudaSuccess ||
	    cudaMallocAsync(&f->d_perm, sizeof(int) * (n > 0 ? n : 1), s) != cudaSuccess)
		rc = bsg_set_error(BSG_ERR_NOMEM, "IC(0) factor");
	if (!rc) {
		f->d_l = f->d_u;
		cudaMemcpyAsync(f->d_iu, m->d_iu, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, s);
		cudaMemcpyAsync(f->d_ju, m->d_ju, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s);
		BSG_COUNT(3);
		k_ic0_scatter_diag<<<nb(n, 256), 256, 0, s>>>(n, m->d_iu, (double *)ddinv.p, f->d_u);
		k_ic0_scatter_off<<<nb(nk, 256), 256, 0, s>>>(nk, lpos, (double *)dlv.p, f->d_u);
		// the level schedule of the triangular solves: rows by (depth, index)
		if (cudaMallocAsync(&dkeys.p, sizeof(unsigned long long) * (n > 0 ? n : 1), s) != cudaSuccess ||
		    cudaMallocAsync(&dk2.p, sizeof(unsigned long long) * (n > 0 ? n : 1), s) != cudaSuccess ||
		    cudaMallocAsync(&dvals.p, sizeof(int) * (n > 0 ? n : 1), s) != cudaSuccess)
			rc = bsg_set_error(BSG_ERR_NOMEM, "IC(0) level schedule");
	}
	if (!rc) {
		k_ic0_level_keys<<<nb(n, 256), 256, 0, s>>>(n, (int *)dlev.p, (unsigned long long *)dkeys.p, (int *)dvals.p);
		size_t tb = 0;
		cub::DeviceRadixSort::SortPairs(nullptr, tb, (unsigned long long *)dkeys.p, (unsigned long long *)dk2.p,
		                                (int *)dvals.p, f->d_perm, n, 0, 64, s);
		if (cudaMallocAsync(&dtmp.p, tb > 0 ? tb : 1, s) != cudaSuccess) rc = bsg_set_error(BSG_ERR_NOMEM, "IC(0) sort");
		if (!rc && cub::DeviceRadixSort::SortPairs(dtmp.p, tb, (unsigned long long *)dkeys.p, (unsigned long long *)dk2.p,
		                                           (int *)dvals.p, f->d_perm, n, 0, 64, s) != cudaSuccess)
			rc = bsg_set_error(BSG_ERR_CUDA, "IC(0) sort");
	}
	if (!rc) {
		unsigned long long last = 0;
		if (n > 0)
			cudaMemcpyAsync(&last, (unsigned long long *)dk2.p + (n - 1), sizeof(last), cudaMemcpyDeviceToHost, s);
		if (cudaStreamSynchronize(s) != cudaSuccess) rc = bsg_set_error(BSG_ERR_CUDA, "IC(0)");
		f->levels_l = f->levels_u = n > 0 ? (int)(last >> 32) + 1 : 0;
	}
	cudaEventRecord(c->ev1, s);
	if (!rc) rc = bsg_fct_finish(c, f);
	if (rc) {
		bsg_fct_free(f);
		return rc;
	}
	*out = f;
	return BSG_OK;
}
