// Block (3 x 3) second-order incomplete LU: the reference's CSMatrixRS::Ilu2
// (Bslib/ilu2rs.cpp:1458-1820) on the GPU, with its SVD scaling of the
// diagonal blocks (Ilu2AllocScale, :25-315), block filtering with diagonal
// compensation (Ilu2FiltrRow, :616-692), SVD pivots (Ilu2PivScaleRow,
// :694-852) and the final back-scaling (Ich2StoreScaleU,
// Bslib/ich2rs.cpp:822-943); and the block triangular solves of its factor
// (CSMatrixRS::SolveL / SolveU, Bslib/mvm.cpp:3140 / 3410).
//
// Blocks are column-major 3 x 3 (entry (r, c) at r + 3 c), as CSMatrixRS
// keeps them.
//
// Rows.  The block rows are factored by the point factorisation's kernel in
// its block mode (k_fact.cu, bsg_bfact_dyn): a warp per block row on the
// dynamic schedule (closure of the members over finished rows, admission,
// waiting, parking); the members' updates are applied in ascending member
// order, the compensations of dropped blocks reach the dropped column's
// pivot block through exact fixed-point sums, so the factor does not depend
// on the schedule.  This file builds the scaled CombineLU block matrix
// before, and the reference layout and the solve-ready forms after.  The SVD
// is this file's own, so the factor agrees with the reference to rounding,
// not bit for bit; a singular vector's sign cancels in L U, but for (nearly)
// repeated singular values the reference's vectors and these differ by a
// rotation, which can move a block across a threshold.
#include "bsg_internal.cuh"
#include "bsg_blk3.cuh"
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace {

inline int nb_(long long n, int t) { return n > 0 ? (int)((n + t - 1) / t) : 1; }

// ---- CombineLU of a block matrix on the device ----------------------------
// keys (row, col) of the union pattern: upper blocks (j >= i) at (i, j),
// lower blocks (j <= i) transposed to (j, i); the source is 2 p (upper) or
// 2 p + 1 (lower) for the block p of A
__global__ void k_bc_keys(int nb, const int *ia, const int *ja, const int *off, unsigned long long *keys, int *src) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nb) return;
	int o = off[i];
	for (int p = ia[i]; p < ia[i + 1]; p++) {
		const int j = ja[p];
		if (j >= i) {
			keys[o] = ((unsigned long long)i << 32) | (unsigned)j;
			src[o++] = 2 * p;
		}
		if (j <= i) {
			keys[o] = ((unsigned long long)j << 32) | (unsigned)i;
			src[o++] = 2 * p + 1;
		}
	}
}
__global__ void k_bc_count(int nb, const int *ia, const int *ja, int *cnt) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nb) return;
	int c = 0;
	for (int p = ia[i]; p < ia[i + 1]; p++) c += (ja[p] >= i) + (ja[p] <= i);
	cnt[i] = c;
}
__global__ void k_bc_flags(int nk, const unsigned long long *keys, int *flag) {
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e < nk) flag[e] = (e == 0 || keys[e] != keys[e - 1]) ? 1 : 0;
}
// id[e] = inclusive count of distinct keys - 1; row counts of the pattern
__global__ void k_bc_pattern(int nk, const unsigned long long *keys, const int *id, const int *flag, int *bja,
                             int *rowcnt) {
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= nk || !flag[e]) return;
	bja[id[e] - 1] = (int)(keys[e] & 0xffffffffu);
	atomicAdd(rowcnt + (int)(keys[e] >> 32), 1);
}
// values: au = the block (column-major), al = the block transposed
// (column-major); A's blocks arrive row-major
__global__ void k_bc_values(int nk, const int *src, const int *id, const double *a, double *al, double *au) {
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= nk) return;
	const int s = src[e], p = s >> 1;
	const double *b = a + (size_t)p * 9; // row-major: (r, c) at 3 r + c
	double *o = ((s & 1) ? al : au) + (size_t)(id[e] - 1) * 9;
	for (int r = 0; r < 3; r++)
		for (int c = 0; c < 3; c++) o[r + 3 * c] = (s & 1) ? b[3 * c + r] : b[3 * r + c];
}

// ---- scaling of the diagonal blocks (Ilu2AllocScale) ----------------------
// sym (block IC2, Ich2AllocScale Bslib/ich2rs.cpp:26-250): the diagonal
// block is symmetric; its eigenvectors (V) scale both sides, no sclmin
// clamp, and a negative eigenvalue (u_k . v_k < 0) is a pivot error
__global__ void k_bscale(int nb, int sym, const int *bia, const double *au, double sclmin, double *scll, double *sclu,
                         double *sinvl, double *sinvu, double *diagg, bsg_devstat *st) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nb) return;
	const double *d = au + (size_t)bia[i] * 9;
	double u[9], v[9], s[3];
	svd3(d, u, s, v);
	if (sym) {
		for (int k = 0; k < 3; k++) {
			if (u[3 * k] * v[3 * k] + u[1 + 3 * k] * v[1 + 3 * k] + u[2 + 3 * k] * v[2 + 3 * k] < 0.0 && s[k] > 0.0)
				devstat_fail(st, BSG_ERR_PIVOT, i, 1);
			for (int r = 0; r < 3; r++) u[r + 3 * k] = v[r + 3 * k];
		}
		for (int k = 0; k < 3; k++) s[k] = sqrt(s[k]);
	} else {
		for (int k = 0; k < 3; k++) s[k] = sqrt(s[k] < sclmin ? sclmin : s[k]);
	}
	double *il = sinvl + (size_t)i * 9, *iu = sinvu + (size_t)i * 9, *sl = scll + (size_t)i * 9,
	       *su = sclu + (size_t)i * 9;
	for (int r = 0; r < 3; r++)
		for (int c = 0; c < 3; c++) {
			il[r + 3 * c] = u[r + 3 * c] * s[c]; // U diag(s^1/2)
			iu[r + 3 * c] = v[r + 3 * c] * s[c]; // V diag(s^1/2)
			sl[r + 3 * c] = u[c + 3 * r] / s[r]; // diag(s^-1/2) U^T
			su[r + 3 * c] = v[c + 3 * r] / s[r]; // diag(s^-1/2) V^T
		}
	double t[9];
	mm3(sl, 1, 3, d, 1, 3, t);                 // scll D
	mm3(t, 1, 3, su, 3, 1, diagg + (size_t)i * 9); // ... sclu^T
}

// ---- final: the U part scaled back (Ich2StoreScaleU) ----------------------
__global__ void k_bfin_count(int nb, const int *ig, const int *jg, int *cnt) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nb) return;
	int c = 0;
	for (int q = ig[i]; q < ig[i + 1]; q++) c += jg[q] >= 0;
	cnt[i] = c;
}
__global__ void k_bfin_fill(int nb, const int *ig, const int *jg, const double *gl, const double *gu,
                            const double *scll, const double *sclu, const double *sinvl, const double *sinvu,
                            const int *fi, int *fj, double *fl, double *fu) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nb) return;
	int o = fi[i];
	for (int q = ig[i]; q < ig[i + 1]; q++) {
		const int j = jg[q];
		if (j < 0) continue;
		fj[o] = j;
		if (j == i) { // scl^T g
			mm3(scll + (size_t)i * 9, 3, 1, gl + (size_t)q * 9, 1, 3, fl + (size_t)o * 9);
			mm3(sclu + (size_t)i * 9, 3, 1, gu + (size_t)q * 9, 1, 3, fu + (size_t)o * 9);
		} else { // g sclinv^T
			mm3(gl + (size_t)q * 9, 1, 3, sinvl + (size_t)j * 9, 3, 1, fl + (size_t)o * 9);
			mm3(gu + (size_t)q * 9, 1, 3, sinvu + (size_t)j * 9, 3, 1, fu + (size_t)o * 9);
		}
		o++;
	}
}

// ---- solve-ready forms ------------------------------------------------------
// point rows of the strict parts: the U solve reads row 3 i + r of U's
// strict blocks (U_ik(r, c) at column 3 k + c); the L solve reads the
// transpose of L's strict blocks (L_ki(c, r) at row 3 i + r, column 3 k + c),
// built here by first writing each entry under its (row, column) key
__global__ void k_bsu_count(int nb, const int *fi, int *cnt) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nb) return;
	const int nbk = fi[i + 1] - fi[i] - 1;
	for (int r = 0; r < 3; r++) cnt[3 * i + r] = 3 * nbk;
}
__global__ void k_bsu_fill(int nb, const int *fi, const int *fj, const double *fu, const int *rp, int *ci,
                           double *v) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nb) return;
	for (int r = 0; r < 3; r++) {
		int o = rp[3 * i + r];
		for (int q = fi[i] + 1; q < fi[i + 1]; q++)
			for (int c = 0; c < 3; c++) {
				ci[o] = 3 * fj[q] + c;
				v[o++] = fu[(size_t)q * 9 + r + 3 * c];
			}
	}
}
// keys (row, col) and values of the transposed strict L entries
__global__ void k_bsl_keys(int nb, const int *fi, const int *fj, const double *fl, unsigned long long *keys,
                           double *vals) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x; // block row k of the storage
	if (i >= nb) return;
	long long o = 9LL * (fi[i] - i); // strict blocks before row i
	for (int q = fi[i] + 1; q < fi[i + 1]; q++) {
		const int j = fj[q];
		for (int c = 0; c < 3; c++)
			for (int r = 0; r < 3; r++) { // entry (c, r) of L_ij lands at row 3 j + r, column 3 i + c
				keys[o] = ((unsigned long long)(3 * j + r) << 32) | (unsigned)(3 * i + c);
				vals[o++] = fl[(size_t)q * 9 + c + 3 * r];
			}
	}
}
__global__ void k_keys_to_csr(long long nk, const unsigned long long *keys, int *ci, int *cnt) {
	const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= nk) return;
	ci[e] = (int)(keys[e] & 0xffffffffu);
	atomicAdd(cnt + (int)(keys[e] >> 32), 1);
}
// diagonal action of the solves: L: y_i = L_ii^T t_i; U: y_i = U_ii t_i
__global__ void k_bdiag_pack(int nb, const int *fi, const double *fl, const double *fu, double *dlt, double *du) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nb) return;
	const double *l = fl + (size_t)fi[i] * 9, *u = fu + (size_t)fi[i] * 9;
	for (int r = 0; r < 3; r++)
		for (int c = 0; c < 3; c++) {
			dlt[(size_t)i * 9 + r + 3 * c] = l[c + 3 * r];
			du[(size_t)i * 9 + r + 3 * c] = u[r + 3 * c];
		}
}
// y = D t per block (D column-major), t and y may alias
// Exact block solve, one warp walking the block rows in dependency order
// (lower: ascending, upper: descending): y_i = D_i (x_i - N_i y) with N's
// point rows 3 i .. 3 i + 2 gathered by the lanes.  Latency-bound: the
// parity mode of the block factor.
__global__ void k_bsolve_seq(int nb, int lower, const int *rp, const int *ci, const double *v, const double *d,
                             const double *x, double *y) {
	const int lane = threadIdx.x;
	for (int s = 0; s < nb; s++) {
		const int i = lower ? s : nb - 1 - s;
		double t[3];
		for (int r = 0; r < 3; r++) {
			double acc = 0.0;
			for (int p = rp[3 * i + r] + lane; p < rp[3 * i + r + 1]; p += 32) acc += v[p] * __ldcg(y + ci[p]);
			t[r] = x[3 * i + r] - warp_sum(acc);
		}
		if (lane < 3) {
			const double *b = d + (size_t)i * 9;
			__stcg(y + 3 * i + lane, b[lane] * t[0] + b[lane + 3] * t[1] + b[lane + 6] * t[2]);
		}
		__threadfence_block();
		__syncwarp();
	}
}

} // namespace

// ---- host ------------------------------------------------------------------
struct DevVec {
	void *p = nullptr;
	cudaStream_t s = nullptr;
	~DevVec() { if (p) cudaFreeAsync(p, s); }
};
#define BALLOC(var, type, count)                                                                           \
	type *var = nullptr;                                                                                   \
	DevVec var##_h;                                                                                        \
	BSG_CUDA(cudaMallocAsync(&var, sizeof(type) * (size_t)((count) > 0 ? (count) : 1), st));             \
	var##_h.p = var;                                                                                       \
	var##_h.s = st;

// point CSR from sorted (row, col) keys
static int keys_csr(cudaStream_t st, int n, long long nk, unsigned long long *keys, double *vals, int **rp,
                    int **ci, double **v) {
	unsigned long long *k2;
	double *v2;
	BSG_CUDA(cudaMallocAsync(&k2, sizeof(unsigned long long) * (nk > 0 ? nk : 1), st));
	BSG_CUDA(cudaMallocAsync(&v2, sizeof(double) * (nk > 0 ? nk : 1), st));
	size_t tmp = 0;
	BSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, k2, vals, v2, (int)nk, 0, 64, st));
	void *dt;
	BSG_CUDA(cudaMallocAsync(&dt, tmp + 1, st));
	BSG_CUDA(cub::DeviceRadixSort::SortPairs(dt, tmp, keys, k2, vals, v2, (int)nk, 0, 64, st));
	cudaFreeAsync(dt, st);
	int *cnt;
	BSG_CUDA(cudaMallocAsync(&cnt, sizeof(int) * (n + 1), st));
	BSG_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (n + 1), st));
	BSG_CUDA(cudaMallocAsync(ci, sizeof(int) * (nk > 0 ? nk : 1), st));
	BSG_COUNT(1);
	if (nk > 0) k_keys_to_csr<<<nb_(nk, 256), 256, 0, st>>>(nk, k2, *ci, cnt);
	BSG_CUDA(cudaMallocAsync(rp, sizeof(int) * (n + 1), st));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, *rp, n + 1, st));
	BSG_CUDA(cudaMallocAsync(&dt, tmp + 1, st));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(dt, tmp, cnt, *rp, n + 1, st));
	cudaFreeAsync(dt, st);
	cudaFreeAsync(cnt, st);
	cudaFreeAsync(k2, st);
	*v = v2;
	return BSG_OK;
}

// Block ILU2 (sym 0) or block IC2 (sym 1, the matrix symmetric) of a 3 x 3
// block matrix: the factor f gets the block form
// (d_bia / d_bja / d_bl / d_bu, column-major blocks) and the solve-ready
// forms (strict parts as point CSR + SELL copies, block diagonals).
int bsg_bfact_run(bsg_ctx *c, bsg_mat *m, int sym, const bsg_param *p, bsg_fct **out) {
	if (m->bs != 3) return bsg_set_error(BSG_ERR_UNSUPPORTED, "block factorisation: 3 x 3 blocks only");
	cudaStream_t st = c->stream;
	const int nb = m->n;
	BSG_CUDA(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), st));
	BSG_CUDA(cudaEventRecord(c->ev0, st));
	// ---- CombineLU on the device
	BALLOC(cnt, int, nb + 1);
	BALLOC(koff, int, nb + 1);
	BSG_CUDA(cudaMemsetAsync(cnt + nb, 0, sizeof(int), st));
	BSG_COUNT(1);
	k_bc_count<<<nb_(nb, 256), 256, 0, st>>>(nb, m->d_ia, m->d_ja, cnt);
	size_t tmp = 0;
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, koff, nb + 1, st));
	BALLOC(dtmp, char, tmp + 1);
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(dtmp, tmp, cnt, koff, nb + 1, st));
	int nk = 0;
	BSG_CUDA(cudaMemcpyAsync(&nk, koff + nb, sizeof(int), cudaMemcpyDeviceToHost, st));
	BSG_CUDA(cudaStreamSynchronize(st));
	BALLOC(keys, unsigned long long, nk);
	BALLOC(keys2, unsigned long long, nk);
	BALLOC(src, int, nk);
	BALLOC(src2, int, nk);
	BSG_COUNT(1);
	k_bc_keys<<<nb_(nb, 256), 256, 0, st>>>(nb, m->d_ia, m->d_ja, koff, keys, src);
	size_t t2 = 0;
	BSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t2, keys, keys2, src, src2, nk, 0, 64, st));
	BALLOC(dtmp2, char, t2 + 1);
	BSG_CUDA(cub::DeviceRadixSort::SortPairs(dtmp2, t2, keys, keys2, src, src2, nk, 0, 64, st));
	BALLOC(flag, int, nk);
	BALLOC(id, int, nk);
	BSG_COUNT(1);
	k_bc_flags<<<nb_(nk, 256), 256, 0, st>>>(nk, keys2, flag);
	size_t t3 = 0;
	BSG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, t3, flag, id, nk, st));
	BALLOC(dtmp3, char, t3 + 1);
	BSG_CUDA(cub::DeviceScan::InclusiveSum(dtmp3, t3, flag, id, nk, st));
	int nnzb = 0;
	BSG_CUDA(cudaMemcpyAsync(&nnzb, id + nk - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
	BSG_CUDA(cudaStreamSynchronize(st));
	BALLOC(bja, int, nnzb);
	BALLOC(bia, int, nb + 1);
	BALLOC(rowcnt, int, nb + 1);
	BSG_CUDA(cudaMemsetAsync(rowcnt, 0, sizeof(int) * (nb + 1), st));
	BALLOC(bal, double, (long long)nnzb * 9);
	BALLOC(bau, double, (long long)nnzb * 9);
	BSG_CUDA(cudaMemsetAsync(bal, 0, sizeof(double) * 9 * (size_t)nnzb, st));
	BSG_CUDA(cudaMemsetAsync(bau, 0, sizeof(double) * 9 * (size_t)nnzb, st));
	BSG_COUNT(2);
	k_bc_pattern<<<nb_(nk, 256), 256, 0, st>>>(nk, keys2, id, flag, bja, rowcnt);
	k_bc_values<<<nb_(nk, 256), 256, 0, st>>>(nk, src2, id, m->d_a, bal, bau);
	size_t t4 = 0;
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t4, rowcnt, bia, nb + 1, st));
	BALLOC(dtmp4, char, t4 + 1);
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(dtmp4, t4, rowcnt, bia, nb + 1, st));
	// ---- scaling
	BALLOC(scll, double, (long long)nb * 9);
	BALLOC(sclu, double, (long long)nb * 9);
	BALLOC(sinvl, double, (long long)nb * 9);
	BALLOC(sinvu, double, (long long)nb * 9);
	BALLOC(diagg, double, (long long)nb * 9);
	BSG_COUNT(1);
	k_bscale<<<nb_(nb, 128), 128, 0, st>>>(nb, sym, bia, bau, p->sclmin, scll, sclu, sinvl, sinvu, diagg, c->d_stat);
	// ---- the rows, a warp each, on the dynamic schedule of the point factorisation
	BALLOC(nstored, unsigned long long, 2);
	int *ig = nullptr, *jg = nullptr;
	double *gl = nullptr, *gu = nullptr;
	{
		const int rcd = bsg_bfact_dyn(c, nb, sym, p, bia, bja, nnzb, bal, bau, scll, sclu, diagg, &ig, &jg, &gl, &gu,
		                              nstored);
		if (rcd) return rcd;
	}
	DevVec ig_h, jg_h, gl_h, gu_h;
	ig_h.p = ig; jg_h.p = jg; gl_h.p = gl; gu_h.p = gu;
	ig_h.s = jg_h.s = gl_h.s = gu_h.s = st;
	int rc = bsg_check_devstat(c);
	if (rc) return rc;
	// ---- U part scaled back
	BALLOC(fcnt, int, nb + 1);
	BSG_CUDA(cudaMemsetAsync(fcnt + nb, 0, sizeof(int), st));
	BSG_COUNT(1);
	k_bfin_count<<<nb_(nb, 256), 256, 0, st>>>(nb, ig, jg, fcnt);
	bsg_fct *f = new bsg_fct();
	f->ctx = c;
	f->n = 3 * nb;
	f->bs = 3;
	f->nb = nb;
	f->kind = sym ? 0 : 1;
	auto fail = [&](int code) {
		bsg_fct_free(f);
		return code;
	};
#define FCUDA(call)                                                             \
	do {                                                                        \
		cudaError_t e_ = (call);                                                \
		if (e_ != cudaSuccess) return fail(bsg_set_cuda_error(e_, #call, __FILE__, __LINE__)); \
	} while (0)
	FCUDA(cudaMallocAsync(&f->d_bia, sizeof(int) * (nb + 1), st));
	size_t t5 = 0;
	FCUDA(cub::DeviceScan::ExclusiveSum(nullptr, t5, fcnt, f->d_bia, nb + 1, st));
	void *dt5;
	FCUDA(cudaMallocAsync(&dt5, t5 + 1, st));
	FCUDA(cub::DeviceScan::ExclusiveSum(dt5, t5, fcnt, f->d_bia, nb + 1, st));
	cudaFreeAsync(dt5, st);
	int nf = 0;
	FCUDA(cudaMemcpyAsync(&nf, f->d_bia + nb, sizeof(int), cudaMemcpyDeviceToHost, st));
	unsigned long long hs[2];
	FCUDA(cudaMemcpyAsync(hs, nstored, sizeof(hs), cudaMemcpyDeviceToHost, st));
	FCUDA(cudaStreamSynchronize(st));
	f->nnz = nf;
	FCUDA(cudaMallocAsync(&f->d_bja, sizeof(int) * (nf > 0 ? nf : 1), st));
	FCUDA(cudaMallocAsync(&f->d_bl, sizeof(double) * 9 * (size_t)(nf > 0 ? nf : 1), st));
	FCUDA(cudaMallocAsync(&f->d_bu, sizeof(double) * 9 * (size_t)(nf > 0 ? nf : 1), st));
	BSG_COUNT(1);
	k_bfin_fill<<<nb_(nb, 128), 128, 0, st>>>(nb, ig, jg, gl, gu, scll, sclu, sinvl, sinvu, f->d_bia, f->d_bja,
	                                           f->d_bl, f->d_bu);
	FCUDA(cudaGetLastError());
	f->density = 9.0 * (double)hs[0] / (9.0 * (double)nnzb);
	f->density2 = 9.0 * (double)hs[1] / (9.0 * (double)nnzb);
	FCUDA(cudaEventRecord(c->ev1, st));
	// ---- solve-ready forms
	const int n = 3 * nb;
	const long long nstrict = 9LL * (nf - nb);
	FCUDA(cudaMallocAsync(&f->d_ur_i, sizeof(int) * (n + 1), st));
	{
		int *ucnt;
		FCUDA(cudaMallocAsync(&ucnt, sizeof(int) * (n + 1), st));
		FCUDA(cudaMemsetAsync(ucnt + n, 0, sizeof(int), st));
		BSG_COUNT(1);
		k_bsu_count<<<nb_(nb, 256), 256, 0, st>>>(nb, f->d_bia, ucnt);
		size_t t6 = 0;
		FCUDA(cub::DeviceScan::ExclusiveSum(nullptr, t6, ucnt, f->d_ur_i, n + 1, st));
		void *dt6;
		FCUDA(cudaMallocAsync(&dt6, t6 + 1, st));
		FCUDA(cub::DeviceScan::ExclusiveSum(dt6, t6, ucnt, f->d_ur_i, n + 1, st));
		cudaFreeAsync(dt6, st);
		cudaFreeAsync(ucnt, st);
	}
	FCUDA(cudaMallocAsync(&f->d_ur_j, sizeof(int) * (nstrict > 0 ? nstrict : 1), st));
	FCUDA(cudaMallocAsync(&f->d_ur_v, sizeof(double) * (nstrict > 0 ? nstrict : 1), st));
	BSG_COUNT(1);
	k_bsu_fill<<<nb_(nb, 256), 256, 0, st>>>(nb, f->d_bia, f->d_bja, f->d_bu, f->d_ur_i, f->d_ur_j, f->d_ur_v);
	{
		unsigned long long *lk;
		double *lv;
		FCUDA(cudaMallocAsync(&lk, sizeof(unsigned long long) * (nstrict > 0 ? nstrict : 1), st));
		FCUDA(cudaMallocAsync(&lv, sizeof(double) * (nstrict > 0 ? nstrict : 1), st));
		BSG_COUNT(1);
		k_bsl_keys<<<nb_(nb, 256), 256, 0, st>>>(nb, f->d_bia, f->d_bja, f->d_bl, lk, lv);
		int rc2 = keys_csr(st, n, nstrict, lk, lv, &f->d_lr_i, &f->d_lr_j, &f->d_lr_v);
		cudaFreeAsync(lk, st);
		cudaFreeAsync(lv, st);
		if (rc2) return fail(rc2);
	}
	f->nnz_strict = (int)nstrict;
	FCUDA(cudaMallocAsync(&f->d_bdl, sizeof(double) * 9 * (size_t)nb, st));
	FCUDA(cudaMallocAsync(&f->d_bdu, sizeof(double) * 9 * (size_t)nb, st));
	BSG_COUNT(1);
	k_bdiag_pack<<<nb_(nb, 256), 256, 0, st>>>(nb, f->d_bia, f->d_bl, f->d_bu, f->d_bdl, f->d_bdu);
	int rc3 = bsg_bsell_build(c, nb, f->d_lr_i, f->d_lr_j, f->d_lr_v, 0, &f->bsl);
	if (!rc3) rc3 = bsg_bsell_build(c, nb, f->d_ur_i, f->d_ur_j, f->d_ur_v, 0, &f->bsu);
	if (rc3) return fail(rc3);
	FCUDA(cudaStreamSynchronize(st));
#undef FCUDA
	*out = f;
	return BSG_OK;
}

// FP32 values for the sweeps' strict parts (block diagonals stay FP64)
int bsg_bfact_make_fp32(bsg_fct *f) {
	cudaStream_t s = f->ctx->stream;
	bsg_bsell_free(&f->bsl, s);
	bsg_bsell_free(&f->bsu, s);
	int rc = bsg_bsell_build(f->ctx, f->nb, f->d_lr_i, f->d_lr_j, f->d_lr_v, 1, &f->bsl);
	if (!rc) rc = bsg_bsell_build(f->ctx, f->nb, f->d_ur_i, f->d_ur_j, f->d_ur_v, 1, &f->bsu);
	if (rc) return rc;
	f->fp32 = 1;
	return BSG_OK;
}

// Block triangular solve (lower: SolveL, else SolveU).  mode 0: exact (one
// warp, rows in order); mode 1: nsweeps Jacobi iterates y <- D (x - N y)
// from y = D x on the block SELL copies, work = n doubles.
int bsg_btrisolve_launch(bsg_ctx *c, const bsg_fct *f, int lower, int mode, int nsweeps, const double *x, double *y,
                         double *work) {
	cudaStream_t s = c->stream;
	const int nb = f->nb;
	const double *d = lower ? f->d_bdl : f->d_bdu;
	if (mode == 0) {
		BSG_COUNT(1);
		if (lower) k_bsolve_seq<<<1, 32, 0, s>>>(nb, 1, f->d_lr_i, f->d_lr_j, f->d_lr_v, d, x, y);
		else k_bsolve_seq<<<1, 32, 0, s>>>(nb, 0, f->d_ur_i, f->d_ur_j, f->d_ur_v, d, x, y);
		BSG_CUDA(cudaGetLastError());
		return BSG_OK;
	}
	if (nsweeps < 1) return bsg_set_error(BSG_ERR_ARG, "block sweeps: nsweeps >= 1");
	return bsg_bsell_sweeps(s, lower ? &f->bsl : &f->bsu, d, nsweeps, 1, x, y, work);
}

// nr block triangular solves, vectors at stride n = 3 nb (work: n nr
// doubles).  Sweeps read the block SELL copy once per 8 vectors and give
// every vector the bits of its own solve; exact solves run one at a time.
int bsg_btrisolve_multi(bsg_ctx *c, const bsg_fct *f, int lower, int mode, int nsweeps, int nr, const double *x,
                        double *y, double *work) {
	const int n = f->n;
	if (mode == 0 || nr == 1) {
		for (int q = 0; q < nr; q++) {
			const size_t o = (size_t)q * n;
			int rc = bsg_btrisolve_launch(c, f, lower, mode, nsweeps, x + o, y + o, work ? work + o : nullptr);
			if (rc) return rc;
		}
		return BSG_OK;
	}
	if (nsweeps < 1) return bsg_set_error(BSG_ERR_ARG, "block sweeps: nsweeps >= 1");
	// the interleaved iterates' scratch, kept with the factor; grown only
	// outside stream capture (inside, the sweeps go through y and work)
	const size_t need = nsweeps > 1 ? bsg_bsell_scratch(f->nb, nr) : 0;
	bsg_fct *fm = const_cast<bsg_fct *>(f);
	if (need > f->swscr_n) {
		cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
		if (cudaStreamIsCapturing(c->stream, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
			if (fm->d_swscr) cudaFreeAsync(fm->d_swscr, c->stream);
			fm->d_swscr = nullptr;
			fm->swscr_n = 0;
			if (cudaMallocAsync(&fm->d_swscr, sizeof(double) * need, c->stream) == cudaSuccess) fm->swscr_n = need;
			else fm->d_swscr = nullptr;
		}
	}
	return bsg_bsell_sweeps(c->stream, lower ? &f->bsl : &f->bsu, lower ? f->d_bdl : f->d_bdu, nsweeps, nr, x, y,
	                        work, need > 0 && need <= f->swscr_n ? fm->d_swscr : nullptr);
}
