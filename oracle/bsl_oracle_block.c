/* Block (CSMatrixRS) part of the CPU oracle -- test infrastructure only.
 *
 * A CPU restatement of the reference's block second-order incomplete LU
 * (CSMatrixRS::Ilu2, Bslib/ilu2rs.cpp:1458-1820) with its block scaling
 * (Ilu2AllocScale, :25-315), and of the block triangular solves
 * (CSMatrixRS::SolveL, Bslib/mvm.cpp:3140; SolveU, :3410).  Only tests,
 * __graft_entry__.smoke() and bench.py's CPU baseline use it; the product
 * never does.
 *
 * Storage: block CSR with a uniform block size B, block k of a matrix at
 * a[k * B * B], column-major (entry (r, c) at r + c * B), each block row's
 * diagonal block first -- the layout of CSMatrixRS (Bslib/smatrix.h:1040).
 *
 * The singular value decompositions of the diagonal blocks are LAPACK's
 * dgesvd (job "A", "A"), the routine the reference calls; the oracle links
 * the same OpenBLAS build.  Products are summed in the reference's order and
 * the updates of a row are applied in the order its linked lists give them
 * (Ich2UpdateTransp, Bslib/ich2r.cpp:296), so the factor agrees with the
 * compiled reference bit for bit.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "bsl_oracle.h"

extern void dsyev_(const char *jobz, const char *uplo, const int *n, double *a, const int *lda, double *w,
                   double *work, const int *lwork, int *info);
extern void dgesvd_(const char *jobu, const char *jobvt, const int *m, const int *n, double *a, const int *lda,
                    double *s, double *u, const int *ldu, double *vt, const int *ldvt, double *work, const int *lwork,
                    int *info);

/* ---- CombineLU (Bslib/smatrixrs.cpp:1645-1806) ---------------------------
 * U: the blocks with column >= row, as stored; L: the blocks with column <=
 * row, transposed into row (column) j, block (i, j) -> (j, i) with its B x B
 * block transposed; then both patterns are extended to their union (missing
 * blocks are zero). */
int orc_combine_lu_block(int nb, int bs, const int *ia, const int *ja, const double *a, int **ia_s, int **ja_s,
                         double **al, double **au) {
	const int b2 = bs * bs;
	int *cl = calloc((size_t)nb + 1, sizeof(int));
	if (!cl) return -1;
	for (int i = 0; i < nb; i++)
		for (int p = ia[i]; p < ia[i + 1]; p++)
			if (ja[p] <= i) cl[ja[p] + 1]++;
	for (int i = 0; i < nb; i++) cl[i + 1] += cl[i];
	int *lj = malloc(sizeof(int) * (cl[nb] > 0 ? cl[nb] : 1));
	double *lv = malloc(sizeof(double) * (size_t)(cl[nb] > 0 ? cl[nb] : 1) * b2);
	int *pos = malloc(sizeof(int) * (nb > 0 ? nb : 1));
	if (!lj || !lv || !pos) return -1;
	memcpy(pos, cl, sizeof(int) * nb);
	for (int i = 0; i < nb; i++) /* ascending rows: each transposed row comes out sorted */
		for (int p = ia[i]; p < ia[i + 1]; p++) {
			const int j = ja[p];
			if (j > i) continue;
			const int q = pos[j]++;
			lj[q] = i;
			for (int r = 0; r < bs; r++)
				for (int c = 0; c < bs; c++) lv[(size_t)q * b2 + c + r * bs] = a[(size_t)p * b2 + r + c * bs];
		}
	/* union of the two patterns, row by row (both sorted; the diagonal first) */
	int *is = malloc(sizeof(int) * ((size_t)nb + 1));
	int cap = ia[nb] + cl[nb];
	int *js = malloc(sizeof(int) * (cap > 0 ? cap : 1));
	double *vl = calloc((size_t)(cap > 0 ? cap : 1) * b2, sizeof(double));
	double *vu = calloc((size_t)(cap > 0 ? cap : 1) * b2, sizeof(double));
	if (!is || !js || !vl || !vu) return -1;
	int nz = 0;
	is[0] = 0;
	for (int i = 0; i < nb; i++) {
		int pu = ia[i], eu = ia[i + 1], pl = cl[i], el = cl[i + 1];
		while (pu < eu && ja[pu] < i) pu++; /* upper part of the row */
		while (pu < eu || pl < el) {
			const int ju = pu < eu ? ja[pu] : 0x7fffffff, jl = pl < el ? lj[pl] : 0x7fffffff;
			const int j = ju < jl ? ju : jl;
			js[nz] = j;
			if (ju == j) {
				memcpy(vu + (size_t)nz * b2, a + (size_t)pu * b2, sizeof(double) * b2);
				pu++;
				while (pu < eu && ja[pu] < i) pu++;
			}
			if (jl == j) {
				memcpy(vl + (size_t)nz * b2, lv + (size_t)pl * b2, sizeof(double) * b2);
				pl++;
			}
			nz++;
		}
		is[i + 1] = nz;
	}
	free(cl);
	free(lj);
	free(lv);
	free(pos);
	*ia_s = is;
	*ja_s = js;
	*al = vl;
	*au = vu;
	return 0;
}

/* One-sided Jacobi (Hestenes) SVD of a 3 x 3 block, s descending, U
 * completed by Gram-Schmidt of unit vectors where a singular value vanishes:
 * the algorithm the GPU path uses for its pivot and scaling blocks
 * (bcm-problems_b200/csrc/k_bfact.cu, svd3).  Restated here so that the GPU
 * factor can be checked against an oracle that takes the same SVD; vt holds
 * V^T like dgesvd's output. */
static void svd3_jacobi(const double *a, double *s, double *u, double *vt) {
	double w[9], vw[9];
	for (int k = 0; k < 9; k++) {
		w[k] = a[k];
		vw[k] = (k % 4) == 0 ? 1.0 : 0.0;
	}
	for (int sweep = 0; sweep < 30; sweep++) {
		double off2 = 0.0; /* largest ga^2 / (al be) of the sweep */
		for (int pq = 0; pq < 3; pq++) {
			const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
			double al = 0.0, be = 0.0, ga = 0.0;
			for (int r = 0; r < 3; r++) {
				al += w[r + 3 * p] * w[r + 3 * p];
				be += w[r + 3 * q] * w[r + 3 * q];
				ga += w[r + 3 * p] * w[r + 3 * q];
			}
			const double ab = al * be, g2 = ga * ga;
			if (ab == 0.0 || g2 <= 1e-32 * ab) continue;
			if (g2 / ab > off2) off2 = g2 / ab;
			const double zeta = (be - al) / (2.0 * ga);
			const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
			const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
			for (int r = 0; r < 3; r++) {
				const double wp = w[r + 3 * p], wq = w[r + 3 * q];
				w[r + 3 * p] = cs * wp - sn * wq;
				w[r + 3 * q] = sn * wp + cs * wq;
				const double vp = vw[r + 3 * p], vq = vw[r + 3 * q];
				vw[r + 3 * p] = cs * vp - sn * vq;
				vw[r + 3 * q] = sn * vp + cs * vq;
			}
		}
		if (off2 <= 1e-30) break;
	}
	double sv[3];
	for (int c = 0; c < 3; c++) sv[c] = sqrt(w[3 * c] * w[3 * c] + w[1 + 3 * c] * w[1 + 3 * c] + w[2 + 3 * c] * w[2 + 3 * c]);
	int o[3] = {0, 1, 2}, good[3];
	if (sv[o[0]] < sv[o[1]]) { const int t = o[0]; o[0] = o[1]; o[1] = t; }
	if (sv[o[1]] < sv[o[2]]) { const int t = o[1]; o[1] = o[2]; o[2] = t; }
	if (sv[o[0]] < sv[o[1]]) { const int t = o[0]; o[0] = o[1]; o[1] = t; }
	const double smax = sv[o[0]];
	for (int c = 0; c < 3; c++) {
		const int k = o[c];
		s[c] = sv[k];
		good[c] = sv[k] > 1e-300 && sv[k] > 1e-14 * smax;
		for (int r = 0; r < 3; r++) {
			u[r + 3 * c] = good[c] ? w[r + 3 * k] / sv[k] : 0.0;
			vt[c + 3 * r] = vw[r + 3 * k]; /* V^T(c, r) = V(r, c) */
		}
	}
	for (int c = 0; c < 3; c++) {
		if (good[c]) continue;
		for (int e = 0; e < 3; e++) {
			double x[3] = {e == 0 ? 1.0 : 0.0, e == 1 ? 1.0 : 0.0, e == 2 ? 1.0 : 0.0};
			for (int d = 0; d < 3; d++) {
				if (d == c || !good[d]) continue;
				const double pr = u[3 * d] * x[0] + u[1 + 3 * d] * x[1] + u[2 + 3 * d] * x[2];
				for (int r = 0; r < 3; r++) x[r] -= pr * u[r + 3 * d];
			}
			const double nx = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
			if (nx > 0.5) {
				for (int r = 0; r < 3; r++) u[r + 3 * c] = x[r] / nx;
				good[c] = 1;
				break;
			}
		}
	}
}

static int g_svd_jacobi = 0; /* orc_ilu2_block_jacobi / orc_ich2_block_jacobi set it for one call */

/* Eigenpairs of a symmetric 3 x 3 block as the GPU path takes them: the
 * Jacobi SVD above, the right singular vectors as eigenvectors (q column-
 * major, descending) and the singular values as eigenvalues; a pair whose
 * left and right vectors point opposite ways (u_k . v_k < 0, s_k > 0) is a
 * negative eigenvalue (-2). */
static int sym_eig3_jacobi(const double *a, double *eig, double *q) {
	double a0[9], s[3], u[9], vt[9];
	memcpy(a0, a, sizeof a0);
	svd3_jacobi(a0, s, u, vt);
	for (int k = 0; k < 3; k++) {
		if (u[3 * k] * vt[k] + u[1 + 3 * k] * vt[k + 3] + u[2 + 3 * k] * vt[k + 6] < 0.0 && s[k] > 0.0) return -2;
		eig[k] = s[k];
		for (int r = 0; r < 3; r++) q[r + 3 * k] = vt[k + 3 * r];
	}
	return 0;
}

/* The SVD of one B x B block as the reference takes it: dgesvd for B > 1,
 * the sign split for B == 1 (Bslib/ilu2rs.cpp:118-140, :717-740).  a is
 * overwritten; u and vt are column-major (vt holds V^T). */
static int block_svd(int bs, double *a, double *s, double *u, double *vt, double *work, int lwork) {
	if (bs == 3 && g_svd_jacobi) {
		double a0[9];
		memcpy(a0, a, sizeof a0);
		svd3_jacobi(a0, s, u, vt);
		return 0;
	}
	if (bs > 1) {
		int info = 0;
		dgesvd_("A", "A", &bs, &bs, a, &bs, s, u, &bs, vt, &bs, work, &lwork, &info);
		return info;
	}
	u[0] = 1.0;
	if (a[0] >= 0.0) {
		vt[0] = 1.0;
		s[0] = a[0];
	} else {
		vt[0] = -1.0;
		s[0] = -a[0];
	}
	return 0;
}

static double block_maxabs(int b2, const double *x, const double *y) {
	double m = 0.0;
	for (int k = 0; k < b2; k++) {
		double v = fabs(x[k]);
		if (v > m) m = v;
	}
	for (int k = 0; k < b2; k++) {
		double v = fabs(y[k]);
		if (v > m) m = v;
	}
	return m;
}

static int cmp_int(const void *x, const void *y) {
	const int a = *(const int *)x, b = *(const int *)y;
	return (a > b) - (a < b);
}

/* out(kii, kjj) = sum_k p(kii, k) q(k, kjj) with p given transposed-or-not by
 * strides: element (r, c) of p at p[r * pr + c * pc]; sums from 0 in k order */
static void mm(int bs, const double *p, int pr, int pc, const double *q, int qr, int qc, double *out) {
	for (int r = 0; r < bs; r++)
		for (int c = 0; c < bs; c++) {
			double s = 0.0;
			for (int k = 0; k < bs; k++) s += p[r * pr + k * pc] * q[k * qr + c * qc];
			out[r + c * bs] = s;
		}
}

/* Block ILU2 of a CombineLU'd block matrix (is, js: union pattern, diagonal
 * block first; al: transposed lower blocks; au: upper blocks).  Output: the
 * U part of the factor, L and U on the same pattern (ia_f / ja_f, blocks in
 * l / u), scaled back as Ich2StoreScaleU does (Bslib/ich2rs.cpp:822-943).
 * stats: [0] density, [1] density2 (as CSlvParam), [2] factor seconds (0).
 * Returns 0, -1 (allocation) or -3 (LAPACK failure). */
int orc_ilu2_block(int nb, int bs, const int *is, const int *js, const double *al, const double *au, double tau1,
                   double tau2, double theta, double sclmin, double pivmin, int **ia_f, int **ja_f, double **l,
                   double **u, double *stats) {
	const int b2 = bs * bs, lwork = 10 * bs;
	double *scll = malloc(sizeof(double) * (size_t)nb * b2), *sclu = malloc(sizeof(double) * (size_t)nb * b2);
	double *sinvl = malloc(sizeof(double) * (size_t)nb * b2), *sinvu = malloc(sizeof(double) * (size_t)nb * b2);
	double *diagg = malloc(sizeof(double) * (size_t)nb * b2);
	double *fml = calloc((size_t)nb * b2, sizeof(double)), *fmu = calloc((size_t)nb * b2, sizeof(double));
	int *imask = malloc(sizeof(int) * nb), *lstloc = malloc(sizeof(int) * nb), *lstupd = malloc(sizeof(int) * nb);
	int *indlst = malloc(sizeof(int) * nb), *iv = malloc(sizeof(int) * nb), *madj = malloc(sizeof(int) * nb);
	int *ibegm = malloc(sizeof(int) * nb);
	double aloc[64], vloc[64], uloc[64], eig[8], work[80], deleml[64], delemu[64], lel[64], uel[64];
	if (bs > 8 || !scll || !sclu || !sinvl || !sinvu || !diagg || !fml || !fmu || !imask || !lstloc || !lstupd ||
	    !indlst || !iv || !madj || !ibegm)
		return -1;
	int rc = 0;

	/* ---- scaling of every diagonal block (Ilu2AllocScale) ---- */
	for (int i = 0; i < nb; i++) {
		const double *d = au + (size_t)is[i] * b2;
		double *sl = scll + (size_t)i * b2, *su = sclu + (size_t)i * b2;
		double *il = sinvl + (size_t)i * b2, *iu = sinvu + (size_t)i * b2;
		memcpy(aloc, d, sizeof(double) * b2);
		if (block_svd(bs, aloc, eig, uloc, vloc, work, lwork)) return -3;
		for (int k = 0; k < bs; k++) {
			if (eig[k] < sclmin) eig[k] = sclmin;
			eig[k] = sqrt(eig[k]);
		}
		for (int r = 0; r < bs; r++)
			for (int c = 0; c < bs; c++) {
				il[r + c * bs] = uloc[r + c * bs] * eig[c]; /* U diag(s^1/2) */
				iu[r + c * bs] = vloc[c + r * bs] * eig[c]; /* V diag(s^1/2) */
			}
		for (int k = 0; k < bs; k++) eig[k] = 1.0 / eig[k];
		for (int r = 0; r < bs; r++)
			for (int c = 0; c < bs; c++) {
				sl[r + c * bs] = uloc[c + r * bs] * eig[r]; /* diag(s^-1/2) U^T */
				su[r + c * bs] = vloc[r + c * bs] * eig[r]; /* diag(s^-1/2) V^T */
			}
		/* diagg = scll * D * sclu^T */
		mm(bs, sl, 1, bs, d, 1, bs, aloc);
		mm(bs, aloc, 1, bs, su, bs, 1, diagg + (size_t)i * b2);
	}

	/* ---- factor storage (grows as needed) ---- */
	int cap = is[nb] * 2 + nb + 16, nzjg = 0;
	int *ig = malloc(sizeof(int) * ((size_t)nb + 1)), *jg = malloc(sizeof(int) * cap), *addrg = malloc(sizeof(int) * cap);
	double *gl = malloc(sizeof(double) * (size_t)cap * b2), *gu = malloc(sizeof(double) * (size_t)cap * b2);
	if (!ig || !jg || !addrg || !gl || !gu) return -1;
	ig[0] = 0;
	int icycle = -1;
	for (int i = 0; i < nb; i++) {
		imask[i] = -1;
		iv[i] = -1;
		madj[i] = -1;
		ibegm[i] = -1;
	}
	long long nzu = 0, nzr = 0;

	for (int irow = 0; irow < nb; irow++) {
		icycle++;
		/* ---- scaled row of A (Ilu2InitRow) ---- */
		int nlist1 = 0;
		lstloc[nlist1++] = irow;
		imask[irow] = icycle;
		memcpy(fml + (size_t)irow * b2, diagg + (size_t)irow * b2, sizeof(double) * b2);
		memcpy(fmu + (size_t)irow * b2, diagg + (size_t)irow * b2, sizeof(double) * b2);
		const double *sli = scll + (size_t)irow * b2, *sui = sclu + (size_t)irow * b2;
		for (int p = is[irow] + 1; p < is[irow + 1]; p++) {
			const int jj = js[p];
			lstloc[nlist1++] = jj;
			imask[jj] = icycle;
			mm(bs, sli, 1, bs, au + (size_t)p * b2, 1, bs, aloc);
			mm(bs, aloc, 1, bs, sclu + (size_t)jj * b2, bs, 1, fmu + (size_t)jj * b2);
			mm(bs, sui, 1, bs, al + (size_t)p * b2, 1, bs, aloc);
			mm(bs, aloc, 1, bs, scll + (size_t)jj * b2, bs, 1, fml + (size_t)jj * b2);
		}
		/* ---- updates by the previous rows, in linked-list order ---- */
		for (int k = ibegm[irow]; k != -1; k = madj[k]) {
			const int j0 = iv[k];
			const int elmisr = jg[j0] < 0;
			memcpy(lel, gl + (size_t)addrg[j0] * b2, sizeof(double) * b2);
			memcpy(uel, gu + (size_t)addrg[j0] * b2, sizeof(double) * b2);
			int nupd = 0;
			for (int q = j0; q < ig[k + 1]; q++) { /* Ilu2InitMask */
				int jc = jg[q];
				if (elmisr && jc < 0) continue;
				if (jc < 0) jc = -jc;
				if (imask[jc] != icycle) {
					imask[jc] = icycle;
					lstloc[nlist1++] = jc;
					memset(fml + (size_t)jc * b2, 0, sizeof(double) * b2);
					memset(fmu + (size_t)jc * b2, 0, sizeof(double) * b2);
				}
				lstupd[nupd] = jc;
				indlst[nupd] = q;
				nupd++;
			}
			/* Ich2UpdateRow twice: fmu -= lel^T gu, fml -= uel^T gl, products
			 * subtracted one by one */
			for (int t = 0; t < nupd; t++) {
				double *fu = fmu + (size_t)lstupd[t] * b2;
				const double *g = gu + (size_t)addrg[indlst[t]] * b2;
				for (int r = 0; r < bs; r++)
					for (int c = 0; c < bs; c++)
						for (int m = 0; m < bs; m++) fu[r + c * bs] -= lel[m + r * bs] * g[m + c * bs];
			}
			for (int t = 0; t < nupd; t++) {
				double *fl = fml + (size_t)lstupd[t] * b2;
				const double *g = gl + (size_t)addrg[indlst[t]] * b2;
				for (int r = 0; r < bs; r++)
					for (int c = 0; c < bs; c++)
						for (int m = 0; m < bs; m++) fl[r + c * bs] -= uel[m + r * bs] * g[m + c * bs];
			}
		}
		/* ---- move the rows of this column's list to their next column ---- */
		{
			int k = ibegm[irow];
			while (k != -1) {
				const int k1 = madj[k];
				if (iv[k] >= ig[k + 1] - 1) {
					madj[k] = -1;
				} else {
					int c = jg[iv[k] + 1];
					if (c < 0) c = -c;
					madj[k] = ibegm[c];
					ibegm[c] = k;
				}
				iv[k]++;
				k = k1;
			}
		}
		/* ---- filtering with diagonal compensation (Ilu2FiltrRow) ---- */
		int nlist2 = 0;
		double *fdi = fmu + (size_t)irow * b2;
		for (int t = 1; t < nlist1; t++) {
			const int j = lstloc[t];
			const double *fl = fml + (size_t)j * b2, *fu = fmu + (size_t)j * b2;
			if (block_maxabs(b2, fl, fu) >= tau2) {
				lstupd[nlist2++] = j;
			} else {
				double *dj = diagg + (size_t)j * b2;
				for (int r = 0; r < bs; r++)
					for (int c = 0; c < bs; c++) {
						double v = fabs(fl[r + c * bs]), w = fabs(fu[r + c * bs]);
						if (w > v) v = w;
						v *= theta;
						fdi[r + r * bs] += v;
						dj[c + c * bs] += v;
					}
			}
		}
		nlist1 = nlist2;
		/* ---- pivot block and row scaling (Ilu2PivScaleRow) ---- */
		memcpy(aloc, fdi, sizeof(double) * b2);
		if (block_svd(bs, aloc, eig, uloc, vloc, work, lwork)) return -3;
		for (int k = 0; k < bs; k++) {
			if (eig[k] < pivmin) eig[k] = pivmin;
			eig[k] = sqrt(eig[k]);
			eig[k] = 1.0 / eig[k];
		}
		for (int r = 0; r < bs; r++)
			for (int c = 0; c < bs; c++) {
				deleml[r + c * bs] = uloc[c + r * bs] * eig[r]; /* diag(s^-1/2) U^T */
				delemu[r + c * bs] = vloc[r + c * bs] * eig[r]; /* diag(s^-1/2) V^T */
			}
		for (int t = 0; t < nlist1; t++) {
			double *fl = fml + (size_t)lstupd[t] * b2, *fu = fmu + (size_t)lstupd[t] * b2;
			mm(bs, delemu, 1, bs, fl, 1, bs, aloc);
			memcpy(fl, aloc, sizeof(double) * b2);
			mm(bs, deleml, 1, bs, fu, 1, bs, aloc);
			memcpy(fu, aloc, sizeof(double) * b2);
		}
		/* ---- store the row: the pivot block, then U / R blocks ---- */
		if (nlist1) qsort(lstupd, nlist1, sizeof(int), cmp_int);
		if (nzjg + nlist1 + 1 > cap) {
			while (nzjg + nlist1 + 1 > cap) cap *= 2;
			jg = realloc(jg, sizeof(int) * cap);
			addrg = realloc(addrg, sizeof(int) * cap);
			gl = realloc(gl, sizeof(double) * (size_t)cap * b2);
			gu = realloc(gu, sizeof(double) * (size_t)cap * b2);
			if (!jg || !addrg || !gl || !gu) return -1;
		}
		if (nlist1) {
			iv[irow] = nzjg + 1;
			madj[irow] = ibegm[lstupd[0]];
			ibegm[lstupd[0]] = irow;
		}
		jg[nzjg] = irow;
		addrg[nzjg] = nzjg;
		for (int r = 0; r < bs; r++)
			for (int c = 0; c < bs; c++) {
				gl[(size_t)nzjg * b2 + r + c * bs] = deleml[c + r * bs];
				gu[(size_t)nzjg * b2 + r + c * bs] = delemu[c + r * bs];
			}
		nzjg++;
		nzu += b2;
		for (int t = 0; t < nlist1; t++) {
			const int j = lstupd[t];
			const double *fl = fml + (size_t)j * b2, *fu = fmu + (size_t)j * b2;
			const int keep = block_maxabs(b2, fl, fu) >= tau1;
			jg[nzjg] = keep ? j : -j;
			addrg[nzjg] = nzjg;
			memcpy(gl + (size_t)nzjg * b2, fl, sizeof(double) * b2);
			memcpy(gu + (size_t)nzjg * b2, fu, sizeof(double) * b2);
			if (keep) nzu += b2;
			else nzr += b2;
			nzjg++;
		}
		ig[irow + 1] = nzjg;
	}

	/* ---- U part, scaled back (Ich2StoreScaleU) ---- */
	int nkeep = 0;
	for (int q = 0; q < nzjg; q++)
		if (jg[q] >= 0) nkeep++;
	int *fi = malloc(sizeof(int) * ((size_t)nb + 1)), *fj = malloc(sizeof(int) * (nkeep > 0 ? nkeep : 1));
	double *fl = malloc(sizeof(double) * (size_t)(nkeep > 0 ? nkeep : 1) * b2);
	double *fu = malloc(sizeof(double) * (size_t)(nkeep > 0 ? nkeep : 1) * b2);
	if (!fi || !fj || !fl || !fu) return -1;
	int o = 0;
	fi[0] = 0;
	for (int i = 0; i < nb; i++) {
		for (int q = ig[i]; q < ig[i + 1]; q++) {
			const int jj = jg[q];
			if (jj < 0) continue;
			fj[o] = jj;
			const double *g1 = gl + (size_t)addrg[q] * b2, *g2 = gu + (size_t)addrg[q] * b2;
			if (jj == i) { /* scl^T g */
				mm(bs, scll + (size_t)i * b2, bs, 1, g1, 1, bs, fl + (size_t)o * b2);
				mm(bs, sclu + (size_t)i * b2, bs, 1, g2, 1, bs, fu + (size_t)o * b2);
			} else { /* g sclinv^T */
				mm(bs, g1, 1, bs, sinvl + (size_t)jj * b2, bs, 1, fl + (size_t)o * b2);
				mm(bs, g2, 1, bs, sinvu + (size_t)jj * b2, bs, 1, fu + (size_t)o * b2);
			}
			o++;
		}
		fi[i + 1] = o;
	}
	if (stats) {
		const double nza = (double)is[nb] * b2;
		stats[0] = (double)nzu / nza;
		stats[1] = (double)nzr / nza;
		stats[2] = 0.0;
	}
	*ia_f = fi;
	*ja_f = fj;
	*l = fl;
	*u = fu;
	free(scll); free(sclu); free(sinvl); free(sinvu); free(diagg); free(fml); free(fmu);
	free(imask); free(lstloc); free(lstupd); free(indlst); free(iv); free(madj); free(ibegm);
	free(ig); free(jg); free(addrg); free(gl); free(gu);
	return rc;
}

/* y = L-solve of x with L stored by block columns (CSMatrixRS::SolveL):
 * y_i = D_i^T (x_i - ...), then y_k -= L_ik^T y_i for the row's other blocks */
void orc_solve_l_block(int nb, int bs, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	const int b2 = bs * bs;
	double v[8];
	memcpy(y, x, sizeof(double) * (size_t)nb * bs);
	for (int i = 0; i < nb; i++) {
		const double *d = a + (size_t)ia[i] * b2;
		double *yi = y + (size_t)i * bs;
		for (int r = 0; r < bs; r++) {
			double s = 0.0;
			for (int c = 0; c < bs; c++) s += d[c + r * bs] * yi[c];
			v[r] = s;
		}
		memcpy(yi, v, sizeof(double) * bs);
		for (int p = ia[i] + 1; p < ia[i + 1]; p++) {
			const double *b = a + (size_t)p * b2;
			double *yk = y + (size_t)ja[p] * bs;
			for (int r = 0; r < bs; r++)
				for (int c = 0; c < bs; c++) yk[r] -= b[c + r * bs] * yi[c];
		}
	}
}

/* y = U-solve of x with U stored by block rows (CSMatrixRS::SolveU):
 * y_i = D_i (x_i - sum_k U_ik y_k), rows from last to first */
void orc_solve_u_block(int nb, int bs, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	const int b2 = bs * bs;
	double v[8];
	for (int i = nb - 1; i >= 0; i--) {
		memcpy(v, x + (size_t)i * bs, sizeof(double) * bs);
		for (int p = ia[i] + 1; p < ia[i + 1]; p++) {
			const double *b = a + (size_t)p * b2;
			const double *yk = y + (size_t)ja[p] * bs;
			for (int r = 0; r < bs; r++)
				for (int c = 0; c < bs; c++) v[r] -= b[r + c * bs] * yk[c];
		}
		const double *d = a + (size_t)ia[i] * b2;
		double *yi = y + (size_t)i * bs;
		for (int r = 0; r < bs; r++) {
			double s = 0.0;
			for (int c = 0; c < bs; c++) s += d[r + c * bs] * v[c];
			yi[r] = s;
		}
	}
}

/* orc_ilu2_block with the GPU path's Jacobi SVD in place of dgesvd (3 x 3
 * blocks): the oracle that the GPU block factor is checked against value by
 * value. */
int orc_ilu2_block_jacobi(int nb, int bs, const int *is, const int *js, const double *al, const double *au,
                          double tau1, double tau2, double theta, double sclmin, double pivmin, int **ia_f, int **ja_f,
                          double **l, double **u, double *stats) {
	g_svd_jacobi = 1;
	const int rc = orc_ilu2_block(nb, bs, is, js, al, au, tau1, tau2, theta, sclmin, pivmin, ia_f, ja_f, l, u, stats);
	g_svd_jacobi = 0;
	return rc;
}

/* Block IC2 of an upper-stored symmetric block matrix (CSMatrixRS::Ich2,
 * Bslib/ich2rs.cpp:1075-1380): the symmetric form of the block ILU2 above
 * with one mask, the diagonal blocks scaled by their eigenvectors (LAPACK
 * dsyev, Ich2AllocScale :26-250) and the pivots taken from the
 * eigendecomposition of the pivot block, eigenvalues in descending order
 * (Ich2PivScaleRow :532-647).  A negative eigenvalue is an error (-2), as
 * the reference throws.  Output: U (L = U^T) on its pattern, scaled back
 * (Ich2StoreScaleU :822-943); stats as orc_ilu2_block. */
int orc_ich2_block(int nb, int bs, const int *ia, const int *ja, const double *a, double tau1, double tau2,
                   double theta, int **ia_f, int **ja_f, double **uo, double *stats) {
	const int b2 = bs * bs, lwork = 10 * bs;
	double *scl = malloc(sizeof(double) * (size_t)nb * b2), *sinv = malloc(sizeof(double) * (size_t)nb * b2);
	double *diagg = malloc(sizeof(double) * (size_t)nb * b2), *fm = calloc((size_t)nb * b2, sizeof(double));
	int *imask = malloc(sizeof(int) * nb), *lstloc = malloc(sizeof(int) * nb), *lstupd = malloc(sizeof(int) * nb);
	int *indlst = malloc(sizeof(int) * nb), *iv = malloc(sizeof(int) * nb), *madj = malloc(sizeof(int) * nb);
	int *ibegm = malloc(sizeof(int) * nb);
	double aloc[64], vloc[64], eig[8], work[80], delem[64], lel[64];
	if (bs > 8 || !scl || !sinv || !diagg || !fm || !imask || !lstloc || !lstupd || !indlst || !iv || !madj || !ibegm)
		return -1;
	for (int i = 0; i < nb; i++) { /* Ich2AllocScale */
		const double *d = a + (size_t)ia[i] * b2;
		double *sl = scl + (size_t)i * b2, *si = sinv + (size_t)i * b2;
		int info = 0;
		if (bs == 3 && g_svd_jacobi) {
			if (sym_eig3_jacobi(d, eig, aloc)) return -2;
		} else {
			memcpy(aloc, d, sizeof(double) * b2);
			dsyev_("V", "U", &bs, aloc, &bs, eig, work, &lwork, &info);
			if (info) return -3;
		}
		for (int k = 0; k < bs; k++)
			if (eig[k] < 0.0) return -2;
		for (int k = 0; k < bs; k++) eig[k] = sqrt(eig[k]);
		for (int r = 0; r < bs; r++)
			for (int c = 0; c < bs; c++) si[r + c * bs] = aloc[r + c * bs] * eig[c]; /* Q diag(l^1/2) */
		for (int k = 0; k < bs; k++) eig[k] = 1.0 / eig[k];
		for (int r = 0; r < bs; r++)
			for (int c = 0; c < bs; c++) sl[r + c * bs] = aloc[c + r * bs] * eig[r]; /* diag(l^-1/2) Q^T */
		mm(bs, sl, 1, bs, d, 1, bs, aloc);
		mm(bs, aloc, 1, bs, sl, bs, 1, diagg + (size_t)i * b2);
	}
	int cap = ia[nb] * 2 + nb + 16, nzjg = 0;
	int *ig = malloc(sizeof(int) * ((size_t)nb + 1)), *jg = malloc(sizeof(int) * cap), *addrg = malloc(sizeof(int) * cap);
	double *g = malloc(sizeof(double) * (size_t)cap * b2);
	if (!ig || !jg || !addrg || !g) return -1;
	ig[0] = 0;
	int icycle = -1;
	for (int i = 0; i < nb; i++) {
		imask[i] = -1;
		iv[i] = -1;
		madj[i] = -1;
		ibegm[i] = -1;
	}
	long long nzu = 0, nzr = 0;
	for (int irow = 0; irow < nb; irow++) {
		icycle++;
		int nlist1 = 0; /* Ich2InitRow */
		lstloc[nlist1++] = irow;
		imask[irow] = icycle;
		memcpy(fm + (size_t)irow * b2, diagg + (size_t)irow * b2, sizeof(double) * b2);
		for (int p = ia[irow] + 1; p < ia[irow + 1]; p++) {
			const int jj = ja[p];
			lstloc[nlist1++] = jj;
			imask[jj] = icycle;
			mm(bs, scl + (size_t)irow * b2, 1, bs, a + (size_t)p * b2, 1, bs, aloc);
			mm(bs, aloc, 1, bs, scl + (size_t)jj * b2, bs, 1, fm + (size_t)jj * b2);
		}
		for (int k = ibegm[irow]; k != -1; k = madj[k]) { /* updates, linked-list order */
			const int j0 = iv[k];
			const int elmisr = jg[j0] < 0;
			memcpy(lel, g + (size_t)addrg[j0] * b2, sizeof(double) * b2);
			int nupd = 0;
			for (int q = j0; q < ig[k + 1]; q++) {
				int jc = jg[q];
				if (elmisr && jc < 0) continue;
				if (jc < 0) jc = -jc;
				if (imask[jc] != icycle) {
					imask[jc] = icycle;
					lstloc[nlist1++] = jc;
					memset(fm + (size_t)jc * b2, 0, sizeof(double) * b2);
				}
				lstupd[nupd] = jc;
				indlst[nupd] = q;
				nupd++;
			}
			for (int t = 0; t < nupd; t++) {
				double *f = fm + (size_t)lstupd[t] * b2;
				const double *gg = g + (size_t)addrg[indlst[t]] * b2;
				for (int r = 0; r < bs; r++)
					for (int c = 0; c < bs; c++)
						for (int m2 = 0; m2 < bs; m2++) f[r + c * bs] -= lel[m2 + r * bs] * gg[m2 + c * bs];
			}
		}
		{
			int k = ibegm[irow];
			while (k != -1) {
				const int k1 = madj[k];
				if (iv[k] >= ig[k + 1] - 1) {
					madj[k] = -1;
				} else {
					int c = jg[iv[k] + 1];
					if (c < 0) c = -c;
					madj[k] = ibegm[c];
					ibegm[c] = k;
				}
				iv[k]++;
				k = k1;
			}
		}
		int nlist2 = 0; /* Ich2FiltrRow */
		double *fdi = fm + (size_t)irow * b2;
		for (int t = 1; t < nlist1; t++) {
			const int j = lstloc[t];
			const double *f = fm + (size_t)j * b2;
			double mx = 0.0;
			for (int k = 0; k < b2; k++) {
				const double v = fabs(f[k]);
				if (v > mx) mx = v;
			}
			if (mx >= tau2) {
				lstupd[nlist2++] = j;
			} else {
				double *dj = diagg + (size_t)j * b2;
				for (int r = 0; r < bs; r++)
					for (int c = 0; c < bs; c++) {
						const double v = fabs(f[r + c * bs]) * theta;
						fdi[r + r * bs] += v;
						dj[c + c * bs] += v;
					}
			}
		}
		nlist1 = nlist2;
		{ /* Ich2PivScaleRow */
			int info = 0;
			if (bs == 3 && g_svd_jacobi) { /* descending already */
				if (sym_eig3_jacobi(fdi, eig, aloc)) return -2;
			} else {
				memcpy(aloc, fdi, sizeof(double) * b2);
				dsyev_("V", "U", &bs, aloc, &bs, eig, work, &lwork, &info);
				if (info) return -3;
				for (int r = 0; r < bs; r++) /* eigenpairs in descending order */
					for (int c = 0; c < bs; c++) delem[(bs - r - 1) * bs + c] = aloc[r * bs + c];
				memcpy(aloc, delem, sizeof(double) * b2);
				for (int k = 0; k < bs; k++) work[bs - k - 1] = eig[k];
				for (int k = 0; k < bs; k++) eig[k] = work[k];
			}
			for (int k = 0; k < bs; k++) {
				if (eig[k] < 0.0) return -2;
				eig[k] = sqrt(eig[k]);
				eig[k] = 1.0 / eig[k];
			}
			for (int r = 0; r < bs; r++)
				for (int c = 0; c < bs; c++) delem[r + c * bs] = aloc[c + r * bs] * eig[r];
			for (int t = 0; t < nlist1; t++) {
				double *f = fm + (size_t)lstupd[t] * b2;
				mm(bs, delem, 1, bs, f, 1, bs, vloc);
				memcpy(f, vloc, sizeof(double) * b2);
			}
		}
		if (nlist1) qsort(lstupd, nlist1, sizeof(int), cmp_int);
		if (nzjg + nlist1 + 1 > cap) {
			while (nzjg + nlist1 + 1 > cap) cap *= 2;
			jg = realloc(jg, sizeof(int) * cap);
			addrg = realloc(addrg, sizeof(int) * cap);
			g = realloc(g, sizeof(double) * (size_t)cap * b2);
			if (!jg || !addrg || !g) return -1;
		}
		if (nlist1) {
			iv[irow] = nzjg + 1;
			madj[irow] = ibegm[lstupd[0]];
			ibegm[lstupd[0]] = irow;
		}
		jg[nzjg] = irow; /* Ich2StoreRow */
		addrg[nzjg] = nzjg;
		for (int r = 0; r < bs; r++)
			for (int c = 0; c < bs; c++) g[(size_t)nzjg * b2 + r + c * bs] = delem[c + r * bs];
		nzjg++;
		nzu += b2;
		for (int t = 0; t < nlist1; t++) {
			const int j = lstupd[t];
			const double *f = fm + (size_t)j * b2;
			double mx = 0.0;
			for (int k = 0; k < b2; k++) {
				const double v = fabs(f[k]);
				if (v > mx) mx = v;
			}
			const int keep = mx >= tau1;
			jg[nzjg] = keep ? j : -j;
			addrg[nzjg] = nzjg;
			memcpy(g + (size_t)nzjg * b2, f, sizeof(double) * b2);
			if (keep) nzu += b2;
			else nzr += b2;
			nzjg++;
		}
		ig[irow + 1] = nzjg;
	}
	int nkeep = 0;
	for (int q = 0; q < nzjg; q++)
		if (jg[q] >= 0) nkeep++;
	int *fi = malloc(sizeof(int) * ((size_t)nb + 1)), *fj = malloc(sizeof(int) * (nkeep > 0 ? nkeep : 1));
	double *fu = malloc(sizeof(double) * (size_t)(nkeep > 0 ? nkeep : 1) * b2);
	if (!fi || !fj || !fu) return -1;
	int o = 0;
	fi[0] = 0;
	for (int i = 0; i < nb; i++) {
		for (int q = ig[i]; q < ig[i + 1]; q++) {
			const int jj = jg[q];
			if (jj < 0) continue;
			fj[o] = jj;
			const double *gg = g + (size_t)addrg[q] * b2;
			if (jj == i) mm(bs, scl + (size_t)i * b2, bs, 1, gg, 1, bs, fu + (size_t)o * b2);
			else mm(bs, gg, 1, bs, sinv + (size_t)jj * b2, bs, 1, fu + (size_t)o * b2);
			o++;
		}
		fi[i + 1] = o;
	}
	if (stats) {
		const double nza = (double)ia[nb] * b2;
		stats[0] = (double)nzu / nza;
		stats[1] = (double)nzr / nza;
		stats[2] = 0.0;
	}
	*ia_f = fi;
	*ja_f = fj;
	*uo = fu;
	free(scl); free(sinv); free(diagg); free(fm); free(imask); free(lstloc); free(lstupd); free(indlst);
	free(iv); free(madj); free(ibegm); free(ig); free(jg); free(addrg); free(g);
	return 0;
}

/* orc_ich2_block with the GPU path's Jacobi eigenpairs (sym_eig3_jacobi) in
 * place of dsyev (3 x 3 blocks): the oracle that the GPU block IC2 factor is
 * checked against value by value. */
int orc_ich2_block_jacobi(int nb, int bs, const int *ia, const int *ja, const double *a, double tau1, double tau2,
                          double theta, int **ia_f, int **ja_f, double **uo, double *stats) {
	g_svd_jacobi = 1;
	const int rc = orc_ich2_block(nb, bs, ia, ja, a, tau1, tau2, theta, ia_f, ja_f, uo, stats);
	g_svd_jacobi = 0;
	return rc;
}
