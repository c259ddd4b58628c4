/* CPU oracle for the Bslib Krylov hot path -- TEST INFRASTRUCTURE ONLY.
 * See bsl_oracle.h for the contract; never linked into the product. */
#include "bsl_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

void orc_free(void *p) { free(p); }

/* y = A x, full storage.  Bslib/mvm.cpp:2489 (CSMatrixR::MvmA). */
void orc_mvm(int n, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	for (int i = 0; i < n; i++) {
		double s = 0.0;
		for (int j = ia[i]; j < ia[i + 1]; j++) s += a[j] * x[ja[j]];
		y[i] = s;
	}
}

/* y = A x, upper triangle stored, transpose scattered.  Bslib/mvm.cpp:2637. */
void orc_mvm_symm(int n, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	for (int i = 0; i < n; i++) y[i] = 0.0;
	for (int i = 0; i < n; i++)
		for (int j = ia[i]; j < ia[i + 1]; j++) {
			int jj = ja[j];
			y[i] += a[j] * x[jj];
			if (jj != i) y[jj] += a[j] * x[i];
		}
}

/* y = A x for uniform bs x bs column-major blocks.  Bslib/mvm.cpp:2530-2568
 * (CSMatrixRS::MvmA): block j of row i at a[bs*bs*j], element (r,c) at
 * a[bs*bs*j + c*bs + r]. */
void orc_bsr_mvm(int nb, int bs, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	for (int i = 0; i < nb * bs; i++) y[i] = 0.0;
	for (int i = 0; i < nb; i++)
		for (int j = ia[i]; j < ia[i + 1]; j++) {
			const double *blk = a + (size_t)j * bs * bs;
			const double *xj = x + (size_t)ja[j] * bs;
			for (int r = 0; r < bs; r++) {
				double s = y[(size_t)i * bs + r];
				for (int c = 0; c < bs; c++) s += blk[c * bs + r] * xj[c];
				y[(size_t)i * bs + r] = s;
			}
		}
}

/* L stored by columns, inverse pivot first.  Bslib/mvm.cpp:3042-3058. */
void orc_solve_l(int n, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	for (int i = 0; i < n; i++) y[i] = x[i];
	for (int i = 0; i < n; i++) {
		y[i] *= a[ia[i]];
		for (int j = ia[i] + 1; j < ia[i + 1]; j++) y[ja[j]] -= a[j] * y[i];
	}
}

/* U stored by rows, inverse pivot first.  Bslib/mvm.cpp:3343-3358. */
void orc_solve_u(int n, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	for (int i = n - 1; i >= 0; i--) {
		double s = x[i];
		for (int j = ia[i] + 1; j < ia[i + 1]; j++) s -= a[j] * y[ja[j]];
		y[i] = s * a[ia[i]];
	}
}

static int cmp_int(const void *a, const void *b) {
	int x = *(const int *)a, y = *(const int *)b;
	return (x > y) - (x < y);
}

/* CombineLU restated: Bslib/smatrixr.cpp:1142-1258 (upper rows, transposed
 * lower rows, both extended to the union pattern). */
int orc_combine_lu(int n, const int *ia, const int *ja, const double *a, int **ia_s, int **ja_s, double **al,
                   double **au) {
	int nz = ia[n];
	int *cnt = (int *)calloc((size_t)n + 1, sizeof(int));
	/* union pattern row i = {j >= i : A(i,j) != 0 or A(j,i) != 0} */
	int *tmpc = (int *)malloc(sizeof(int) * (size_t)(2 * nz + n));
	int *tmpr = (int *)malloc(sizeof(int) * (size_t)(2 * nz + n));
	double *tl = (double *)malloc(sizeof(double) * (size_t)(2 * nz + n));
	double *tu = (double *)malloc(sizeof(double) * (size_t)(2 * nz + n));
	if (!cnt || !tmpc || !tmpr || !tl || !tu) return -1;
	int m = 0;
	for (int i = 0; i < n; i++)
		for (int k = ia[i]; k < ia[i + 1]; k++) {
			int j = ja[k];
			if (j >= i) { tmpr[m] = i; tmpc[m] = j; tu[m] = a[k]; tl[m] = (j == i) ? a[k] : 0.0; m++; }
			if (j < i) { tmpr[m] = j; tmpc[m] = i; tl[m] = a[k]; tu[m] = 0.0; m++; }
		}
	/* bucket by row, then merge duplicates inside each row */
	for (int e = 0; e < m; e++) cnt[tmpr[e] + 1]++;
	for (int i = 0; i < n; i++) cnt[i + 1] += cnt[i];
	int *pos = (int *)malloc(sizeof(int) * (size_t)n);
	int *ord = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
	memcpy(pos, cnt, sizeof(int) * (size_t)n);
	for (int e = 0; e < m; e++) ord[pos[tmpr[e]]++] = e;
	int *ris = (int *)malloc(sizeof(int) * ((size_t)n + 1));
	int *rjs = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
	double *rl = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
	double *ru = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
	int out = 0;
	ris[0] = 0;
	for (int i = 0; i < n; i++) {
		int b = cnt[i], e = cnt[i + 1];
		/* insertion sort of this row's entries by column (diagonal is the minimum) */
		for (int s = b + 1; s < e; s++)
			for (int t = s; t > b && tmpc[ord[t - 1]] > tmpc[ord[t]]; t--) { int w = ord[t]; ord[t] = ord[t - 1]; ord[t - 1] = w; }
		for (int s = b; s < e; s++) {
			int k = ord[s];
			if (out > ris[i] && rjs[out - 1] == tmpc[k]) {
				rl[out - 1] += tl[k];
				ru[out - 1] += tu[k];
			} else {
				rjs[out] = tmpc[k]; rl[out] = tl[k]; ru[out] = tu[k]; out++;
			}
		}
		ris[i + 1] = out;
		if (ris[i + 1] == ris[i] || rjs[ris[i]] != i) { /* structurally missing diagonal */
			free(cnt); free(tmpc); free(tmpr); free(tl); free(tu); free(pos); free(ord);
			free(ris); free(rjs); free(rl); free(ru);
			return -1;
		}
	}
	free(cnt); free(tmpc); free(tmpr); free(tl); free(tu); free(pos); free(ord);
	*ia_s = ris; *ja_s = rjs; *al = rl; *au = ru;
	return out;
}

/* Optional dependency-depth outputs of orc_fact (see orc_fact_levels). */
static int *g_lev_fact, *g_lev_solve, *g_dropdep, *g_nmember, *g_nmask;

/* Theta compensations received by a row are summed in 64-bit fixed point
 * (value * 2^bits, truncated per term): integer addition makes the sum
 * independent of the order of the terms, which is what lets the GPU collect
 * them from rows that finish in any order.  A compensation is below
 * tau2 * theta < 2^e (frexp), and bits = 51 - e leaves room for 2^12 maximal
 * terms in 63 bits. */
static double g_acc_scale = 0x1p64, g_acc_inv = 0x1p-64;
static void acc_setup(double tau2, double theta) {
	int e = -13;
	double maxterm = tau2 * theta;
	if (maxterm > 0.0) frexp(maxterm, &e);
	int bits = 51 - e;
	if (bits > 1000) bits = 1000;
	g_acc_scale = ldexp(1.0, bits);
	g_acc_inv = ldexp(1.0, -bits);
}
static void acc_push(unsigned long long *acc, int j, double comp) {
	acc[j] += (unsigned long long)(comp * g_acc_scale);
}
static double acc_value(const unsigned long long *acc, int j) { return (double)acc[j] * g_acc_inv; }

/* Growable arrays for the stored rows of the working factor. */
typedef struct { int *col; signed char *flag; double *gl, *gu; size_t len, cap; } pool_t;

static int pool_reserve(pool_t *p, size_t need) {
	if (p->len + need <= p->cap) return 0;
	size_t nc = p->cap ? p->cap : 1024;
	while (nc < p->len + need) nc *= 2;
	int *c = (int *)realloc(p->col, nc * sizeof(int));
	if (!c) return -1;
	p->col = c;
	signed char *f = (signed char *)realloc(p->flag, nc);
	if (!f) return -1;
	p->flag = f;
	double *l = (double *)realloc(p->gl, nc * sizeof(double));
	if (!l) return -1;
	p->gl = l;
	double *u = (double *)realloc(p->gu, nc * sizeof(double));
	if (!u) return -1;
	p->gu = u;
	p->cap = nc;
	return 0;
}

/* IC2 / ILU2 restated from Bslib/ich2r.cpp:956-1195 (IC2 main loop), helpers
 * :60-420 and :756-955, and Bslib/ilu2r.cpp:1122-1395 (ILU2 main loop),
 * helpers :28-350 and :758-803.
 *
 * Per row i: init the scaled row (Ich2InitRow :161 / Ilu2InitRow), apply
 * updates from every earlier row k whose stored part contains column i
 * (R x R products skipped, Ich2InitMask :202-222), filter by tau2 with theta
 * compensation of both diagonals (Ich2FiltrRow :316 / Ilu2FiltrRow), pivot
 * and scale (Ich2PivScaleRow :348 / Ilu2PivScaleRow), split kept entries into
 * U (>= tau1) and R (Ich2StoreRow :756), and at the end unscale the U part
 * (Ich2StoreScaleU :910).
 *
 * Deliberate, documented difference: the reference applies the updates of
 * row i in the order of its transposed linked lists (ibegm/madj) and adds the
 * compensations of the rows that dropped column i as they come; this
 * restatement applies the updates in ascending order of the updating row,
 * then adds the received compensations (an exact fixed-point sum), then the
 * row's own theta compensations in ascending column order.  Products are
 * accumulated with fma().  The GPU kernel uses exactly this order, so its
 * factor can be compared bit for bit; against the reference the entries
 * agree to rounding (checked in tests/test_oracle_pin.py). */
int orc_fact(int kind, int n, const int *ia, const int *ja, const double *al, const double *au, double tau1,
             double tau2, double theta, double sclmin, double pivmin, int **iu_out, int **ju_out, double **lval_out,
             double **uval_out, double *stats) {
	const int ilu = (kind == 1);
	if (!ilu) au = al;
	double *scll = (double *)malloc(sizeof(double) * (size_t)n);
	double *sclu = (double *)malloc(sizeof(double) * (size_t)n);
	double *diagg = (double *)malloc(sizeof(double) * (size_t)n);
	double *fl = (double *)calloc((size_t)n, sizeof(double));
	double *fu = (double *)calloc((size_t)n, sizeof(double));
	int *imask = (int *)malloc(sizeof(int) * (size_t)n);
	int *lst = (int *)malloc(sizeof(int) * (size_t)n);
	int *keep = (int *)malloc(sizeof(int) * (size_t)n);
	int *rowbeg = (int *)malloc(sizeof(int) * ((size_t)n + 1));
	/* transposed lists: rows whose next stored column is c (ascending not required: sorted per use) */
	int *ibegm = (int *)malloc(sizeof(int) * (size_t)n);
	int *madj = (int *)malloc(sizeof(int) * (size_t)n);
	int *iv = (int *)malloc(sizeof(int) * (size_t)n);
	int *contrib = (int *)malloc(sizeof(int) * (size_t)n);
	unsigned long long *acc = (unsigned long long *)calloc((size_t)n, sizeof(unsigned long long));
	acc_setup(tau2, theta);
	pool_t P = {0};
	int rc = 0;
	if (!scll || !sclu || !diagg || !fl || !fu || !imask || !lst || !keep || !rowbeg || !ibegm || !madj || !iv ||
	    !contrib || !acc) { rc = -1; goto done; }

	for (int i = 0; i < n; i++) {
		double d = al[ia[i]];
		if (!ilu) {
			double s = sqrt(d); /* Ich2AllocScale, Bslib/ich2r.cpp:75-85 */
			scll[i] = sclu[i] = 1.0 / s;
			diagg[i] = d * scll[i] * scll[i];
		} else {
			double m = fabs(d); /* Ilu2AllocScale, Bslib/ilu2r.cpp:45-62 */
			if (m < sclmin) m = sclmin;
			m = 1.0 / sqrt(m);
			scll[i] = m;
			sclu[i] = (d < 0.0) ? m : -m;
			diagg[i] = d * scll[i] * sclu[i];
		}
		imask[i] = -1; ibegm[i] = -1; madj[i] = -1; iv[i] = -1;
	}
	size_t nzu = 0, nzr = 0;
	rowbeg[0] = 0;
	for (int i = 0; i < n; i++) {
		int nl = 0;
		/* init (Ich2InitRow / Ilu2InitRow) */
		lst[nl++] = i; imask[i] = i;
		fl[i] = diagg[i];
		fu[i] = fl[i];
		for (int k = ia[i] + 1; k < ia[i + 1]; k++) {
			int j = ja[k];
			lst[nl++] = j; imask[j] = i;
			fl[j] = al[k] * sclu[i] * scll[j];
			fu[j] = au[k] * scll[i] * sclu[j];
			if (!ilu) fl[j] = fu[j] = al[k] * scll[i] * scll[j];
		}
		/* contributors: rows on the transposed list of column i, ascending */
		int nc = 0;
		for (int r = ibegm[i]; r != -1; r = madj[r]) contrib[nc++] = r;
		qsort(contrib, (size_t)nc, sizeof(int), cmp_int);
		if (g_lev_fact) {
			/* dependency depth: 1 + deepest row that updated or compensated i */
			int lf = g_dropdep ? g_dropdep[i] : 0, ls = 0;
			for (int t = 0; t < nc; t++) {
				int k = contrib[t];
				if (g_lev_fact[k] + 1 > lf) lf = g_lev_fact[k] + 1;
				if (P.flag[iv[k]] == 0 && g_lev_solve[k] + 1 > ls) ls = g_lev_solve[k] + 1;
			}
			g_lev_fact[i] = lf;
			g_lev_solve[i] = ls;
			if (g_nmember) g_nmember[i] += nc; /* plus the droppers counted in the filter */
		}
		for (int t = 0; t < nc; t++) {
			int k = contrib[t];
			size_t e0 = (size_t)iv[k];
			double lel = P.gl[e0], uel = P.gu[e0];
			int isr = P.flag[e0] == 1;
			for (size_t e = e0; e < (size_t)rowbeg[k + 1]; e++) {
				if (isr && P.flag[e] == 1) continue;
				int c = P.col[e];
				if (imask[c] != i) { imask[c] = i; lst[nl++] = c; fl[c] = 0.0; fu[c] = 0.0; }
				if (ilu) {
					fl[c] = fma(-uel, P.gl[e], fl[c]);
					fu[c] = fma(-lel, P.gu[e], fu[c]);
				} else {
					fl[c] = fma(-lel, P.gl[e], fl[c]);
				}
			}
		}
		/* advance the contributors to their next stored column (Ich2UpdateTransp :296) */
		{
			int r = ibegm[i];
			while (r != -1) {
				int nxt = madj[r];
				if (iv[r] + 1 >= rowbeg[r + 1]) {
					madj[r] = -1;
				} else {
					int c = P.col[iv[r] + 1];
					madj[r] = ibegm[c];
					ibegm[c] = r;
				}
				iv[r]++;
				r = nxt;
			}
		}
		/* the theta compensations received from the rows that dropped column
		 * i, summed exactly (fixed point), join the diagonal after the updates */
		{
			const double cv = acc_value(acc, i);
			fl[i] = fl[i] + cv;
			fu[i] = fu[i] + cv;
		}
		if (!ilu) for (int s = 0; s < nl; s++) fu[lst[s]] = fl[lst[s]];
		/* filter in ascending column order (Ich2FiltrRow / Ilu2FiltrRow) */
		qsort(lst + 1, (size_t)(nl - 1), sizeof(int), cmp_int);
		if (g_nmask) g_nmask[i] = nl - 1;
		int nk = 0;
		for (int s = 1; s < nl; s++) {
			int j = lst[s];
			double v = fabs(fl[j]);
			if (ilu && fabs(fu[j]) > v) v = fabs(fu[j]);
			if (v >= tau2) {
				keep[nk++] = j;
			} else {
				v *= theta;
				fl[i] += v;
				fu[i] += v;
				acc_push(acc, j, v);
				if (g_dropdep && g_lev_fact[i] + 1 > g_dropdep[j]) g_dropdep[j] = g_lev_fact[i] + 1;
				if (g_nmember) g_nmember[j]++;
			}
		}
		/* pivot and scale */
		double dl, du;
		if (!ilu) {
			double d = fl[i];
			if (!(d > 0.0)) {
				if (stats) stats[2] = i;
				rc = -2;
				goto done;
			}
			d = sqrt(d);
			dl = du = 1.0 / d;
			for (int s = 0; s < nk; s++) { fl[keep[s]] *= dl; }
		} else {
			double d = fl[i];
			double m = fabs(d);
			if (m < pivmin) m = pivmin;
			m = sqrt(m);
			dl = 1.0 / m;
			du = (d < 0.0) ? -dl : dl;
			for (int s = 0; s < nk; s++) { fl[keep[s]] *= du; fu[keep[s]] *= dl; }
		}
		/* store: diagonal, then kept entries ascending, flagged U (0) or R (1) */
		if (pool_reserve(&P, (size_t)nk + 1)) { rc = -1; goto done; }
		size_t b = P.len;
		P.col[b] = i; P.flag[b] = 0; P.gl[b] = dl; P.gu[b] = du;
		P.len++;
		nzu++;
		for (int s = 0; s < nk; s++) {
			int j = keep[s];
			double v = fabs(fl[j]);
			double lv = fl[j], uv = ilu ? fu[j] : fl[j];
			if (ilu && fabs(fu[j]) > v) v = fabs(fu[j]);
			P.col[P.len] = j;
			P.flag[P.len] = (v >= tau1) ? 0 : 1;
			P.gl[P.len] = lv; P.gu[P.len] = uv;
			if (v >= tau1) nzu++; else nzr++;
			P.len++;
		}
		rowbeg[i + 1] = (int)P.len;
		if (nk > 0) {
			iv[i] = (int)b + 1;
			madj[i] = ibegm[keep[0]];
			ibegm[keep[0]] = i;
		}
	}
	/* Ich2StoreScaleU (Bslib/ich2r.cpp:910-954): keep U, undo the scaling */
	{
		int *iu = (int *)malloc(sizeof(int) * ((size_t)n + 1));
		int *ju = (int *)malloc(sizeof(int) * (nzu > 0 ? nzu : 1));
		double *lv = (double *)malloc(sizeof(double) * (nzu > 0 ? nzu : 1));
		double *uv = ilu ? (double *)malloc(sizeof(double) * (nzu > 0 ? nzu : 1)) : lv;
		if (!iu || !ju || !lv || !uv) { rc = -1; goto done; }
		size_t z = 0;
		iu[0] = 0;
		for (int i = 0; i < n; i++) {
			for (int e = rowbeg[i]; e < rowbeg[i + 1]; e++) {
				if (P.flag[e] != 0) continue;
				int j = P.col[e];
				ju[z] = j;
				if (j == i) {
					lv[z] = P.gl[e] * scll[i];
					if (ilu) uv[z] = P.gu[e] * sclu[i];
				} else {
					lv[z] = P.gl[e] / scll[j];
					if (ilu) uv[z] = P.gu[e] / sclu[j];
				}
				z++;
			}
			iu[i + 1] = (int)z;
		}
		*iu_out = iu; *ju_out = ju; *lval_out = lv; *uval_out = uv;
		if (stats) {
			stats[0] = (double)nzu / (double)ia[n];
			stats[1] = (double)nzr / (double)ia[n];
		}
	}
done:
	free(scll); free(sclu); free(diagg); free(fl); free(fu); free(imask); free(lst); free(keep); free(rowbeg);
	free(ibegm); free(madj); free(iv); free(contrib); free(acc);
	free(P.col); free(P.flag); free(P.gl); free(P.gu);
	return rc;
}

static double dot(int n, const double *x, const double *y) {
	double s = 0.0;
	for (int i = 0; i < n; i++) s += x[i] * y[i];
	return s;
}

/* PCG restated from Bslib/cg.cpp:31-350 (CSVector::Cg, matrix form):
 * residual from x0 = 0, per iteration SolveL+SolveU (:142-143), the dots
 * (:153-155), stop test on the recursive residual (:239-241), p = beta p + z
 * (:247-248), MvmASymm (:259), alpha = gamma/(p.Ap) with the non-SPD exit
 * (:266-278), and the two updates (:284-285).  Returns the solution that
 * corresponds to the last tested residual, as the reference does. */
int orc_pcg(int n, const int *ia, const int *ja, const double *a, const int *iu, const int *ju, const double *u,
            const double *b, double *x, int ittype, double eps, int niter, double *resfin) {
	double *r = (double *)malloc(sizeof(double) * (size_t)n), *p = (double *)calloc((size_t)n, sizeof(double));
	double *q = (double *)malloc(sizeof(double) * (size_t)n), *z = (double *)malloc(sizeof(double) * (size_t)n);
	double *sol = (double *)calloc((size_t)n, sizeof(double));
	double gamma0 = 0, enrsq0 = 0, enrsq = 0, gamold = 0, alpha = 1, beta = 0;
	int k, nit = 0;
	orc_mvm_symm(n, ia, ja, a, sol, r);
	for (int i = 0; i < n; i++) r[i] = b[i] - r[i];
	for (k = 1; k < niter; k++) {
		orc_solve_l(n, iu, ju, u, r, q);
		orc_solve_u(n, iu, ju, u, q, z);
		enrsq = dot(n, r, r);
		double gamma = dot(n, r, z);
		if (k == 1) { gamma0 = gamma; enrsq0 = enrsq; }
		memcpy(x, sol, sizeof(double) * (size_t)n);
		nit = k;
		if (ittype == 0 && enrsq <= eps * eps * enrsq0) break;
		if (ittype == 1 && enrsq <= eps * eps) break;
		if (k > 1) beta = gamma / gamold;
		for (int i = 0; i < n; i++) p[i] = beta * p[i] + z[i];
		orc_mvm_symm(n, ia, ja, a, p, z);
		alpha = gamma / dot(n, p, z);
		if (alpha < 0.0) break;
		gamold = gamma;
		for (int i = 0; i < n; i++) { r[i] -= alpha * z[i]; sol[i] += alpha * p[i]; }
	}
	if (k >= niter) memcpy(x, sol, sizeof(double) * (size_t)n);
	if (resfin) *resfin = enrsq0 > 0 ? sqrt(enrsq / enrsq0) : 0.0;
	(void)gamma0;
	free(r); free(p); free(q); free(z); free(sol);
	return nit;
}

/* Right-preconditioned GMRES(m).  The reference's real GMRES
 * (Bslib/gmres.cpp:337) is an unrestarted block-Householder method; this is
 * the restarted FP64 modified-Gram-Schmidt form the GPU solver implements,
 * with the Givens recurrence of Bslib/gmres.cpp:30-101 for one right-hand
 * side and the triangular solve of :140.  Returns the total iterations. */
int orc_gmres(int n, const int *ia, const int *ja, const double *a, const int *iu, const int *ju, const double *l,
              const double *u, const double *b, double *x, int m, double eps, int sttype, int niter,
              double *resfin) {
	double *V = (double *)malloc(sizeof(double) * (size_t)n * (m + 1));
	double *Z = (double *)malloc(sizeof(double) * (size_t)n * m);
	double *H = (double *)calloc((size_t)(m + 1) * m, sizeof(double));
	double *cs = (double *)malloc(sizeof(double) * m), *sn = (double *)malloc(sizeof(double) * m);
	double *g = (double *)malloc(sizeof(double) * (m + 1)), *y = (double *)malloc(sizeof(double) * m);
	double *w = (double *)malloc(sizeof(double) * n), *t = (double *)malloc(sizeof(double) * n);
	int it = 0;
	double bnorm = sqrt(dot(n, b, b));
	double target = (sttype == 0) ? eps : eps * bnorm;
	double beta = 0;
	for (int i = 0; i < n; i++) x[i] = 0.0;
	while (it < niter) {
		orc_mvm(n, ia, ja, a, x, w);
		for (int i = 0; i < n; i++) V[i] = b[i] - w[i];
		beta = sqrt(dot(n, V, V));
		if (beta <= target) break;
		for (int i = 0; i < n; i++) V[i] /= beta;
		for (int i = 0; i <= m; i++) g[i] = 0.0;
		g[0] = beta;
		int j;
		for (j = 0; j < m && it < niter; j++, it++) {
			double *vj = V + (size_t)j * n, *zj = Z + (size_t)j * n, *vn = V + (size_t)(j + 1) * n;
			orc_solve_l(n, iu, ju, l, vj, t);
			orc_solve_u(n, iu, ju, u, t, zj);
			orc_mvm(n, ia, ja, a, zj, vn);
			for (int k = 0; k <= j; k++) {
				double h = dot(n, vn, V + (size_t)k * n);
				H[k * m + j] = h;
				for (int i = 0; i < n; i++) vn[i] -= h * V[(size_t)k * n + i];
			}
			double hn = sqrt(dot(n, vn, vn));
			H[(j + 1) * m + j] = hn;
			if (hn > 0) for (int i = 0; i < n; i++) vn[i] /= hn;
			for (int k = 0; k < j; k++) {
				double h0 = H[k * m + j], h1 = H[(k + 1) * m + j];
				H[k * m + j] = cs[k] * h0 + sn[k] * h1;
				H[(k + 1) * m + j] = -sn[k] * h0 + cs[k] * h1;
			}
			double h0 = H[j * m + j], h1 = H[(j + 1) * m + j];
			double rr = sqrt(h0 * h0 + h1 * h1);
			cs[j] = (rr > 0) ? h0 / rr : 1.0;
			sn[j] = (rr > 0) ? h1 / rr : 0.0;
			H[j * m + j] = rr;
			H[(j + 1) * m + j] = 0.0;
			g[j + 1] = -sn[j] * g[j];
			g[j] = cs[j] * g[j];
			if (fabs(g[j + 1]) <= target) { j++; it++; break; }
		}
		for (int k = j - 1; k >= 0; k--) {
			double s = g[k];
			for (int q = k + 1; q < j; q++) s -= H[k * m + q] * y[q];
			y[k] = s / H[k * m + k];
		}
		for (int k = 0; k < j; k++)
			for (int i = 0; i < n; i++) x[i] += y[k] * Z[(size_t)k * n + i];
		if (fabs(g[j]) <= target) {
			orc_mvm(n, ia, ja, a, x, w);
			for (int i = 0; i < n; i++) w[i] = b[i] - w[i];
			beta = sqrt(dot(n, w, w));
			if (beta <= target) break;
		}
	}
	if (resfin) *resfin = bnorm > 0 ? beta / bnorm : 0.0;
	free(V); free(Z); free(H); free(cs); free(sn); free(g); free(y); free(w); free(t);
	return it;
}

/* orc_fact plus, per row, the depth of the row in the factorisation's
 * dependency graph (lev_fact: longest chain of updating / compensating rows)
 * and in the forward-solve graph (lev_solve: longest chain through U
 * entries), and optionally the size of C(i) (rows that update or
 * compensate row i) and of row i's mask before filtering.  Used to size and
 * check the GPU schedule. */
int orc_fact_levels(int kind, int n, const int *ia, const int *ja, const double *al, const double *au, double tau1,
                    double tau2, double theta, double sclmin, double pivmin, int *lev_fact, int *lev_solve,
                    int *nmember, int *nmask) {
	int *iu, *ju;
	double *lv, *uv;
	g_lev_fact = lev_fact;
	g_lev_solve = lev_solve;
	g_nmember = nmember;
	g_nmask = nmask;
	if (nmember) memset(nmember, 0, sizeof(int) * (size_t)n);
	g_dropdep = (int *)calloc((size_t)n, sizeof(int));
	int rc = orc_fact(kind, n, ia, ja, al, au, tau1, tau2, theta, sclmin, pivmin, &iu, &ju, &lv, &uv, NULL);
	free(g_dropdep);
	g_lev_fact = g_lev_solve = g_dropdep = g_nmember = g_nmask = NULL;
	if (rc == 0) {
		free(iu); free(ju); free(lv);
		if (uv != lv) free(uv);
	}
	return rc;
}

/* y = A^T x (the gather-free transpose product of CSMatrixR::MvmAt). */
void orc_mvm_t(int n, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	for (int i = 0; i < n; i++) y[i] = 0.0;
	for (int i = 0; i < n; i++)
		for (int j = ia[i]; j < ia[i + 1]; j++) y[ja[j]] += a[j] * x[i];
}

/* Preconditioned two-sided Lanczos of CSVector::Lanczos (Bslib/lanczos.cpp:34-370)
 * with the factor in the reference layout (l, u on the pattern iu, ju: L by
 * columns, U by rows, inverse pivots first) and the weight vector of the
 * max-norm error equal to one.  Per iteration: delta-products with A and
 * M^{-1} = U^{-1} L^{-1}, the scalars gamma / ro (:148-159), the three-term
 * updates of the solution (:163-182) and of delta (:250-262), the true
 * residual and its max-norm (:187-205), and the transposed products
 * L^{-T} U^{-T} (SolveL on U, SolveU on L, :266-270) and A^T (:274).  The
 * returned solution is the iterate of least max-norm residual, as in the
 * reference (:210-214, :364-368).  Returns the iteration count; *errmin gets
 * the least max-norm residual. */
int orc_lanczos(int n, const int *ia, const int *ja, const double *a, const int *iu, const int *ju, const double *l,
                const double *u, const double *b, double *x, double eps, int sttype, int niter, double *errmin_out) {
	double *sol = (double *)calloc((size_t)n, sizeof(double)), *r = (double *)malloc(sizeof(double) * n);
	double *good = (double *)malloc(sizeof(double) * n), *sol1 = (double *)calloc((size_t)n, sizeof(double));
	double *D = (double *)malloc(sizeof(double) * n), *D1 = (double *)calloc((size_t)n, sizeof(double));
	double *d = (double *)malloc(sizeof(double) * n), *d1 = (double *)calloc((size_t)n, sizeof(double));
	double *img = (double *)malloc(sizeof(double) * n), *p = (double *)malloc(sizeof(double) * n);
	for (int i = 0; i < n; i++) sol[i] = x[i];
	orc_mvm(n, ia, ja, a, sol, r);
	for (int i = 0; i < n; i++) r[i] = b[i] - r[i];
	double errmin = 0.0, resini = 0.0;
	for (int i = 0; i < n; i++) {
		errmin = fabs(r[i]) > errmin ? fabs(r[i]) : errmin;
		resini += r[i] * r[i];
	}
	resini = sqrt(resini);
	for (int i = 0; i < n; i++) { good[i] = sol[i]; D[i] = r[i]; }
	orc_solve_l(n, iu, ju, l, r, p);
	orc_solve_u(n, iu, ju, u, p, d);
	double gamma = 0.0, gamma1, ro = 1.0, delDel = 0.0, delDel1, resi = resini;
	int k;
	for (k = 1; k < niter; k++) {
		orc_mvm(n, ia, ja, a, d, r);
		orc_solve_l(n, iu, ju, l, r, p);
		orc_solve_u(n, iu, ju, u, p, img);
		gamma1 = gamma;
		delDel1 = delDel;
		delDel = 0.0;
		double dtemp = 0.0;
		for (int i = 0; i < n; i++) delDel += d[i] * D[i];
		for (int i = 0; i < n; i++) dtemp += img[i] * D[i];
		gamma = delDel / dtemp;
		if (k > 1) ro = 1.0 / (1.0 - (gamma / gamma1) * (delDel / delDel1) / ro);
		const double rogamma = ro * gamma, unitro = 1.0 - ro;
		for (int i = 0; i < n; i++) {
			const double t = sol[i];
			sol[i] = (t * ro + sol1[i] * unitro) + d[i] * rogamma;
			sol1[i] = t;
		}
		orc_mvm(n, ia, ja, a, sol, r);
		double errloc = 0.0;
		resi = 0.0;
		for (int i = 0; i < n; i++) {
			r[i] = b[i] - r[i];
			errloc = fabs(r[i]) > errloc ? fabs(r[i]) : errloc;
			resi += r[i] * r[i];
		}
		resi = sqrt(resi);
		if (errloc < errmin) {
			for (int i = 0; i < n; i++) good[i] = sol[i];
			errmin = errloc;
		}
		const int brk = fabs(delDel) < 1.e-100 && fabs(delDel1) < 1.e-100;
		if ((sttype == 2 && errmin <= eps) || (sttype == 0 && resi <= eps) || (sttype == 1 && resi <= eps * resini) ||
		    brk)
			break;
		for (int i = 0; i < n; i++) {
			const double t = d[i];
			d[i] = (t * ro + d1[i] * unitro) - img[i] * rogamma;
			d1[i] = t;
		}
		orc_solve_l(n, iu, ju, u, D, p);   /* U^T, U's storage read as L by columns */
		orc_solve_u(n, iu, ju, l, p, r);   /* L^T, L's storage read as U by rows */
		orc_mvm_t(n, ia, ja, a, r, img);
		for (int i = 0; i < n; i++) {
			const double t = D[i];
			D[i] = (t * ro + D1[i] * unitro) - img[i] * rogamma;
			D1[i] = t;
		}
	}
	for (int i = 0; i < n; i++) x[i] = good[i];
	if (errmin_out) *errmin_out = errmin;
	free(sol); free(r); free(good); free(sol1); free(D); free(D1); free(d); free(d1); free(img); free(p);
	return k;
}

/* IC(0) on A's pattern: CSMatrixR::Ich (Bslib/ich2r.cpp:1821-1895).  The
 * reference transposes the upper-stored A (rows of A^T: columns ascending,
 * the diagonal last), computes for every row i and each off-diagonal column
 * k, ascending,
 *     l_ik = (a_ik - sum_m l_km l_im) * d_k      (merge over m < k)
 * then the pivot a_ii - sum_k l_ik^2, clamped below at 1e-20, d_i = 1/sqrt,
 * and transposes back.  Every term is a product then a subtraction (no fused
 * multiply-add).  Output: U by rows on A's upper pattern (iu/ju copies of
 * ia/ja), d_i in the diagonal slot, u(k,i) = l_ik.  Returns 0, or -1 for bad
 * input (a row that does not start with its diagonal). */
int orc_ich0(int n, const int *ia, const int *ja, const double *a, int **iu_out, int **ju_out, double **u_out) {
	const int nz = ia[n];
	/* rows of A^T: strict lower columns ascending, positions in the upper arrays */
	int *tcnt = (int *)calloc((size_t)n + 1, sizeof(int));
	int *tja = (int *)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
	int *tpos = (int *)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
	double *lv = (double *)malloc(sizeof(double) * (size_t)(nz > 0 ? nz : 1));
	double *dinv = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
	int *iu = (int *)malloc(sizeof(int) * (size_t)(n + 1));
	int *ju = (int *)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
	double *u = (double *)malloc(sizeof(double) * (size_t)(nz > 0 ? nz : 1));
	int rc = 0;
	if (!tcnt || !tja || !tpos || !lv || !dinv || !iu || !ju || !u) { rc = -1; goto done; }
	for (int i = 0; i < n; i++) {
		if (ia[i + 1] <= ia[i] || ja[ia[i]] != i) { rc = -1; goto done; }
		for (int k = ia[i] + 1; k < ia[i + 1]; k++) tcnt[ja[k] + 1]++;
	}
	for (int i = 0; i < n; i++) tcnt[i + 1] += tcnt[i];
	{
		int *fill = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
		if (!fill) { rc = -1; goto done; }
		for (int i = 0; i < n; i++) fill[i] = tcnt[i];
		/* rows of A visited in ascending order: each column list comes out ascending */
		for (int k = 0; k < n; k++)
			for (int p = ia[k] + 1; p < ia[k + 1]; p++) {
				const int i = ja[p];
				tja[fill[i]] = k;
				tpos[fill[i]] = p;
				fill[i]++;
			}
		free(fill);
	}
	for (int i = 0; i < n; i++) {
		const int i1 = tcnt[i], i2 = tcnt[i + 1];
		for (int j = i1; j < i2; j++) {
			const int k = tja[j];
			double r = a[tpos[j]];
			int ik = tcnt[k], ik2 = tcnt[k + 1], q = i1;
			while (ik < ik2 && q < j) {
				if (tja[ik] < tja[q]) {
					ik++;
				} else if (tja[ik] > tja[q]) {
					q++;
				} else {
					const double pr = lv[ik] * lv[q];
					r = r - pr;
					q++;
					ik++;
				}
			}
			lv[j] = r * dinv[k];
		}
		double r = a[ia[i]];
		for (int j = i1; j < i2; j++) {
			const double pr = lv[j] * lv[j];
			r = r - pr;
		}
		if (r < 1.0e-20) r = 1.0e-20;
		dinv[i] = 1.0 / sqrt(r);
	}
	for (int i = 0; i <= n; i++) iu[i] = ia[i];
	for (int p = 0; p < nz; p++) ju[p] = ja[p];
	for (int i = 0; i < n; i++) u[ia[i]] = dinv[i];
	for (int i = 0; i < n; i++)
		for (int j = tcnt[i]; j < tcnt[i + 1]; j++) u[tpos[j]] = lv[j];
	*iu_out = iu;
	*ju_out = ju;
	*u_out = u;
	iu = NULL;
	ju = NULL;
	u = NULL;
done:
	free(tcnt); free(tja); free(tpos); free(lv); free(dinv); free(iu); free(ju); free(u);
	return rc;
}
