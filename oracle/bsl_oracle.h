/* CPU oracle for the Bslib Krylov hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithms (file:line citations at
 * each function in bsl_oracle.c).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it, and only as the checker; the
 * product library never links or calls it.
 *
 * Pinning: every routine here is checked against the reference Bslib itself,
 * compiled from its sources into oracle/_ref/libbslib_ref.so by
 * oracle/Makefile (tests/test_oracle_pin.py).  The reference ships no golden
 * vectors, so the pinned outputs are committed under tests/golden/.
 *
 * Conventions: 0-based CSR, each row's diagonal first.  Factor "a" arrays
 * hold the inverse pivot in the diagonal slot, as the reference does.
 */
#ifndef BSL_ORACLE_H
#define BSL_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

void orc_mvm(int n, const int *ia, const int *ja, const double *a, const double *x, double *y);
void orc_mvm_symm(int n, const int *ia, const int *ja, const double *a, const double *x, double *y);
/* Block CSR, uniform block size bs, blocks column-major (CSMatrixRS). */
void orc_bsr_mvm(int nb, int bs, const int *ia, const int *ja, const double *a, const double *x, double *y);
void orc_solve_l(int n, const int *ia, const int *ja, const double *a, const double *x, double *y);
void orc_solve_u(int n, const int *ia, const int *ja, const double *a, const double *x, double *y);

/* Split a full CSR matrix into the shared upper pattern used by ILU2: row i
 * holds the columns j >= i of (pattern(A) U pattern(A)^T), diagonal first,
 * others ascending; al[] = A(j,i), au[] = A(i,j) (0 where absent).  Arrays are
 * malloc'ed; returns nnz or -1. */
int orc_combine_lu(int n, const int *ia, const int *ja, const double *a, int **ia_s, int **ja_s, double **al,
                   double **au);

/* Second-order threshold factorisation.  kind 0: IC2 (au ignored, uses al);
 * kind 1: ILU2.  On success returns 0 and malloc'ed factor arrays
 * (iu[n+1], ju, lval, uval; lval == uval for IC2).  stats[0] = density
 * (U nnz / A nnz), stats[1] = density2 (R nnz / A nnz).  Errors: -1 bad
 * input, -2 nonpositive IC2 pivot (row in stats[2]). */
int orc_fact(int kind, int n, const int *ia, const int *ja, const double *al, const double *au, double tau1,
             double tau2, double theta, double sclmin, double pivmin, int **iu, int **ju, double **lval,
             double **uval, double *stats);

/* IC(0) on A's pattern (CSMatrixR::Ich): upper-stored A in, U by rows on
 * the same pattern out (inverse pivots in the diagonal slots), malloc'ed. */
int orc_ich0(int n, const int *ia, const int *ja, const double *a, int **iu, int **ju, double **u);

/* Preconditioned CG with an upper-stored SPD matrix and an IC factor, the
 * reference's stopping rules (ittype 0: relative, 1: absolute on the
 * recursively updated residual).  Returns iterations; x holds the solution. */
int orc_pcg(int n, const int *ia, const int *ja, const double *a, const int *iu, const int *ju, const double *u,
            const double *b, double *x, int ittype, double eps, int niter, double *resfin);

/* Right-preconditioned restarted GMRES(m) with the factor pair (L by
 * columns, U by rows); FP64 modified Gram-Schmidt and Givens rotations.
 * Full-storage A.  Stops when the recursive residual estimate reaches
 * eps*||b|| (sttype 1) or eps (sttype 0).  Returns iterations. */
int orc_gmres(int n, const int *ia, const int *ja, const double *a, const int *iu, const int *ju, const double *l,
              const double *u, const double *b, double *x, int m, double eps, int sttype, int niter,
              double *resfin);

/* y = A^T x */
void orc_mvm_t(int n, const int *ia, const int *ja, const double *a, const double *x, double *y);
/* Preconditioned two-sided Lanczos (CSVector::Lanczos, Bslib/lanczos.cpp:34),
 * weight vector of the max-norm error = 1; returns the iterations, x gets
 * the iterate of least max-norm residual. */
int orc_lanczos(int n, const int *ia, const int *ja, const double *a, const int *iu, const int *ju, const double *l,
                const double *u, const double *b, double *x, double eps, int sttype, int niter, double *errmin);

void orc_free(void *p);

#ifdef __cplusplus
}
#endif

/* block (CSMatrixRS) part: bsl_oracle_block.c */
int orc_combine_lu_block(int nb, int bs, const int *ia, const int *ja, const double *a, int **ia_s, int **ja_s,
                         double **al, double **au);
int orc_ilu2_block(int nb, int bs, const int *is, const int *js, const double *al, const double *au, double tau1,
                   double tau2, double theta, double sclmin, double pivmin, int **ia_f, int **ja_f, double **l,
                   double **u, double *stats);
int orc_ilu2_block_jacobi(int nb, int bs, const int *is, const int *js, const double *al, const double *au,
                          double tau1, double tau2, double theta, double sclmin, double pivmin, int **ia_f, int **ja_f,
                          double **l, double **u, double *stats);
int orc_ich2_block(int nb, int bs, const int *ia, const int *ja, const double *a, double tau1, double tau2,
                   double theta, int **ia_f, int **ja_f, double **uo, double *stats);
int orc_ich2_block_jacobi(int nb, int bs, const int *ia, const int *ja, const double *a, double tau1, double tau2,
                          double theta, int **ia_f, int **ja_f, double **uo, double *stats);
void orc_solve_l_block(int nb, int bs, const int *ia, const int *ja, const double *a, const double *x, double *y);
void orc_solve_u_block(int nb, int bs, const int *ia, const int *ja, const double *a, const double *x, double *y);

#endif
