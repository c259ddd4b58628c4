/* bslib_gpu.h -- C ABI of the B200 (sm_100a) solver library libbsg.so.
 *
 * A drop-in replacement, on one GPU, for Bslib's preconditioned Krylov path:
 * point/block CSR SpMV, the second-order threshold IC2/ILU2 numeric
 * factorisation, the forward/backward triangular solves, and the PCG /
 * GMRES(m) / FGMRES(m) loops.  Matrices cross the boundary in the reference
 * storage (CSMatrixR: 0-based CSR, diagonal first in every row; CSMatrixRS:
 * block CSR with column-major blocks); solver settings in bsg_param, a plain-C
 * mirror of the CSlvParam fields the path reads and writes.
 *
 * Every function returns an int status: BSG_OK (0) or a negative BSG_ERR_*
 * code, mirroring the integer convention of the reference's C API
 * (Bslib/parfbss.cpp:37,74); bsg_last_error() gives the message, using the
 * reference's own exception strings where one exists.
 *
 * Threading: one context = one CUDA stream; a context and the objects made
 * from it are not thread-safe.  Separate contexts are independent.
 * Host pointers are borrowed for the duration of a call only.  Functions
 * named *_dev take device pointers and never copy between host and device.
 */
#ifndef BSLIB_GPU_H
#define BSLIB_GPU_H
#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
#define BSG_OK 0
#define BSG_ERR_ARG (-1)         /* invalid argument or malformed CSR/BSR       */
#define BSG_ERR_PIVOT (-2)       /* " Ich2: Diagonal pivot is nonpositive"       */
#define BSG_ERR_WORKSPACE (-3)   /* " Insufficient workspace in Ich2/Ilu2"       */
#define BSG_ERR_BREAKDOWN (-4)   /* Krylov breakdown (CG: matrix not SPD)       */
#define BSG_ERR_CUDA (-5)        /* CUDA runtime error                          */
#define BSG_ERR_TIMEOUT (-6)     /* a device spin-wait reached its time limit   */
#define BSG_ERR_NOCONV (-7)      /* iteration limit reached before tolerance    */
#define BSG_ERR_UNSUPPORTED (-8) /* option not implemented on the GPU path      */
#define BSG_ERR_NOMEM (-9)       /* device allocation failed                    */

/* ---- solver parameters ---------------------------------------------------- */
/* Fields up to `timeitr` carry the meaning of the CSlvParam member of the same
 * name (Bslib/slvparam.h:19-120, defaults :121-214).  The fields after it are
 * extensions of the GPU path that the reference does not have. */
typedef struct bsg_param {
	int msglev;       /* output level (0 quiet)                                   */
	int fcttyp;       /* bsg_fct_ich2 of a symmetric point matrix: 1 IC(0) on A's
	                     pattern (CSMatrixR::Ich), else the second-order IC2;
	                     block matrices and ILU2 always second order          */
	int ordtype;      /* ordering; only 0 (natural) is accepted on the GPU        */
	double memory;    /* factor workspace, multiples of nnz(A) (|memory| used)    */
	double tau1;      /* first-order threshold: |v| >= tau1 kept in U            */
	double tau2;      /* second-order threshold: tau2 <= |v| < tau1 kept in R    */
	double theta;     /* diagonal compensation factor for dropped entries        */
	double sclmin;    /* minimal scaling value (ILU2)                            */
	double pivmin;    /* minimal pivot (ILU2)                                    */
	int ittype;       /* CG stop rule on the recursive residual: 0 relative, 1
	                     absolute, 2 max |r_i| <= |eps| (Bslib/cg.cpp:239-241)    */
	int sttype;       /* GMRES / Lanczos stop rule: 0 absolute, 1 relative; 2 max-norm
	                     of the residual (Lanczos; GMRES: relative)                */
	int niter;        /* maximal number of iterations                            */
	double eps;       /* stopping tolerance                                      */
	int ichk;         /* iterations between convergence checks                   */
	/* outputs, as filled by the reference */
	int nitperf;      /* iterations performed                                    */
	double resfin;    /* final relative FP64 true residual ||b-Ax||/||b||        */
	double density;   /* nnz(U) / nnz(A)                                         */
	double density2;  /* nnz(R) / nnz(A)                                         */
	double timefct;   /* factorisation time, seconds (device events)            */
	double timeitr;   /* iteration time, seconds (device events)                */
	/* GPU-path extensions */
	int precision;    /* 0: FP64 factor values; 1: FP32 factor values, FP64 pivots */
	int trisolve;     /* 0: exact sync-free level solve; 1: Jacobi sweeps         */
	int nsweeps;      /* Jacobi sweeps per triangular solve when trisolve == 1   */
	int krylov;       /* 0: method of the driver (PCG symm / Lanczos nonsymm),
	                     1: GMRES(restart), 2: FGMRES(restart)                   */
	int restart;      /* GMRES/FGMRES restart length m                           */
	int true_residual;/* 1: recompute r = b - Ax in FP64 at every restart/stop   */
	void *learned;    /* optional learned preconditioner stage (bsg_unet*) for FGMRES */
	double resrec;    /* output: last recursive residual estimate (relative)     */
	int blockfct;     /* 3x3 block matrices: 1 (default) block factorisation with
	                     SVD / eigenvector-scaled diagonal blocks (CSMatrixRS::Ilu2
	                     / Ich2), 0 point factorisation of the point expansion */
	int pad[3];
} bsg_param;

/* CSlvParam's constructor defaults (Bslib/slvparam.h:121-214) plus the
 * GPU-path defaults (FP64, exact solves, restart 50). */
void bsg_param_default(bsg_param *p);

const char *bsg_last_error(void);
const char *bsg_version(void);

/* ---- context -------------------------------------------------------------- */
typedef struct bsg_ctx bsg_ctx;
typedef struct bsg_mat bsg_mat;
typedef struct bsg_fct bsg_fct;

/* Create a context on `device` that runs on the caller's cudaStream_t
 * (NULL: the device's default stream), or on a private non-blocking stream
 * when stream == BSG_OWN_STREAM. */
#define BSG_OWN_STREAM ((void *)-1)
int bsg_create(bsg_ctx **ctx, int device, void *stream);
int bsg_destroy(bsg_ctx *ctx);
int bsg_sync(bsg_ctx *ctx);
/* Time limit of every device spin-wait (the sync-free triangular solves, the
 * factorisation scheduler, the tensor-core pipeline of the learned stage), in
 * nanoseconds of GPU time: a wait that reaches it gives up, the call returns
 * BSG_ERR_TIMEOUT and the context stays usable.  Default 2 s; accepted range
 * 1 us .. 600 s.  It holds for the context's device, for every context on it,
 * from the next launch on; the call synchronises the context's stream first.
 * No counterpart in the reference (its loops have no waits). */
int bsg_set_spin_limit_ns(bsg_ctx *ctx, unsigned long long ns);

/* ---- matrices (CSMatrixR / CSMatrixRS, Bslib/smatrix.h:540-546, :1040-1048) */
/* Point CSR from host arrays.  symm_upper = 1: only the upper triangle is
 * given (the input of SolveSymm / MvmASymm, Bslib/mvm.cpp:2637); the device
 * copy is expanded to both triangles for gather SpMV. */
int bsg_mat_csr(bsg_ctx *ctx, int n, const int *ia, const int *ja, const double *a, int symm_upper,
                bsg_mat **out);
/* Same from device arrays (copied device-to-device). */
int bsg_mat_csr_dev(bsg_ctx *ctx, int n, const int *d_ia, const int *d_ja, const double *d_a, int symm_upper,
                    bsg_mat **out);
/* Block CSR with uniform block size bs >= 1, blocks column-major as in
 * CSMatrixRS (a[9*j + 3*c + r] for bs == 3).  bs == 3 keeps the 3x3 block
 * path (block SpMV, the block IC2 / ILU2 of CSMatrixRS); bs == 1 is point
 * CSR; any other size is expanded to point CSR on the host, and the point
 * factorisations then apply to it. */
int bsg_mat_bsr(bsg_ctx *ctx, int nsup, int bs, const int *ia, const int *ja, const double *a, int symm_upper,
                bsg_mat **out);
/* Block CSR with variable block sizes: the CSMatrixRS layout with
 * sprndr = sprndc = sprnd (Bslib/smatrix.h:1040-1048), as the reference's
 * AbstractSolver / AbstractSymmSolver assemble it (Bslib/solvers.cpp:
 * 5638-5736).  Block row i has sprnd[i+1] - sprnd[i] rows; its blocks follow
 * one another in `a`, each column-major, columns ascending in every block row
 * (symm_upper: upper blocks only, the diagonal block first).  All blocks 3x3:
 * the block path of bsg_mat_bsr; all 1x1: point CSR; otherwise the point
 * expansion (upper triangle of each diagonal block when symm_upper).
 * symm_upper | BSG_VBSR_POINT: the point expansion whatever the sizes. */
#define BSG_VBSR_POINT 2
int bsg_mat_vbsr(bsg_ctx *ctx, int nsup, const int *sprnd, const int *ia, const int *ja, const double *a,
                 int symm_upper, bsg_mat **out);
int bsg_mat_free(bsg_mat *m);
int bsg_mat_info(const bsg_mat *m, int *n, int *bs, int *nnz);

/* y = A x (CSMatrixR::MvmA Bslib/mvm.cpp:2489, MvmASymm :2637;
 * CSMatrixRS::MvmA :2530, MvmASymm :3008).  FP64. */
int bsg_mvm_dev(bsg_ctx *ctx, const bsg_mat *m, const double *d_x, double *d_y);
int bsg_mvm(bsg_ctx *ctx, const bsg_mat *m, const double *x, double *y); /* host buffers */
/* Y = A X for nrhs column vectors stored one after another (leading dim n*bs):
 * the matrix is read once for all right-hand sides (CSMatrixRS::MvmA loops
 * irhs outside the sweep, Bslib/mvm.cpp:2545). */
int bsg_mvm_multi_dev(bsg_ctx *ctx, const bsg_mat *m, int nrhs, const double *d_X, double *d_Y);

/* ---- factorisation (CSMatrixR::Ich2 Bslib/ich2r.cpp:956; CSMatrixR::Ilu2
 * Bslib/ilu2r.cpp:1122; CSMatrixRS::Ich2 Bslib/ich2rs.cpp:1075;
 * CSMatrixRS::Ilu2 Bslib/ilu2rs.cpp:1458) ---------------------------------- */
/* IC2 of a symmetric matrix (created with symm_upper = 1 or symmetric full). */
int bsg_fct_ich2(bsg_ctx *ctx, bsg_mat *m, bsg_param *p, bsg_fct **out);
/* ILU2 of a general matrix (the CombineLU split, Bslib/smatrixr.cpp:1142,
 * is done on the device). */
int bsg_fct_ilu2(bsg_ctx *ctx, bsg_mat *m, bsg_param *p, bsg_fct **out);
/* Convert the factor values to FP32 (pivots stay FP64) for the mixed path. */
int bsg_fct_to_fp32(bsg_fct *f);
/* Copy the factor to host in the reference layout: iu[n+1], ju[nnz],
 * l[nnz] (L by columns) and u[nnz] (U by rows), inverse pivots first.  Call
 * with NULL arrays to get nnz only. */
int bsg_fct_export(const bsg_fct *f, int *nnz, int *iu, int *ju, double *l, double *u);
/* The block factor of a block ILU2 / IC2 (CSMatrixRS layout,
 * Bslib/smatrix.h:1040; for IC2, l == u and L = U^T):
 * nb block rows, *nnzb blocks, ia[nb + 1], ja[nnzb], l / u [9 nnzb] column-
 * major 3x3 blocks, the pivot block first in each row (SolveL / SolveU apply
 * it as Bslib/mvm.cpp:3140 / 3410 do).  BSG_ERR_ARG for a point factor.
 * Any output pointer may be NULL (query *nnzb first). */
int bsg_fct_export_block(const bsg_fct *f, int *nb, int *nnzb, int *ia, int *ja, double *l, double *u);
int bsg_fct_info(const bsg_fct *f, int *n, int *nnz, int *levels_l, int *levels_u, double *density,
                 double *density2);
int bsg_fct_free(bsg_fct *f);

/* ---- triangular solves (CSMatrixR::SolveL Bslib/mvm.cpp:3042 / SolveU :3343;
 * CSMatrixRS::SolveL :3140 / SolveU :3410) -------------------------------- */
/* mode 0: exact (sync-free, dependency-ordered); mode 1: nsweeps Jacobi
 * sweeps (approximate, fully parallel).  `work` may be NULL for mode 0. */
int bsg_solve_l_dev(bsg_ctx *ctx, const bsg_fct *f, int mode, int nsweeps, const double *d_x, double *d_y);
int bsg_solve_u_dev(bsg_ctx *ctx, const bsg_fct *f, int mode, int nsweeps, const double *d_x, double *d_y);
/* nrhs solves with L (lower != 0) or U, vectors at stride n in d_x / d_y.
 * Sweeps (mode 1) read the factor once for up to 8 vectors, and every vector
 * gets the bits of its own bsg_solve_l_dev / bsg_solve_u_dev; exact solves
 * run one vector at a time.  The batched PCG applies its preconditioner to
 * all right-hand sides this way. */
int bsg_solve_multi_dev(bsg_ctx *ctx, const bsg_fct *f, int lower, int mode, int nsweeps, int nrhs,
                        const double *d_x, double *d_y);
/* Transposed solves: which 0 with U^T (SolveL applied to U's storage), 1 with
 * L^T (SolveU applied to L's storage) -- the transposed preconditioner of
 * Bslib/lanczos.cpp:266-270; same modes.  The transposed forms of an ILU2
 * factor are built on first use. */
int bsg_solve_t_dev(bsg_ctx *ctx, bsg_fct *f, int which, int mode, int nsweeps, const double *d_x, double *d_y);
/* Sweep-mode solve (lower != 0: L, else U) that allocates nothing: the same
 * kernels as bsg_solve_l_dev / bsg_solve_u_dev with mode 1, with the work
 * vector taken from a fixed 2^21-row device array instead of the memory
 * pool.  For callers that cannot allocate device memory while they iterate.
 * Factors above 2^21 rows are rejected (BSG_ERR_ARG).  The first call on a
 * device looks the array up and should come before any stream capture; the
 * array is shared per device, so calls must not overlap in time.  The
 * array's address is kept for the life of the process: after a device reset
 * (cudaDeviceReset) the entry point must not be used until the process
 * restarts.  Queued on the context stream without a host synchronisation.
 * No counterpart in the reference (its SolveL / SolveU need no work
 * vector). */
int bsg_solve_sweep_static(bsg_ctx *ctx, const bsg_fct *f, int lower, int nsweeps, const double *d_x, double *d_y);

/* ---- Krylov loops --------------------------------------------------------- */
/* PCG (CSVector::Cg, Bslib/cg.cpp:31) with A symmetric and an IC2 factor;
 * x0 = d_x on entry. */
int bsg_pcg_dev(bsg_ctx *ctx, const bsg_mat *m, const bsg_fct *f, const double *d_b, double *d_x, bsg_param *p);
/* Right-preconditioned GMRES(restart) / FGMRES(restart) (the restarted FP64
 * counterpart of CSVector::BlockGMRES, Bslib/gmres.cpp:337). */
int bsg_gmres_dev(bsg_ctx *ctx, const bsg_mat *m, const bsg_fct *f, const double *d_b, double *d_x,
                  bsg_param *p);

/* Preconditioned two-sided Lanczos (CSVector::Lanczos, Bslib/lanczos.cpp:34),
 * the reference's iteration for nonsymmetric systems: M^{-1} = U^{-1} L^{-1}
 * and its transpose, A and A^T, the iterate of least max-norm residual
 * returned (weights = 1); stopping per sttype (0: ||r|| <= eps, 1: ||r|| <=
 * eps ||r0||, 2: max |r_i| <= eps).  Point matrices; x0 = d_x on entry. */
int bsg_lanczos_dev(bsg_ctx *ctx, const bsg_mat *m, const bsg_fct *f, const double *d_b, double *d_x, bsg_param *p);

/* Block Lanczos of the CSMatrixRS driver (CSVector::BlockLanczosCentral /
 * BlockLanczosRight / BlockLanczosLeft, Bslib/lanczos.cpp:2467 / :932 /
 * :1719; CSVector::Solver(CSMatrixRS&) runs them for ittype 2 / 3 / 4,
 * Bslib/solvers.cpp:1798-1800): block Golub-Kahan bidiagonalisation of the
 * preconditioned matrix (central L^{-1} A U^{-1}, right A (LU)^{-1}, left
 * (LU)^{-1} A) with block Givens rotations, on nrhs <= 16 right-hand sides at
 * once.  Point matrices with a point factor.  d_B, d_X: [nrhs][n], d_X holds
 * x0.  Stops, tested every p->ichk steps as the reference tests, when every
 * right-hand side has ||b_j - A x_j|| < eps ||b_j - A x0_j|| (right variant:
 * or the preconditioned normal residual has fallen by eps).  res (host,
 * nrhs, may be NULL): final ||b_j - A x_j|| / ||b_j||; p->resfin their
 * maximum, p->nitperf the steps made. */
int bsg_block_lanczos_dev(bsg_ctx *ctx, const bsg_mat *m, const bsg_fct *f, int ittype, int nrhs, const double *d_B,
                          double *d_X, bsg_param *p, double *res);

/* Batched PCG (CSVector::Cg's recurrence, Bslib/cg.cpp:31-350, which handles
 * one right-hand side, :375-377): nrhs right-hand sides times nseg diagonal
 * blocks ("segments") of A that no entry couples -- e.g. the load cases of
 * one cell, or many independent problems assembled as one block-diagonal
 * matrix.  Each (right-hand side, segment) pair is its own system with its
 * own scalars and stopping test (ittype 0: ||r|| <= eps ||r0||), solved
 * together: one SpMM, one preconditioner pass per right-hand side and
 * segmented reductions per iteration.  The iteration loop is one CUDA graph
 * launched once: a conditional while node whose body runs 8 iterations and
 * decides on the device whether another pass is needed; the host reads the
 * result only when every system has stopped (and once more per
 * true-residual restart).  d_B, d_X: [nrhs][n] (n = point rows), d_X holds x0.  seg_off: host,
 * nseg + 1 point-row offsets (whole block rows; NULL when nseg == 1).
 * iters / res (host, nrhs * nseg, may be NULL): per-system iterations and
 * FP64 true relative residuals; p->nitperf / p->resfin get their maxima.
 * tuned (host, 4 ints, may be NULL): reduction chunk, SpMM group, iterations
 * per pass of the graph's loop body, passes made. */
int bsg_pcg_batch_dev(bsg_ctx *ctx, const bsg_mat *m, const bsg_fct *f, int nrhs, int nseg, const int *seg_off,
                      const double *d_B, double *d_X, bsg_param *p, int *iters, double *res, int *tuned);

/* ---- whole drivers with host buffers ------------------------------------- */
/* The iteration of CSVector::SolveSymm / Solver (Bslib/solvers.cpp:4452,
 * :4615, :1339, :1568) on a matrix and its factor, host buffers: x holds the
 * initial guess on entry (the drivers start from the vector itself) and the
 * solution on exit, also when the iteration limit stopped the loop
 * (BSG_ERR_NOCONV).  p->krylov 0: PCG (CSVector::Cg) for a symmetric matrix;
 * for a nonsymmetric one the iteration of CSVector::Solver(CSMatrixRS&):
 * p->ittype 2 / 3 / 4 the block Lanczos variants (bsg_block_lanczos_dev,
 * point matrices), otherwise the two-sided Lanczos (CSVector::Lanczos) for a
 * point matrix and GMRES(restart) for a 3x3 block matrix; krylov 1 / 2:
 * GMRES / FGMRES. */
int bsg_solve(bsg_ctx *ctx, const bsg_mat *m, const bsg_fct *f, const double *b, double *x, bsg_param *p);
/* The preconditioner with host buffers: which 0 applies SolveL then SolveU
 * (the CSOLVELU of Bslib/svector.h:40 that the callback Krylov loops call),
 * 1 SolveL only, 2 SolveU only (CSMatrixR::SolveL / SolveU,
 * Bslib/mvm.cpp:3042 / :3343); mode / nsweeps as bsg_solve_l_dev. */
int bsg_solve_lu(bsg_ctx *ctx, const bsg_fct *f, int which, int mode, int nsweeps, const double *x, double *y);
/* CSVector::SolveSymm(CSMatrixR&) (Bslib/solvers.cpp:4615): upper-stored SPD
 * CSR in, IC2 + PCG (or GMRES/FGMRES per p->krylov), solution out. */
int bsg_solve_symm_csr(bsg_ctx *ctx, int n, const int *ia, const int *ja, const double *a, const double *b,
                       double *x, bsg_param *p);
/* CSVector::Solver(CSMatrixR&) (Bslib/solvers.cpp:1339): full CSR in,
 * CombineLU + ILU2 + Lanczos (p->krylov == 0, as the reference) or
 * GMRES(restart) / FGMRES (krylov 1 / 2), solution out. */
int bsg_solver_csr(bsg_ctx *ctx, int n, const int *ia, const int *ja, const double *a, const double *b, double *x,
                   bsg_param *p);

/* ---- matrix and vector files in the reference's formats (host only) -------
 * Each reader works at the byte offset *offset of the file; with every array
 * NULL it returns the sizes only (offset unchanged), else it fills the arrays
 * and moves *offset past what it read, so the pieces of one file (a matrix
 * followed by its vectors, as ConvertToBinary writes them,
 * Bslib/smatrixr.cpp:4010) are read one after another.  Writers truncate the
 * file, or append when append != 0.  BSG_ERR_ARG for a malformed or
 * truncated file, with its path in the message. */
/* CSMatrixR::ReadMtrBin (Bslib/smatrixr.cpp:3852): int m, n, nlist, nzja;
 * int list[nlist], ia[nlist+1], ja[nzja]; double a[nzja], native order. */
int bsg_read_mtr_bin(const char *path, long long *offset, int *m, int *n, int *nlist, int *nzja, int *list, int *ia,
                     int *ja, double *a);
/* CSMatrixR::WriteMtrBin (Bslib/smatrixr.cpp:3984), the same layout. */
int bsg_write_mtr_bin(const char *path, int append, int m, int n, int nlist, const int *list, const int *ia,
                      const int *ja, const double *a);
/* CSMatrixR::ReadMtr (Bslib/smatrixr.cpp:3888), the text form: n and nzja,
 * a label line, ia[n+1], a label line, ja[nzja], a label line, a[nzja]. */
int bsg_read_mtr(const char *path, long long *offset, int *n, int *nzja, int *ia, int *ja, double *a);
/* CSVector::ReadVect (Bslib/svector.cpp:465): a label line, then nv values. */
int bsg_read_vect(const char *path, long long *offset, int nv, double *v);
/* CSVector::WriteVectBin / ReadVectBin (Bslib/svector.cpp:537 / :488):
 * int nparts, nrhs, nv; double v[nv*nrhs]; int blksv[nparts+1], inda[nparts]. */
int bsg_write_vect_bin(const char *path, int append, int nv, int nrhs, int nparts, const double *v, const int *blksv,
                       const int *inda);
int bsg_read_vect_bin(const char *path, long long *offset, int *nv, int *nrhs, int *nparts, double *v, int *blksv,
                      int *inda);

/* ---- learned preconditioner stage (no counterpart in the reference) --------
 * A 4-level 3D convolutional U-Net (16 base channels, bf16 weights, FP32
 * accumulation) on an nx x ny x nz grid (sides multiples of 8), natural
 * order.  Inside FGMRES (p->krylov == 2, p->learned = the network) it follows
 * the ILU2 step z = M^{-1} v with z += |r1| N(r1 / |r1|), r1 = v - A z; a
 * non-finite network output leaves the plain ILU2 step.  Weights are a flat
 * FP32 vector: W0..W6 as [27 taps][cout][cin], then the 16 head weights. */
typedef struct bsg_unet bsg_unet;
int bsg_unet_create(bsg_ctx *ctx, int nx, int ny, int nz, int train, bsg_unet **out);
int bsg_unet_free(bsg_unet *u);
int bsg_unet_nparam(const bsg_unet *u);                   /* BSG_ERR_ARG for a null network */
int bsg_unet_set_weights(bsg_unet *u, const float *w);   /* host, nparam floats */
int bsg_unet_get_weights(bsg_unet *u, float *w);
int bsg_unet_get_grads(bsg_unet *u, float *g);           /* accumulated sums */
/* the operator: its diagonal is the second input channel; FGMRES forms r1 with it */
int bsg_unet_set_matrix(bsg_unet *u, const bsg_mat *m);
/* the second input channel from a device vector of diagonal values only */
int bsg_unet_set_diag(bsg_unet *u, const double *d_diag);
/* d_y = |r| N(r / |r|), device FP64 vectors of the grid's length */
int bsg_unet_forward_dev(bsg_unet *u, const double *d_r, double *d_y);
/* one training sample (device r and target t); accumulates weight gradients
 * of |N(r/|r|) - t/|r||^2 / |t/|r||^2, writes that loss to *loss if given */
int bsg_unet_train_sample(bsg_unet *u, const double *d_r, const double *d_t, double *loss);
int bsg_unet_adam(bsg_unet *u, float lr, float beta1, float beta2, float eps, int step);
int bsg_unet_zero_grads(bsg_unet *u);

/* ---- measurement (no counterpart in the reference; it times with clock())  */
/* Number of kernels this library has launched in the process so far. */
unsigned long long bsg_launch_count(void);
/* Average device time of `reps` launches of one kernel (kind 0: SpMV of m;
 * 1 / 2: forward / backward solve with f in `mode`/`nsweeps`; 3: product of
 * m with `nsweeps` vectors at once, 1..64), CUDA events. */
int bsg_time_kernel(bsg_ctx *ctx, int kind, const bsg_mat *m, const bsg_fct *f, int mode, int nsweeps, int reps,
                    double *ms_per_launch);
/* Scheduler counters of the last factorisation (see k_fact.cu); the first
 * nout of them (BSG_ERR_ARG for a null out with nout > 0). */
int bsg_fact_stats(unsigned long long *out, int nout);
/* Stored entries, padding included, of the sliced copies the bandwidth-bound
 * products read: out[0] matrix, out[1] strict L, out[2] strict U; out[3] /
 * out[4] tiles of the tiled FP32 L / U sweeps (0: untiled, columns gathered
 * from global memory), out[5] most 32-float x blocks one tile stages;
 * out[6] / out[7] / out[8] rows of the matrix / L / U longer than 256
 * entries, kept out of the slices and summed by a warp or block each.  For
 * a 3x3 block factor out[1] / out[2] count 9 entries per stored block of
 * its block-sliced copies and out[7] / out[8] block rows of more than 64
 * blocks.
 * out holds 9 values. */
int bsg_sell_stats(const bsg_mat *m, const bsg_fct *f, long long *out);

#ifdef __cplusplus
}
#endif
#endif
