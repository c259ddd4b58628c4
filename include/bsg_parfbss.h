/* bsg_parfbss.h -- Bslib's ParFBSS_* interface (Bslib/parfbss.h:10-27) on
 * one GPU, implemented in libbsg.so.
 *
 * The reference's functions keep their names, signatures and C++ linkage, so
 * a program written against parfbss.h links against libbsg.so unchanged; the
 * bsg_parfbss_* twins are the same functions with C linkage.  One process
 * holds all rows: LIST must number the rows 0 .. NI-1 once each (the rows of
 * other MPI ranks cannot be reached), and the communicator argument is not
 * used.  SolveSymm factors the upper triangle of the rows with IC2 and runs
 * PCG; Solve factors with ILU2 and runs GMRES(restart); both in natural
 * order, to eps (relative when eps > 0, absolute when eps < 0, as
 * Bslib/parfbss.cpp:1700-1709).  Return values are the reference's: 0 on
 * success, -1 for a bad object number or malformed data, 1 when no object
 * can be allocated; a failure of the GPU solve returns its BSG_ERR_* code.
 * Up to 20 objects at a time (ParFBSS_Array, Bslib/parfbss_data.h:20-33).
 */
#ifndef BSG_PARFBSS_H
#define BSG_PARFBSS_H
#include "bslib_gpu.h"

#ifdef __cplusplus
/* The reference's declarations, identical (Bslib/parfbss.h:10-27). */
int ParFBSS_Create(void *_Comm, int _NI, int _NZAI, int *_ObjId);
int ParFBSS_ReCreate(int _ObjId, int _NI, int _NZAI);
int ParFBSS_LinearEquationsData(int _ObjId, int **_LIST, int **_IA, int **_JA, double **_A, double **_RightHandSide,
                                double **_InitialGuess);
int ParFBSS_NormalizationData(int _ObjId, double **_Norm);
int ParFBSS_NonLinearEquationsData(int _ObjId, double **_Poly2);
int ParFBSS_SetSolverParameters(int _ObjId, int _NpDistr, double _Tau1, double _Tau2, double _Theta, int _NIterMax,
                                double _Eps);
int ParFBSS_SetMsglevAndFilename(int _ObjId, int _Msglev, char *_FileName);
int ParFBSS_SetSchurtype(int _ObjId, int _Schurtype, int _Ncycle);
int ParFBSS_SetNcpuext(int _ObjId, int _NcpuExt);
int ParFBSS_SolveSymm(int _ObjId, int _Job, int *_NIterPerf);
int ParFBSS_Solve(int _ObjId, int _Job, int *_NIterPerf);
int ParFBSS_Solution(int _ObjId, double **_Solution);
int ParFBSS_Distribution(int _ObjId, int *_NIOpt, int **_LISTOpt);
int ParFBSS_Destroy(int _ObjId);
extern "C" {
#endif

/* ParFBSS_Create (Bslib/parfbss.cpp:24): an object for NI rows and NZAI
 * entries; its number in *objid; -1 when all 20 are taken. */
int bsg_parfbss_create(void *comm, int ni, int nzai, int *objid);
/* ParFBSS_ReCreate (:55): new arrays for NI rows and NZAI entries. */
int bsg_parfbss_recreate(int objid, int ni, int nzai);
/* ParFBSS_LinearEquationsData (:69): pointers to the object's arrays for the
 * caller to fill -- LIST[NI] (global row numbers), IA[NI+1], JA[NZAI] (global
 * columns, any order), A[NZAI], the right-hand side and the initial guess. */
int bsg_parfbss_linear_equations_data(int objid, int **list, int **ia, int **ja, double **a, double **rhs,
                                      double **x0);
/* ParFBSS_NormalizationData (:89) / ParFBSS_NonLinearEquationsData (:107):
 * the norm vector (ones) and the second-order term (zeros), kept for the
 * caller; the linear solve does not read them. */
int bsg_parfbss_normalization_data(int objid, double **norm);
int bsg_parfbss_nonlinear_equations_data(int objid, double **poly2);
/* ParFBSS_SetSolverParameters (:125): distribution size (kept), IC2 / ILU2
 * thresholds and theta, iteration limit, eps (sign: relative / absolute). */
int bsg_parfbss_set_solver_parameters(int objid, int npdistr, double tau1, double tau2, double theta, int niter,
                                      double eps);
/* ParFBSS_SetMsglevAndFilename (:148), ParFBSS_SetSchurtype (:166),
 * ParFBSS_SetNcpuext (:184): kept; they steer the reference's MPI
 * distribution, which one GPU does not have. */
int bsg_parfbss_set_msglev_and_filename(int objid, int msglev, const char *filename);
int bsg_parfbss_set_schurtype(int objid, int schurtype, int ncycle);
int bsg_parfbss_set_ncpuext(int objid, int ncpuext);
/* The GPU-path fields of bsg_param (precision, trisolve, nsweeps, restart,
 * true_residual, learned) for this object's later solves; no counterpart in
 * the reference. */
int bsg_parfbss_set_gpu_options(int objid, const bsg_param *p);
/* ParFBSS_SolveSymm (:202) / ParFBSS_Solve (:220); job 1 computes the
 * distribution, other values reuse it (the same on one process). */
int bsg_parfbss_solve_symm(int objid, int job, int *niterperf);
int bsg_parfbss_solve(int objid, int job, int *niterperf);
/* ParFBSS_Solution (:238): the solution, in the order of the object's rows. */
int bsg_parfbss_solution(int objid, double **solution);
/* ParFBSS_Distribution (:256): the rows this process solved (all of them). */
int bsg_parfbss_distribution(int objid, int *niopt, int **listopt);
/* ParFBSS_Destroy (:280). */
int bsg_parfbss_destroy(int objid);

#ifdef __cplusplus
}
#endif
#endif
