/* bsg_bslib.h -- GPU drop-ins for Bslib's abstract-interface solvers.
 *
 * Bslib's AbstractSymmSolver / AbstractSolver (declared in Bslib/smatrix.h:
 * 27-34, defined in Bslib/solvers.cpp:5383 and :5591) assemble a block
 * matrix through seven generator callbacks and solve it with
 * CSVector::SolveSymm / CSVector::Solver.  The functions below have the same
 * signatures, call the callbacks in the same order with the same ownership
 * rules, and solve on the GPU through libbsg.so:
 *
 *   1. _fnsup(obj, nsup)                 number of block rows
 *   2. _fsprnds(obj, sprnds[nsup + 1])   prefix block sizes
 *   3. _fiaja(obj, ia, ja)               block pattern, allocated by the callee
 *                                        with new[]; released here with delete[]
 *   4. _fblockrow(obj, i, arow)          block row i, blocks in the callee's ja
 *                                        order, each column-major; sorted here
 *   5. _frhs(obj, i, b_i), 6. _finiguess(obj, i, x_i)   per block row
 *   7. after the solve, _fstoresol(obj, i, x_i)          per block row
 *
 * AbstractSymmSolver expects the upper block triangle (SolveSymm's storage)
 * and runs block IC2 (3x3 blocks: CSMatrixRS::Ich2 with eigenvector scaling)
 * or point IC2 of the point expansion (other block sizes) and PCG;
 * AbstractSolver runs block / point ILU2 and the Krylov method of
 * bsg_solve().  The CSlvParam outputs nitperf, resfin, density, density2,
 * timefct and timeitr are filled.  Errors are thrown as const char *, as the
 * reference does, with the library's message.  The GPU runs natural order:
 * a nonzero ordtype (a choice of preconditioner quality in the reference)
 * is read as 0.
 *
 * The C++ drop-ins need the reference's CSlvParam (Bslib/slvparam.h) and the
 * callback types of Bslib/smatrix.h: include those headers before this one.
 * C callers use bsg_bslib_abstract() with bsg_param, which mirrors the
 * CSlvParam fields the path reads and writes.
 */
#ifndef BSG_BSLIB_H
#define BSG_BSLIB_H
#include "bslib_gpu.h"

#ifdef __cplusplus
#include <fstream>
namespace bsg_bslib {
/* Drop-in for AbstractSymmSolver (Bslib/solvers.cpp:5383). */
void AbstractSymmSolver(void *_pgener, std::ofstream &_fout, CSlvParam &_param, CNSUP _fnsup, CSPRNDS _fsprnds,
                        CIAJA _fiaja, CBLOCKROW _fblockrow, CRHS _frhs, CINIGUESS _finiguess, CSTORESOL _fstoresol);
/* Drop-in for AbstractSolver (Bslib/solvers.cpp:5591). */
void AbstractSolver(void *_pgener, std::ofstream &_fout, CSlvParam &_param, CNSUP _fnsup, CSPRNDS _fsprnds,
                    CIAJA _fiaja, CBLOCKROW _fblockrow, CRHS _frhs, CINIGUESS _finiguess, CSTORESOL _fstoresol);
/* Drop-in for AbstractParSolver (Bslib/solvers.cpp:5799) on one process:
 * the same callbacks, and _comm a CMPIComm of one rank (BSG_ERR_UNSUPPORTED,
 * thrown, for more ranks; NULL is taken as one rank).  Every block row is this
 * rank's; the solution of every block row goes back through _fstoresol, as
 * the reference stores the exchanged whole solution on every rank. */
void AbstractParSolver(void *_pgener, void *_comm, std::ofstream &_fout, CSlvParam &_param, CNSUP _fnsup,
                       CSPRNDS _fsprnds, CIAJA _fiaja, CBLOCKROW _fblockrow, CRHS _frhs, CINIGUESS _finiguess,
                       CSTORESOL _fstoresol);
/* The GPU-path fields of bsg_param (precision, trisolve, nsweeps, krylov,
 * restart, true_residual, blockfct, learned) that later drop-in calls of this
 * thread use; the CSlvParam fields come from each call's _param. */
void SetGpuOptions(const bsg_param &ext);

/* GPU operators for the reference's callback Krylov loops (CSVector::Cg /
 * Lanczos / BlockGMRES with a CTree, Bslib/cg.cpp:355, Bslib/lanczos.cpp:376,
 * Bslib/gmres.cpp:337), in the role CParMvmA / CParSolveLU play in the
 * reference's parallel driver (Bslib/gsmatrix.h:758, :1008): the object comes
 * from bsg_bslib_operator_create, and these functions have the CMVM /
 * CSOLVELU / CSOLVEL / CSOLVEU types of Bslib/svector.h:34-41.  Each call
 * copies the CSVector to the GPU, applies the matrix or the factor there and
 * copies the result back (all nrhs columns of the vector). */
void MvmA(void *_obj, CSVector &_x, CSVector &_ax);
void SolveLU(void *_obj, CSVector &_x, CSVector &_lux);
void SolveL(void *_obj, CSVector &_x, CSVector &_lx);
void SolveU(void *_obj, CSVector &_x, CSVector &_ux);
} // namespace bsg_bslib
extern "C" {
#endif

/* C form of the drop-ins: symm 1 is AbstractSymmSolver, 0 AbstractSolver,
 * 2 AbstractParSolver on one process (no communicator); fns holds the seven callbacks in the order above (int &
 * parameters are int * at the C level); p carries the CSlvParam fields
 * mirrored in bsg_param (and the GPU-path fields) in and the outputs out.
 * Returns BSG_OK, BSG_ERR_NOCONV when the iteration limit stopped the loop
 * (the last iterate is stored, as the reference stores it without an
 * error), or another error code; bsg_bslib_last_error() gives the message. */
int bsg_bslib_abstract(int symm, void *gener, void *const fns[7], bsg_param *p);
const char *bsg_bslib_last_error(void);

/* A GPU operator object for the callbacks above: point CSR host arrays
 * (symm_upper: upper triangle of an SPD matrix, diagonal first, factored
 * with IC2; else the full matrix, factored with ILU2), factorisation
 * parameters in p (tau1, tau2, theta, memory, precision, trisolve, nsweeps).
 * The density and factor time land in p. */
int bsg_bslib_operator_create(int n, const int *ia, const int *ja, const double *a, int symm_upper, bsg_param *p,
                              void **op);
int bsg_bslib_operator_free(void *op);
/* The four callbacks, as plain pointers: fns[0] MvmA, [1] SolveLU,
 * [2] SolveL, [3] SolveU (the functions of the C++ section). */
void bsg_bslib_operator_fns(void *fns[4]);

#ifdef __cplusplus
}
#endif
#endif
