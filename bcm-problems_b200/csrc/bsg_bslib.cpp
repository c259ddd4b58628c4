// GPU drop-ins for Bslib's abstract-interface solvers (include/bsg_bslib.h).
//
// AbstractSymmSolver / AbstractSolver (Bslib/solvers.cpp:5383, :5591) read a
// block system through seven generator callbacks, sort each block row by
// column, and hand the CSMatrixRS to CSVector::SolveSymm / Solver.  This file
// keeps the callback protocol exactly (order, the callee-allocated ia / ja
// released with delete[], block rows delivered in the callee's column order
// and sorted here, right-hand side and initial guess per block row, the
// solution stored back per block row) and replaces the assembly target and
// the solve: the sorted block CSR goes to bsg_mat_vbsr, the factorisation to
// bsg_fct_ich2 / bsg_fct_ilu2 and the iteration to bsg_solve.
//
// Built against the reference's own headers (slvparam.h for CSlvParam,
// smatrix.h for the callback types), so the signatures are the reference's.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <vector>

#include "slvparam.h"
#include "smatrix.h"
#include "ExchangeMPI.h"
#include "bsg_bslib.h"

namespace {

thread_local char g_msg[512];
thread_local int g_code = BSG_OK;
thread_local bool g_ext_set = false;
thread_local bsg_param g_ext;

// The reference throws const char*; so do the drop-ins.
[[noreturn]] void raise(int code, const char *msg) {
	g_code = code;
	std::snprintf(g_msg, sizeof g_msg, "%s", msg ? msg : "error");
	throw static_cast<const char *>(g_msg);
}

void check(int rc) {
	if (rc != BSG_OK) raise(rc, bsg_last_error());
}

// One library context per thread, on the device named by BSG_DEVICE (0 by
// default), created on first use and kept for the thread's life.
bsg_ctx *context() {
	thread_local bsg_ctx *c = nullptr;
	if (!c) {
		const char *d = std::getenv("BSG_DEVICE");
		check(bsg_create(&c, d ? std::atoi(d) : 0, nullptr));
	}
	return c;
}

void to_bsg(const CSlvParam &p, bsg_param &q) {
	bsg_param_default(&q);
	if (g_ext_set) {
		q.precision = g_ext.precision;
		q.trisolve = g_ext.trisolve;
		q.nsweeps = g_ext.nsweeps;
		q.krylov = g_ext.krylov;
		q.restart = g_ext.restart;
		q.true_residual = g_ext.true_residual;
		q.blockfct = g_ext.blockfct;
		q.learned = g_ext.learned;
	}
	q.msglev = p.msglev;
	q.fcttyp = p.fcttyp;
	q.ordtype = 0; // natural order on the GPU (see the header)
	q.memory = p.memory;
	q.tau1 = p.tau1;
	q.tau2 = p.tau2;
	q.theta = p.theta;
	q.sclmin = p.sclmin;
	q.pivmin = p.pivmin;
	q.ittype = p.ittype;
	q.sttype = p.sttype;
	q.niter = p.niter;
	q.eps = p.eps;
	q.ichk = p.ichk;
}

void from_bsg(const bsg_param &q, CSlvParam &p) {
	p.nitperf = q.nitperf;
	p.resfin = q.resfin;
	p.density = q.density;
	p.density2 = q.density2;
	p.timefct = q.timefct;
	p.timeitr = q.timeitr;
}

// The system as the callbacks deliver it, block rows sorted by column.
struct Assembled {
	int nsup = 0;
	std::vector<int> sprnd, ia, ja;
	std::vector<double> a, b, x;
};

Assembled assemble(void *g, CNSUP fnsup, CSPRNDS fsprnds, CIAJA fiaja, CBLOCKROW fblockrow, CRHS frhs,
                   CINIGUESS finiguess) {
	Assembled s;
	int nsup = 0;
	fnsup(g, nsup);
	if (nsup < 0) raise(BSG_ERR_ARG, "AbstractSolver: negative number of block rows");
	s.nsup = nsup;
	s.sprnd.assign(nsup + 1, 0);
	fsprnds(g, s.sprnd.data());
	for (int i = 0; i < nsup; i++)
		if (s.sprnd[i + 1] <= s.sprnd[i]) raise(BSG_ERR_ARG, "AbstractSolver: block sizes must be positive");
	const int n = s.sprnd[nsup];
	int *cia = nullptr, *cja = nullptr;
	fiaja(g, cia, cja);
	if (!cia || (cia[nsup] > 0 && !cja)) raise(BSG_ERR_ARG, "AbstractSolver: the pattern callback gave no arrays");
	// the callee allocated ia / ja; the solver releases them (Bslib/solvers.cpp:5786-5788)
	struct Owned {
		int *p;
		~Owned() { delete[] p; }
	} oia{cia}, oja{cja};
	if (cia[0] != 0) raise(BSG_ERR_ARG, "AbstractSolver: ia[0] != 0");
	const int nzj = cia[nsup];
	s.ia.assign(cia, cia + nsup + 1);
	s.ja.resize(nzj);
	// sizes of the block rows and of the largest one
	long long nza = 0, rowmax = 0;
	for (int i = 0; i < nsup; i++) {
		if (cia[i + 1] < cia[i]) raise(BSG_ERR_ARG, "AbstractSolver: ia not monotone");
		const long long bi = s.sprnd[i + 1] - s.sprnd[i];
		long long row = 0;
		for (int k = cia[i]; k < cia[i + 1]; k++) {
			const int j = cja[k];
			if (j < 0 || j >= nsup) raise(BSG_ERR_ARG, "AbstractSolver: block column out of range");
			row += bi * (s.sprnd[j + 1] - s.sprnd[j]);
		}
		nza += row;
		rowmax = std::max(rowmax, row);
	}
	s.a.resize((size_t)nza);
	std::vector<double> arow((size_t)std::max<long long>(rowmax, 1));
	std::vector<std::pair<int, long long>> order; // (column, offset in arow)
	size_t out = 0;
	for (int i = 0; i < nsup; i++) {
		const int bi = s.sprnd[i + 1] - s.sprnd[i];
		order.clear();
		long long off = 0;
		for (int k = cia[i]; k < cia[i + 1]; k++) {
			const int j = cja[k];
			order.push_back({j, off});
			off += (long long)bi * (s.sprnd[j + 1] - s.sprnd[j]);
		}
		fblockrow(g, i, arow.data());
		std::sort(order.begin(), order.end());
		for (size_t q = 0; q < order.size(); q++) {
			const int j = order[q].first;
			if (q > 0 && order[q - 1].first == j) raise(BSG_ERR_ARG, "AbstractSolver: repeated block column");
			const size_t len = (size_t)bi * (s.sprnd[j + 1] - s.sprnd[j]);
			s.ja[cia[i] + q] = j;
			std::memcpy(s.a.data() + out, arow.data() + order[q].second, sizeof(double) * len);
			out += len;
		}
	}
	s.b.assign(n, 0.0);
	s.x.assign(n, 0.0);
	for (int i = 0; i < nsup; i++) frhs(g, i, s.b.data() + s.sprnd[i]);
	for (int i = 0; i < nsup; i++) finiguess(g, i, s.x.data() + s.sprnd[i]);
	return s;
}

void solve(bool symm, void *g, CSlvParam &param, CNSUP fnsup, CSPRNDS fsprnds, CIAJA fiaja, CBLOCKROW fblockrow,
           CRHS frhs, CINIGUESS finiguess, CSTORESOL fstoresol) {
	g_code = BSG_OK;
	Assembled s = assemble(g, fnsup, fsprnds, fiaja, fblockrow, frhs, finiguess);
	bsg_param q;
	to_bsg(param, q);
	bsg_ctx *c = context();
	bsg_mat *m = nullptr;
	bsg_fct *f = nullptr;
	// the block Lanczos variants of Solver(CSMatrixRS&) (ittype 2 / 3 / 4)
	// run on the point form: the GPU's transposed solves are point solves
	const bool point = !symm && q.krylov == 0 && q.ittype >= 2 && q.ittype <= 4;
	int rc = bsg_mat_vbsr(c, s.nsup, s.sprnd.data(), s.ia.data(), s.ja.data(), s.a.data(),
	                      (symm ? 1 : 0) | (point ? BSG_VBSR_POINT : 0), &m);
	if (!rc) rc = symm ? bsg_fct_ich2(c, m, &q, &f) : bsg_fct_ilu2(c, m, &q, &f);
	if (!rc) rc = bsg_solve(c, m, f, s.b.data(), s.x.data(), &q);
	bsg_fct_free(f);
	bsg_mat_free(m);
	// the iteration limit is not an exception in the reference: the last
	// iterate is stored and nitperf / resfin tell the caller
	if (rc != BSG_OK && rc != BSG_ERR_NOCONV) check(rc);
	g_code = rc;
	from_bsg(q, param);
	for (int i = 0; i < s.nsup; i++) fstoresol(g, i, s.x.data() + s.sprnd[i]);
}

} // namespace

namespace bsg_bslib {

void AbstractSymmSolver(void *_pgener, std::ofstream &_fout, CSlvParam &_param, CNSUP _fnsup, CSPRNDS _fsprnds,
                        CIAJA _fiaja, CBLOCKROW _fblockrow, CRHS _frhs, CINIGUESS _finiguess, CSTORESOL _fstoresol) {
	(void)_fout;
	solve(true, _pgener, _param, _fnsup, _fsprnds, _fiaja, _fblockrow, _frhs, _finiguess, _fstoresol);
}

void AbstractSolver(void *_pgener, std::ofstream &_fout, CSlvParam &_param, CNSUP _fnsup, CSPRNDS _fsprnds,
                    CIAJA _fiaja, CBLOCKROW _fblockrow, CRHS _frhs, CINIGUESS _finiguess, CSTORESOL _fstoresol) {
	(void)_fout;
	solve(false, _pgener, _param, _fnsup, _fsprnds, _fiaja, _fblockrow, _frhs, _finiguess, _fstoresol);
}

void AbstractParSolver(void *_pgener, void *_comm, std::ofstream &_fout, CSlvParam &_param, CNSUP _fnsup,
                       CSPRNDS _fsprnds, CIAJA _fiaja, CBLOCKROW _fblockrow, CRHS _frhs, CINIGUESS _finiguess,
                       CSTORESOL _fstoresol) {
	(void)_fout;
	if (_comm && static_cast<CMPIComm *>(_comm)->GetNproc() != 1)
		raise(BSG_ERR_UNSUPPORTED, "AbstractParSolver: the GPU path runs on one process (nproc must be 1)");
	solve(false, _pgener, _param, _fnsup, _fsprnds, _fiaja, _fblockrow, _frhs, _finiguess, _fstoresol);
}

void SetGpuOptions(const bsg_param &ext) {
	g_ext = ext;
	g_ext_set = true;
}

} // namespace bsg_bslib

// ---- GPU operators for the reference's callback Krylov loops -----------------

namespace {

struct Operator {
	bsg_ctx *c = nullptr;
	bsg_mat *m = nullptr;
	bsg_fct *f = nullptr;
	int n = 0;
	int mode = 0, nsweeps = 3;
	std::vector<double> tmp;
};

// The vector's columns (nv entries each, nrhs of them) one after another.
template <class F>
void each_column(CSVector &x, CSVector &y, int n, F fn) {
	const int nv = x.GetNv(), nr = x.GetNrhs();
	if (nv != n || y.GetNv() != n || y.GetNrhs() != nr) raise(BSG_ERR_ARG, "GPU operator: vector of the wrong size");
	for (int k = 0; k < nr; k++) check(fn(x.GetVect() + (size_t)k * n, y.GetVect() + (size_t)k * n));
}

} // namespace

namespace bsg_bslib {

void MvmA(void *_obj, CSVector &_x, CSVector &_ax) {
	Operator *o = static_cast<Operator *>(_obj);
	each_column(_x, _ax, o->n, [o](const double *x, double *y) { return bsg_mvm(o->c, o->m, x, y); });
}
void SolveLU(void *_obj, CSVector &_x, CSVector &_lux) {
	Operator *o = static_cast<Operator *>(_obj);
	each_column(_x, _lux, o->n,
	            [o](const double *x, double *y) { return bsg_solve_lu(o->c, o->f, 0, o->mode, o->nsweeps, x, y); });
}
void SolveL(void *_obj, CSVector &_x, CSVector &_lx) {
	Operator *o = static_cast<Operator *>(_obj);
	each_column(_x, _lx, o->n,
	            [o](const double *x, double *y) { return bsg_solve_lu(o->c, o->f, 1, o->mode, o->nsweeps, x, y); });
}
void SolveU(void *_obj, CSVector &_x, CSVector &_ux) {
	Operator *o = static_cast<Operator *>(_obj);
	each_column(_x, _ux, o->n,
	            [o](const double *x, double *y) { return bsg_solve_lu(o->c, o->f, 2, o->mode, o->nsweeps, x, y); });
}

} // namespace bsg_bslib

extern "C" int bsg_bslib_operator_create(int n, const int *ia, const int *ja, const double *a, int symm_upper,
                                         bsg_param *p, void **op) {
	g_msg[0] = 0;
	if (!op || !p) return BSG_ERR_ARG;
	*op = nullptr;
	Operator *o = new (std::nothrow) Operator();
	if (!o) return BSG_ERR_NOMEM;
	int rc = BSG_OK;
	try {
		o->c = context();
	} catch (const char *) {
		rc = g_code;
	}
	bsg_param q = *p;
	q.ordtype = 0;
	if (!rc) rc = bsg_mat_csr(o->c, n, ia, ja, a, symm_upper, &o->m);
	if (!rc) rc = symm_upper ? bsg_fct_ich2(o->c, o->m, &q, &o->f) : bsg_fct_ilu2(o->c, o->m, &q, &o->f);
	if (rc) {
		std::snprintf(g_msg, sizeof g_msg, "%s", bsg_last_error());
		bsg_fct_free(o->f);
		bsg_mat_free(o->m);
		delete o;
		return rc;
	}
	o->n = n;
	o->mode = q.trisolve;
	o->nsweeps = q.nsweeps;
	p->density = q.density;
	p->density2 = q.density2;
	p->timefct = q.timefct;
	*op = o;
	return BSG_OK;
}

extern "C" int bsg_bslib_operator_free(void *op) {
	Operator *o = static_cast<Operator *>(op);
	if (!o) return BSG_OK;
	bsg_fct_free(o->f);
	bsg_mat_free(o->m);
	delete o;
	return BSG_OK;
}

extern "C" void bsg_bslib_operator_fns(void *fns[4]) {
	fns[0] = reinterpret_cast<void *>(static_cast<CMVM>(&bsg_bslib::MvmA));
	fns[1] = reinterpret_cast<void *>(static_cast<CSOLVELU>(&bsg_bslib::SolveLU));
	fns[2] = reinterpret_cast<void *>(static_cast<CSOLVEL>(&bsg_bslib::SolveL));
	fns[3] = reinterpret_cast<void *>(static_cast<CSOLVEU>(&bsg_bslib::SolveU));
}

extern "C" const char *bsg_bslib_last_error(void) { return g_msg; }

extern "C" int bsg_bslib_abstract(int symm, void *gener, void *const fns[7], bsg_param *p) {
	g_code = BSG_OK;
	g_msg[0] = 0;
	if (!fns || !p) {
		std::snprintf(g_msg, sizeof g_msg, "bsg_bslib_abstract: null argument");
		return BSG_ERR_ARG;
	}
	for (int k = 0; k < 7; k++)
		if (!fns[k]) {
			std::snprintf(g_msg, sizeof g_msg, "bsg_bslib_abstract: callback %d is null", k + 1);
			return BSG_ERR_ARG;
		}
	CSlvParam cp;
	cp.msglev = p->msglev;
	cp.fcttyp = p->fcttyp;
	cp.ordtype = p->ordtype;
	cp.memory = p->memory;
	cp.tau1 = p->tau1;
	cp.tau2 = p->tau2;
	cp.theta = p->theta;
	cp.sclmin = p->sclmin;
	cp.pivmin = p->pivmin;
	cp.ittype = p->ittype;
	cp.sttype = p->sttype;
	cp.niter = p->niter;
	cp.eps = p->eps;
	cp.ichk = p->ichk;
	const bool had = g_ext_set;
	const bsg_param saved = g_ext;
	g_ext = *p;
	g_ext_set = true;
	int rc = BSG_OK;
	try {
		std::ofstream nowhere;
		const auto f0 = reinterpret_cast<CNSUP>(fns[0]);
		const auto f1 = reinterpret_cast<CSPRNDS>(fns[1]);
		const auto f2 = reinterpret_cast<CIAJA>(fns[2]);
		const auto f3 = reinterpret_cast<CBLOCKROW>(fns[3]);
		const auto f4 = reinterpret_cast<CRHS>(fns[4]);
		const auto f5 = reinterpret_cast<CINIGUESS>(fns[5]);
		const auto f6 = reinterpret_cast<CSTORESOL>(fns[6]);
		if (symm == 2)
			bsg_bslib::AbstractParSolver(gener, nullptr, nowhere, cp, f0, f1, f2, f3, f4, f5, f6);
		else
			solve(symm != 0, gener, cp, f0, f1, f2, f3, f4, f5, f6);
		p->nitperf = cp.nitperf;
		p->resfin = cp.resfin;
		p->density = cp.density;
		p->density2 = cp.density2;
		p->timefct = cp.timefct;
		p->timeitr = cp.timeitr;
		rc = g_code;
		if (rc == BSG_ERR_NOCONV) std::snprintf(g_msg, sizeof g_msg, "iteration limit reached");
	} catch (const char *) {
		rc = g_code != BSG_OK ? g_code : BSG_ERR_ARG;
	}
	g_ext = saved;
	g_ext_set = had;
	return rc;
}
