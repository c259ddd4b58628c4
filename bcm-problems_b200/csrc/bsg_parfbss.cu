// The ParFBSS_* C interface of Bslib (Bslib/parfbss.h:10-27,
// Bslib/parfbss.cpp:24-290) on one GPU (host code).
//
// The reference keeps up to 20 solver objects (ParFBSS_Array, :20-33 of
// Bslib/parfbss_data.h).  Each owns the arrays of its rank's rows -- the
// global row numbers LIST, the CSR IA / JA / A of those rows with global
// column numbers, the right-hand side, the initial guess, a norm vector
// (ones) and a second-order term (zeros) -- and hands the caller pointers into
// them to fill (ParFBSS_LinearEquationsData, :362).  ParFBSS_SolveSymm /
// ParFBSS_Solve check the data (ParFBSS_Solve_Ini, :712: ia[0] == 0, no empty
// row, columns in range), sort every row by column, reorder and distribute the
// rows over the MPI ranks, factor (IC2 / ILU2 with tau1, tau2, theta) and
// iterate to eps (relative when eps > 0, absolute when eps < 0, :1700-1709),
// and leave the solution in the rows' own order (ParFBSS_Solution, :2259).
//
// Here one process holds every row: LIST must be a permutation of 0 .. NI-1
// (the rows of other ranks cannot be reached; such data is refused with -1),
// the matrix is assembled in global row order with the diagonal first in
// every row, and the solve runs on the GPU through bsg_fct_ich2 + PCG
// (SolveSymm, upper triangle) or bsg_fct_ilu2 + GMRES(restart) (Solve), in
// natural order.  Return values follow the reference: 0 on success, -1 for a
// bad object number or malformed data, 1 when no object can be created; a
// failure of the GPU solve returns its BSG_ERR_* code (negative, below -1).
#include "bsg_internal.cuh"
#include "../../include/bsg_parfbss.h"
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

namespace {

struct Fbss {
	int ni = 0, nzai = 0;
	std::vector<int> list, ia, ja;
	std::vector<double> a, rhs, x, sol, norm, poly2;
	// CSlvParam fields ParFBSS_SetSolverParameters / ParFBSS_SetMsglev... set
	// (Bslib/parfbss.cpp:432-510)
	int npdistr = 1, msglev = 0, schurtype = 0, ncycle = 0, ncpuext = 1;
	double tau1 = 1e-2, tau2 = 1e-4, theta = 0.1, eps = 1e-9;
	int niter = 1000;
	std::string path;
	bool have_gpu = false;
	bsg_param gpu;          // GPU-path fields (bsg_parfbss_set_gpu_options)
	std::vector<int> dist;  // ParFBSS_Distribution's list: the rows solved here
	void alloc(int n, int nz) {
		ni = n;
		nzai = nz;
		list.assign(n, 0);
		ia.assign(n + 1, 0);
		ja.assign(nz, 0);
		a.assign(nz, 0.0);
		rhs.assign(n, 0.0);
		x.assign(n, 0.0);
		sol.assign(n, 0.0);
		norm.assign(n, 1.0);
		poly2.assign(n, 0.0);
	}
};

constexpr int kObjects = 20;
Fbss *g_obj[kObjects];
std::mutex g_mu;
bsg_ctx *g_ctx = nullptr;

Fbss *get(int id) {
	if (id < 0 || id >= kObjects) return nullptr;
	return g_obj[id];
}

// One library context for the interface, on the device BSG_DEVICE (0 by
// default), created by the first solve.
int context(bsg_ctx **out) {
	std::lock_guard<std::mutex> lk(g_mu);
	if (!g_ctx) {
		const char *d = std::getenv("BSG_DEVICE");
		int rc = bsg_create(&g_ctx, d ? std::atoi(d) : 0, nullptr);
		if (rc) return rc;
	}
	*out = g_ctx;
	return BSG_OK;
}

// ParFBSS_Solve_Ini's checks plus what one process needs: every global row
// present once.  Builds the global CSR (rows sorted by column; symm: upper
// triangle, diagonal first).
int assemble(const Fbss &o, bool symm, std::vector<int> &gia, std::vector<int> &gja, std::vector<double> &ga) {
	const int n = o.ni;
	if (n <= 0 || o.ia[0] != 0) return bsg_set_error(-1, "ParFBSS: ia[0] != 0 or no rows");
	for (int i = 0; i < n; i++)
		if (o.ia[i + 1] <= o.ia[i]) return bsg_set_error(-1, "ParFBSS: empty row or ia not increasing");
	if (o.ia[n] > o.nzai) return bsg_set_error(-1, "ParFBSS: ia[NI] exceeds NZAI");
	std::vector<int> where(n, -1);
	for (int i = 0; i < n; i++) {
		const int g = o.list[i];
		if (g < 0 || g >= n || where[g] >= 0)
			return bsg_set_error(-1, "ParFBSS: LIST must number the rows 0 .. NI-1 once each on one process");
		where[g] = i;
	}
	for (int k = 0; k < o.ia[n]; k++)
		if (o.ja[k] < 0 || o.ja[k] >= n) return bsg_set_error(-1, "ParFBSS: column index out of range");
	gia.assign(n + 1, 0);
	gja.clear();
	ga.clear();
	std::vector<std::pair<int, double>> row;
	for (int g = 0; g < n; g++) {
		const int i = where[g];
		row.clear();
		bool diag = false;
		for (int k = o.ia[i]; k < o.ia[i + 1]; k++) {
			const int j = o.ja[k];
			if (symm && j < g) continue;
			if (j == g) diag = true;
			row.push_back({j, o.a[k]});
		}
		std::stable_sort(row.begin(), row.end(),
		                 [](const std::pair<int, double> &p, const std::pair<int, double> &q) { return p.first < q.first; });
		for (size_t q = 1; q < row.size(); q++)
			if (row[q].first == row[q - 1].first) return bsg_set_error(-1, "ParFBSS: repeated column in a row");
		if (symm && !diag) return bsg_set_error(-1, "ParFBSS: a row without its diagonal entry");
		for (auto &e : row) {
			gja.push_back(e.first);
			ga.push_back(e.second);
		}
		gia[g + 1] = (int)gja.size();
	}
	return BSG_OK;
}

int solve(int id, bool symm, int job, int *niterperf) {
	Fbss *o = get(id);
	if (!o) return bsg_set_error(-1, "ParFBSS: bad object number");
	(void)job; // 1: compute the distribution, else reuse it -- one process: the same
	std::vector<int> gia, gja;
	std::vector<double> ga;
	int rc = assemble(*o, symm, gia, gja, ga);
	if (rc) return rc;
	const int n = o->ni;
	bsg_param p;
	bsg_param_default(&p);
	if (o->have_gpu) {
		p.precision = o->gpu.precision;
		p.trisolve = o->gpu.trisolve;
		p.nsweeps = o->gpu.nsweeps;
		p.restart = o->gpu.restart;
		p.true_residual = o->gpu.true_residual;
		p.learned = o->gpu.learned;
	}
	// the settings of ParFBSS_SetSolverParameters (Bslib/parfbss.cpp:432-462)
	// in natural order on the GPU; eps > 0 relative, eps < 0 absolute
	p.msglev = o->msglev;
	p.fcttyp = 2;
	p.ordtype = 0;
	p.memory = 20.0;
	p.tau1 = o->tau1;
	p.tau2 = o->tau2;
	p.theta = o->theta;
	p.niter = o->niter;
	p.eps = o->eps < 0 ? -o->eps : o->eps;
	p.ittype = o->eps < 0 ? 1 : 0;
	p.sttype = o->eps < 0 ? 0 : 1;
	p.krylov = symm ? 0 : 1;
	bsg_ctx *c = nullptr;
	rc = context(&c);
	if (rc) return rc;
	// right-hand side and initial guess to global order
	std::vector<double> b(n), x(n);
	for (int i = 0; i < n; i++) {
		b[o->list[i]] = o->rhs[i];
		x[o->list[i]] = o->x[i];
	}
	bsg_mat *m = nullptr;
	bsg_fct *f = nullptr;
	rc = bsg_mat_csr(c, n, gia.data(), gja.data(), ga.data(), symm ? 1 : 0, &m);
	if (!rc) rc = symm ? bsg_fct_ich2(c, m, &p, &f) : bsg_fct_ilu2(c, m, &p, &f);
	if (!rc) rc = bsg_solve(c, m, f, b.data(), x.data(), &p);
	bsg_fct_free(f);
	bsg_mat_free(m);
	if (rc && rc != BSG_ERR_NOCONV) return rc;
	// the reference reports the iterations it made whether or not eps was met
	for (int i = 0; i < n; i++) o->sol[i] = x[o->list[i]];
	o->dist = o->list;
	if (niterperf) *niterperf = p.nitperf;
	return BSG_OK;
}

} // namespace

extern "C" {

int bsg_parfbss_create(void *comm, int ni, int nzai, int *objid) {
	(void)comm; // one process: the communicator has nothing to distribute over
	if (!objid || ni < 0 || nzai < 0) return -1;
	std::lock_guard<std::mutex> lk(g_mu);
	for (int i = 0; i < kObjects; i++)
		if (!g_obj[i]) {
			Fbss *o = new (std::nothrow) Fbss();
			if (!o) return 1;
			try {
				o->alloc(ni, nzai);
			} catch (...) {
				delete o;
				return 1;
			}
			g_obj[i] = o;
			*objid = i;
			return 0;
		}
	return -1;
}

int bsg_parfbss_recreate(int id, int ni, int nzai) {
	Fbss *o = get(id);
	if (!o || ni < 0 || nzai < 0) return -1;
	try {
		o->alloc(ni, nzai);
	} catch (...) {
		return 1;
	}
	return 0;
}

int bsg_parfbss_linear_equations_data(int id, int **list, int **ia, int **ja, double **a, double **rhs,
                                      double **x0) {
	Fbss *o = get(id);
	if (!o || !list || !ia || !ja || !a || !rhs || !x0) return -1;
	*list = o->list.data();
	*ia = o->ia.data();
	*ja = o->ja.data();
	*a = o->a.data();
	*rhs = o->rhs.data();
	*x0 = o->x.data();
	return 0;
}

int bsg_parfbss_normalization_data(int id, double **norm) {
	Fbss *o = get(id);
	if (!o || !norm) return -1;
	*norm = o->norm.data();
	return 0;
}

int bsg_parfbss_nonlinear_equations_data(int id, double **poly2) {
	Fbss *o = get(id);
	if (!o || !poly2) return -1;
	*poly2 = o->poly2.data();
	return 0;
}

int bsg_parfbss_set_solver_parameters(int id, int npdistr, double tau1, double tau2, double theta, int niter,
                                      double eps) {
	Fbss *o = get(id);
	if (!o) return -1;
	o->npdistr = npdistr;
	o->tau1 = tau1;
	o->tau2 = tau2;
	o->theta = theta;
	o->niter = niter;
	o->eps = eps;
	return 0;
}

int bsg_parfbss_set_msglev_and_filename(int id, int msglev, const char *filename) {
	Fbss *o = get(id);
	if (!o) return -1;
	o->msglev = msglev;
	o->path = filename ? filename : "";
	return 0;
}

int bsg_parfbss_set_schurtype(int id, int schurtype, int ncycle) {
	Fbss *o = get(id);
	if (!o) return -1;
	o->schurtype = schurtype;
	o->ncycle = ncycle;
	return 0;
}

int bsg_parfbss_set_ncpuext(int id, int ncpuext) {
	Fbss *o = get(id);
	if (!o) return -1;
	o->ncpuext = ncpuext;
	return 0;
}

int bsg_parfbss_set_gpu_options(int id, const bsg_param *p) {
	Fbss *o = get(id);
	if (!o || !p) return -1;
	o->gpu = *p;
	o->have_gpu = true;
	return 0;
}

int bsg_parfbss_solve_symm(int id, int job, int *niterperf) { return solve(id, true, job, niterperf); }
int bsg_parfbss_solve(int id, int job, int *niterperf) { return solve(id, false, job, niterperf); }

int bsg_parfbss_solution(int id, double **solution) {
	Fbss *o = get(id);
	if (!o || !solution) return -1;
	*solution = o->sol.data();
	return 0;
}

int bsg_parfbss_distribution(int id, int *niopt, int **listopt) {
	Fbss *o = get(id);
	if (!o || !niopt || !listopt) return -1;
	if (o->dist.empty()) o->dist = o->list;
	*niopt = (int)o->dist.size();
	*listopt = o->dist.data();
	return 0;
}

int bsg_parfbss_destroy(int id) {
	std::lock_guard<std::mutex> lk(g_mu);
	if (id < 0 || id >= kObjects || !g_obj[id]) return -1;
	delete g_obj[id];
	g_obj[id] = nullptr;
	return 0;
}

} // extern "C"

// The reference's own names and C++ linkage (Bslib/parfbss.h:10-27), so a
// caller compiled against parfbss.h links against this library unchanged.
int ParFBSS_Create(void *_Comm, int _NI, int _NZAI, int *_ObjId) { return bsg_parfbss_create(_Comm, _NI, _NZAI, _ObjId); }
int ParFBSS_ReCreate(int _ObjId, int _NI, int _NZAI) { return bsg_parfbss_recreate(_ObjId, _NI, _NZAI); }
int ParFBSS_LinearEquationsData(int _ObjId, int **_LIST, int **_IA, int **_JA, double **_A, double **_RightHandSide,
                                double **_InitialGuess) {
	return bsg_parfbss_linear_equations_data(_ObjId, _LIST, _IA, _JA, _A, _RightHandSide, _InitialGuess);
}
int ParFBSS_NormalizationData(int _ObjId, double **_Norm) { return bsg_parfbss_normalization_data(_ObjId, _Norm); }
int ParFBSS_NonLinearEquationsData(int _ObjId, double **_Poly2) {
	return bsg_parfbss_nonlinear_equations_data(_ObjId, _Poly2);
}
int ParFBSS_SetSolverParameters(int _ObjId, int _NpDistr, double _Tau1, double _Tau2, double _Theta, int _NIterMax,
                                double _Eps) {
	return bsg_parfbss_set_solver_parameters(_ObjId, _NpDistr, _Tau1, _Tau2, _Theta, _NIterMax, _Eps);
}
int ParFBSS_SetMsglevAndFilename(int _ObjId, int _Msglev, char *_FileName) {
	return bsg_parfbss_set_msglev_and_filename(_ObjId, _Msglev, _FileName);
}
int ParFBSS_SetSchurtype(int _ObjId, int _Schurtype, int _Ncycle) {
	return bsg_parfbss_set_schurtype(_ObjId, _Schurtype, _Ncycle);
}
int ParFBSS_SetNcpuext(int _ObjId, int _NcpuExt) { return bsg_parfbss_set_ncpuext(_ObjId, _NcpuExt); }
int ParFBSS_SolveSymm(int _ObjId, int _Job, int *_NIterPerf) { return bsg_parfbss_solve_symm(_ObjId, _Job, _NIterPerf); }
int ParFBSS_Solve(int _ObjId, int _Job, int *_NIterPerf) { return bsg_parfbss_solve(_ObjId, _Job, _NIterPerf); }
int ParFBSS_Solution(int _ObjId, double **_Solution) { return bsg_parfbss_solution(_ObjId, _Solution); }
int ParFBSS_Distribution(int _ObjId, int *_NIOpt, int **_LISTOpt) {
	return bsg_parfbss_distribution(_ObjId, _NIOpt, _LISTOpt);
}
int ParFBSS_Destroy(int _ObjId) { return bsg_parfbss_destroy(_ObjId); }
