// Oracle build support (test infrastructure, not shipped): a generator behind
// Bslib's abstract-interface callbacks (Bslib/smatrix.h:14-20), in the role
// Bcmlib's BCM_draft plays for its drivers (Bcmlib/cdraft.h:777-933), and
// plain C entry points that run the reference's own AbstractSymmSolver /
// AbstractSolver (Bslib/solvers.cpp:5383, :5591) on it.
//
// The generator serves a block matrix given as block CSR (blocks column-major,
// block sizes sprnd), with the blocks of every block row handed out in a
// seeded shuffled column order, so a solver must sort them as the reference
// does; the pattern arrays are allocated with new[] because the solver
// releases them with delete[] (Bslib/solvers.cpp:5786-5788).  The same
// generator object and callbacks drive the GPU drop-ins in the tests.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <fstream>
#include <iostream>
#include <numeric>
#include <random>
#include <vector>
#include "smatrix.h"
#include "slvparam.h"
#include "svector.h"
#include "tree.h"

namespace {

struct Gen {
	int nsup = 0;
	std::vector<int> sprnd, ia, ja;     // shuffled column order inside each block row
	std::vector<long long> off;         // start of block k (shuffled order) in a
	std::vector<double> a, b, x0, sol;
	int calls[7] = {0, 0, 0, 0, 0, 0, 0};
};

void g_nsup(void *o, int &nsup) {
	Gen *g = static_cast<Gen *>(o);
	g->calls[0]++;
	nsup = g->nsup;
}
void g_sprnds(void *o, int *sprnds) {
	Gen *g = static_cast<Gen *>(o);
	g->calls[1]++;
	std::copy(g->sprnd.begin(), g->sprnd.end(), sprnds);
}
void g_iaja(void *o, int *&ia, int *&ja) {
	Gen *g = static_cast<Gen *>(o);
	g->calls[2]++;
	ia = new int[g->ia.size()];
	ja = new int[g->ja.size() > 0 ? g->ja.size() : 1];
	std::copy(g->ia.begin(), g->ia.end(), ia);
	std::copy(g->ja.begin(), g->ja.end(), ja);
}
void g_blockrow(void *o, int i, double *arow) {
	Gen *g = static_cast<Gen *>(o);
	g->calls[3]++;
	const int bi = g->sprnd[i + 1] - g->sprnd[i];
	size_t q = 0;
	for (int k = g->ia[i]; k < g->ia[i + 1]; k++) {
		const int j = g->ja[k];
		const size_t len = (size_t)bi * (g->sprnd[j + 1] - g->sprnd[j]);
		std::memcpy(arow + q, g->a.data() + g->off[k], sizeof(double) * len);
		q += len;
	}
}
void g_rhs(void *o, int i, double *b) {
	Gen *g = static_cast<Gen *>(o);
	g->calls[4]++;
	std::copy(g->b.begin() + g->sprnd[i], g->b.begin() + g->sprnd[i + 1], b);
}
void g_iniguess(void *o, int i, double *x) {
	Gen *g = static_cast<Gen *>(o);
	g->calls[5]++;
	std::copy(g->x0.begin() + g->sprnd[i], g->x0.begin() + g->sprnd[i + 1], x);
}
void g_storesol(void *o, int i, double *x) {
	Gen *g = static_cast<Gen *>(o);
	g->calls[6]++;
	std::copy(x, x + (g->sprnd[i + 1] - g->sprnd[i]), g->sol.begin() + g->sprnd[i]);
}

thread_local char g_err[256];

} // namespace

extern "C" {

// ia/ja/a: block CSR in any column order, blocks of row i one after another,
// each column-major (sprnd[i+1]-sprnd[i]) x (sprnd[j+1]-sprnd[j]).
void *ref_gen_create(int nsup, const int *sprnd, const int *ia, const int *ja, const double *a, const double *b,
                     const double *x0, unsigned seed) {
	Gen *g = new Gen();
	g->nsup = nsup;
	g->sprnd.assign(sprnd, sprnd + nsup + 1);
	const int n = sprnd[nsup];
	g->ia.assign(ia, ia + nsup + 1);
	g->ja.resize(ia[nsup]);
	g->off.resize(ia[nsup]);
	std::vector<long long> src(ia[nsup]);
	long long pos = 0;
	for (int i = 0; i < nsup; i++)
		for (int k = ia[i]; k < ia[i + 1]; k++) {
			src[k] = pos;
			pos += (long long)(sprnd[i + 1] - sprnd[i]) * (sprnd[ja[k] + 1] - sprnd[ja[k]]);
		}
	g->a.assign(a, a + pos);
	std::mt19937 rng(seed);
	for (int i = 0; i < nsup; i++) {
		std::vector<int> perm(ia[i + 1] - ia[i]);
		std::iota(perm.begin(), perm.end(), ia[i]);
		std::shuffle(perm.begin(), perm.end(), rng);
		for (size_t q = 0; q < perm.size(); q++) {
			g->ja[ia[i] + q] = ja[perm[q]];
			g->off[ia[i] + q] = src[perm[q]];
		}
	}
	g->b.assign(b, b + n);
	g->x0.assign(x0, x0 + n);
	g->sol.assign(n, 0.0);
	return g;
}

void ref_gen_free(void *o) { delete static_cast<Gen *>(o); }

void ref_gen_solution(void *o, double *x) {
	Gen *g = static_cast<Gen *>(o);
	std::copy(g->sol.begin(), g->sol.end(), x);
}

// how often each of the seven callbacks was called since creation
void ref_gen_calls(void *o, int *calls) { std::memcpy(calls, static_cast<Gen *>(o)->calls, sizeof(int) * 7); }

// the seven callbacks, in the order of the Abstract*Solver signatures
void ref_gen_fns(void **fns) {
	fns[0] = reinterpret_cast<void *>(&g_nsup);
	fns[1] = reinterpret_cast<void *>(&g_sprnds);
	fns[2] = reinterpret_cast<void *>(&g_iaja);
	fns[3] = reinterpret_cast<void *>(&g_blockrow);
	fns[4] = reinterpret_cast<void *>(&g_rhs);
	fns[5] = reinterpret_cast<void *>(&g_iniguess);
	fns[6] = reinterpret_cast<void *>(&g_storesol);
}

const char *ref_abstract_error() { return g_err; }

// The reference's AbstractSymmSolver (symm != 0) or AbstractSolver on the
// generator, natural ordering; out[0..3] = nitperf, resfin, density, wall s.
int ref_abstract(int symm, void *o, double tau1, double tau2, double theta, double memory, int ittype, int sttype,
                 double eps, int niter, double *out) {
	const std::ios::iostate cst = std::cout.rdstate();
	try {
		CSlvParam p;
		p.msglev = 0; p.ordtype = 0;
		p.tau1 = tau1; p.tau2 = tau2; p.theta = theta; p.memory = memory;
		p.ittype = ittype; p.sttype = sttype; p.eps = eps; p.niter = niter; p.ichk = 1;
		std::ofstream fout("/dev/null");
		// the block factorisations print statistics whatever msglev says
		fout.setstate(std::ios::badbit);
		std::cout.setstate(std::ios::badbit);
		auto t0 = std::chrono::steady_clock::now();
		if (symm)
			AbstractSymmSolver(o, fout, p, &g_nsup, &g_sprnds, &g_iaja, &g_blockrow, &g_rhs, &g_iniguess, &g_storesol);
		else
			AbstractSolver(o, fout, p, &g_nsup, &g_sprnds, &g_iaja, &g_blockrow, &g_rhs, &g_iniguess, &g_storesol);
		auto t1 = std::chrono::steady_clock::now();
		std::cout.clear(cst);
		if (out) {
			out[0] = p.nitperf; out[1] = p.resfin; out[2] = p.density;
			out[3] = std::chrono::duration<double>(t1 - t0).count();
		}
		return 0;
	} catch (const char *e) {
		std::cout.clear(cst);
		std::strncpy(g_err, e ? e : "unknown", sizeof(g_err) - 1);
		return -1;
	}
}

// The reference's callback Krylov loops on one rank (a CTree of one
// processor, as AbstractParSolver builds with nproc = 1): CSVector::Cg
// (Bslib/cg.cpp:355) and CSVector::BlockGMRES (Bslib/gmres.cpp:337), with the
// matrix and preconditioner operators given as CMVM / CSOLVELU function
// pointers and their objects.  x: initial guess in, solution out.
// stats[0..1] = iterations, wall seconds.
// The callback CG stops on sttype (0 absolute, 1 relative residual norm,
// Bslib/cg.cpp:605-612), not on ittype.
int ref_cg_tree(int n, const double *b, double *x, void *obja, void *mvm, void *objlu, void *solvelu, int sttype,
                double eps, int niter, double *stats) {
	const std::ios::iostate cst = std::cout.rdstate();
	try {
		CTree tree(1, 2);
		CSlvParam p;
		p.msglev = 0; p.sttype = sttype; p.eps = eps; p.niter = niter; p.ichk = 1;
		CSVector vb(n), vx(n), sol(n);
		std::memcpy(vb.GetVect(), b, sizeof(double) * n);
		std::memcpy(vx.GetVect(), x, sizeof(double) * n);
		std::ofstream fout("/dev/null");
		fout.setstate(std::ios::badbit);
		std::cout.setstate(std::ios::badbit);
		auto t0 = std::chrono::steady_clock::now();
		sol.Cg(fout, tree, obja, reinterpret_cast<CMVM>(mvm), objlu, reinterpret_cast<CSOLVELU>(solvelu), vx, vb, p);
		auto t1 = std::chrono::steady_clock::now();
		std::cout.clear(cst);
		std::memcpy(x, sol.GetVect(), sizeof(double) * n);
		if (stats) { stats[0] = p.nitperf; stats[1] = std::chrono::duration<double>(t1 - t0).count(); }
		return 0;
	} catch (const char *e) {
		std::cout.clear(cst);
		std::strncpy(g_err, e ? e : "unknown", sizeof(g_err) - 1);
		return -1;
	}
}

int ref_gmres_tree(int n, const double *b, double *x, void *obja, void *mvm, void *objlu, void *solvelu, int sttype,
                   double eps, int niter, double *stats) {
	const std::ios::iostate cst = std::cout.rdstate();
	try {
		CTree tree(1, 2);
		CSlvParam p;
		p.msglev = 0; p.sttype = sttype; p.eps = eps; p.niter = niter; p.ichk = 1; p.ooctyp = 0;
		CSVector vb(n), vx(n), sol(n);
		std::memcpy(vb.GetVect(), b, sizeof(double) * n);
		std::memcpy(vx.GetVect(), x, sizeof(double) * n);
		std::ofstream fout("/dev/null");
		fout.setstate(std::ios::badbit);
		std::cout.setstate(std::ios::badbit);
		auto t0 = std::chrono::steady_clock::now();
		sol.BlockGMRES(fout, p, tree, obja, reinterpret_cast<CMVM>(mvm), objlu, reinterpret_cast<CSOLVELU>(solvelu),
		               vx, vb);
		auto t1 = std::chrono::steady_clock::now();
		std::cout.clear(cst);
		std::memcpy(x, sol.GetVect(), sizeof(double) * n);
		if (stats) { stats[0] = p.nitperf; stats[1] = std::chrono::duration<double>(t1 - t0).count(); }
		return 0;
	} catch (const char *e) {
		std::cout.clear(cst);
		std::strncpy(g_err, e ? e : "unknown", sizeof(g_err) - 1);
		return -1;
	}
}

} // extern "C"
