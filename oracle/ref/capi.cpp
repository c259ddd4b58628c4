// Oracle build support (test infrastructure, not shipped): plain C entry
// points over the reference Bslib classes, so the parity tests can drive the
// reference's own code on identical inputs through ctypes.
//
// Matrices cross this boundary as 0-based CSR arrays (ia[n+1], ja[nz], a[nz]),
// each row's diagonal entry first, which is the layout CSMatrixR keeps
// (Bslib/smatrix.h:540-546).  Factor results are returned in malloc'ed arrays
// that the caller releases with ref_free().
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <chrono>
#include "smatrix.h"
#include "slvparam.h"
#include "svector.h"

namespace {

CSMatrixR make_csr(int n, const int *ia, const int *ja, const double *a) {
	int nz = ia[n];
	CSMatrixR m(n, nz);
	std::memcpy(m.GetIa(), ia, sizeof(int) * (n + 1));
	std::memcpy(m.GetJa(), ja, sizeof(int) * nz);
	std::memcpy(m.GetA(), a, sizeof(double) * nz);
	m.SetNza(nz);
	m.SetNzatot(nz);
	return m;
}

void export_csr(const CSMatrixR &m, int **ia, int **ja, double **a) {
	int n = m.GetNlist();
	int nz = m.GetIa()[n];
	*ia = (int *)std::malloc(sizeof(int) * (n + 1));
	*ja = (int *)std::malloc(sizeof(int) * (nz > 0 ? nz : 1));
	*a = (double *)std::malloc(sizeof(double) * (nz > 0 ? nz : 1));
	std::memcpy(*ia, m.GetIa(), sizeof(int) * (n + 1));
	std::memcpy(*ja, m.GetJa(), sizeof(int) * nz);
	std::memcpy(*a, m.GetA(), sizeof(double) * nz);
}

CSVector make_vec(int n, const double *x) {
	CSVector v(n);
	if (x) std::memcpy(v.GetVect(), x, sizeof(double) * n);
	return v;
}

double now_s() {
	using namespace std::chrono;
	return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// The reference prints to cout in places whatever msglev says, and formatting
// numbers through its streams crashes inside a Python process: calls that
// print keep cout in a failed state meanwhile.
struct QuietCout {
	std::ios::iostate st = std::cout.rdstate();
	QuietCout() { std::cout.setstate(std::ios::badbit); }
	~QuietCout() { std::cout.clear(st); }
};

// Error convention: the reference throws const char*; map it to a negative code
// and keep the message for ref_last_error().
thread_local char g_err[256];
int fail(const char *msg) {
	std::strncpy(g_err, msg ? msg : "unknown", sizeof(g_err) - 1);
	return -1;
}

// Block CSR (CSMatrixRS, Bslib/smatrix.h:1040-1048) with a uniform block
// size: blocks column-major, block k of the arrays at a[k * bs * bs].  The
// reference keeps the partition in protected members, so a derived type
// fills them.
struct RSBuild : public CSMatrixRS {
	RSBuild(int nsup, int bs, const int *ia_, const int *ja_, const double *a_)
	    : CSMatrixRS(nsup, ia_[nsup], ia_[nsup] * bs * bs) {
		const int nzj = ia_[nsup], nz = nzj * bs * bs;
		m = n = nsup * bs;
		nsupr = nsupc = nsup;
		nlist = nsup;
		nzja = nzj;
		nza = nzatot = nz;
		blamx = bs;
		for (int i = 0; i < nsup; i++) list[i] = i;
		std::memcpy(ia, ia_, sizeof(int) * (nsup + 1));
		std::memcpy(ja, ja_, sizeof(int) * nzj);
		std::memcpy(a, a_, sizeof(double) * nz);
		for (int j = 0; j < nzj; j++) bsa[j] = j * bs * bs;
		for (int i = 0; i <= nsup; i++) sprndr[i] = sprndc[i] = i * bs;
	}
	// block CSR of any CSMatrixRS with a uniform block size, blocks in row order
	static void export_rs(const CSMatrixRS &m, int bs, int **ia_o, int **ja_o, double **a_o) {
		CSMatrixRS &mm = const_cast<CSMatrixRS &>(m);
		const int nsup = mm.GetNsupr();
		const int *ia = mm.GetIa(), *ja = mm.GetJa(), *bsa = mm.GetBsa();
		const double *a = mm.GetA();
		const int nzj = ia[nsup], b2 = bs * bs;
		*ia_o = (int *)std::malloc(sizeof(int) * (nsup + 1));
		*ja_o = (int *)std::malloc(sizeof(int) * (nzj > 0 ? nzj : 1));
		*a_o = (double *)std::malloc(sizeof(double) * (nzj > 0 ? nzj * b2 : 1));
		std::memcpy(*ia_o, ia, sizeof(int) * (nsup + 1));
		std::memcpy(*ja_o, ja, sizeof(int) * nzj);
		for (int j = 0; j < nzj; j++) std::memcpy(*a_o + (size_t)j * b2, a + bsa[j], sizeof(double) * b2);
	}
};

} // namespace

extern "C" {

const char *ref_last_error() { return g_err; }
void ref_free(void *p) { std::free(p); }

// y = A x with A stored in full (MvmA, Bslib/mvm.cpp:2489) or symmetric
// upper-only (MvmASymm, Bslib/mvm.cpp:2637) form.
int ref_mvm(int n, const int *ia, const int *ja, const double *a, const double *x, double *y, int symm_upper) {
	CSMatrixR m = make_csr(n, ia, ja, a);
	CSVector vx = make_vec(n, x), vy(n);
	if (symm_upper) m.MvmASymm(vx, vy); else m.MvmA(vx, vy);
	std::memcpy(y, vy.GetVect(), sizeof(double) * n);
	return 0;
}

// Triangular solves with a factor in the reference layout
// (SolveL: L by columns, Bslib/mvm.cpp:3042; SolveU: U by rows, :3343).
int ref_solve_l(int n, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	CSMatrixR m = make_csr(n, ia, ja, a);
	CSVector vx = make_vec(n, x), vy(n);
	m.SolveL(vx, vy);
	std::memcpy(y, vy.GetVect(), sizeof(double) * n);
	return 0;
}
int ref_solve_u(int n, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	CSMatrixR m = make_csr(n, ia, ja, a);
	CSVector vx = make_vec(n, x), vy(n);
	m.SolveU(vx, vy);
	std::memcpy(y, vy.GetVect(), sizeof(double) * n);
	return 0;
}

// IC2 of an upper-stored SPD matrix (CSMatrixR::Ich2, Bslib/ich2r.cpp:956).
// stats[0]=density, stats[1]=density2, stats[2]=factor seconds.
int ref_ich2(int n, const int *ia, const int *ja, const double *a, double tau1, double tau2, double theta,
             double memory, int **ia_u, int **ja_u, double **a_u, double *stats) {
	try {
		CSMatrixR m = make_csr(n, ia, ja, a);
		CSlvParam p;
		p.msglev = 0; p.tau1 = tau1; p.tau2 = tau2; p.theta = theta; p.memory = memory;
		double t0 = now_s();
		CSMatrixR u = m.Ich2(p);
		double t1 = now_s();
		export_csr(u, ia_u, ja_u, a_u);
		if (stats) { stats[0] = p.density; stats[1] = p.density2; stats[2] = t1 - t0; }
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

// CombineLU + ILU2 of a full-stored matrix (Bslib/smatrixr.cpp:1142,
// Bslib/ilu2r.cpp:1122).  L comes back by columns, U by rows, same pattern.
int ref_ilu2(int n, const int *ia, const int *ja, const double *a, double tau1, double tau2, double theta,
             double memory, double sclmin, double pivmin,
             int **ia_l, int **ja_l, double **a_l, int **ia_u, int **ja_u, double **a_u, double *stats) {
	try {
		CSMatrixR m = make_csr(n, ia, ja, a);
		CSlvParam p;
		p.msglev = 0; p.tau1 = tau1; p.tau2 = tau2; p.theta = theta; p.memory = memory;
		p.sclmin = sclmin; p.pivmin = pivmin;
		CSMatrixR al, au, l, u, dummy;
		m.CombineLU(al, au);
		std::ofstream fout("/dev/null");
		double t0 = now_s();
		dummy.Ilu2(fout, p, al, au, l, u);
		double t1 = now_s();
		export_csr(l, ia_l, ja_l, a_l);
		export_csr(u, ia_u, ja_u, a_u);
		if (stats) { stats[0] = p.density; stats[1] = p.density2; stats[2] = t1 - t0; }
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

// Whole symmetric driver CSVector::SolveSymm(CSMatrixR&) (Bslib/solvers.cpp:4615)
// with natural ordering: IC2 (fcttyp != 1) or IC(0) (fcttyp == 1), then PCG
// (Bslib/cg.cpp:31).  stats: [0]=iterations, [1]=resfin, [2]=factor s,
// [3]=iteration s, [4]=density, [5]=density2, [6]=total wall s.
int ref_solve_symm(int n, const int *ia, const int *ja, const double *a, const double *b, double *x,
                   int fcttyp, double tau1, double tau2, double theta, double memory,
                   int ittype, double eps, int niter, int ichk, double *stats) {
	QuietCout quiet; // CSMatrixR::Ich (fcttyp 1) prints its size and time
	try {
		CSMatrixR m = make_csr(n, ia, ja, a);
		CSlvParam p;
		p.msglev = 0; p.fcttyp = fcttyp; p.ordtype = 0;
		p.tau1 = tau1; p.tau2 = tau2; p.theta = theta; p.memory = memory;
		p.ittype = ittype; p.eps = eps; p.niter = niter; p.ichk = ichk;
		CSVector vb = make_vec(n, b), norm(n), sol(n);
		norm.SetSVect(1.0);
		std::ofstream fout("/dev/null");
		double t0 = now_s();
		sol.SolveSymm(fout, m, vb, p, norm);
		double t1 = now_s();
		std::memcpy(x, sol.GetVect(), sizeof(double) * n);
		if (stats) {
			stats[0] = p.nitperf; stats[1] = p.resfin; stats[2] = p.timefct; stats[3] = p.timeitr;
			stats[4] = p.density; stats[5] = p.density2; stats[6] = t1 - t0;
		}
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

// PCG alone (Bslib/cg.cpp:31) with a given upper-stored A and IC factor U.
int ref_cg(int n, const int *ia, const int *ja, const double *a,
           const int *iu, const int *ju, const double *u, const double *b, double *x,
           int ittype, double eps, int niter, int ichk, double *stats) {
	try {
		CSMatrixR m = make_csr(n, ia, ja, a);
		CSMatrixR f = make_csr(n, iu, ju, u);
		CSlvParam p;
		p.msglev = 0; p.ittype = ittype; p.eps = eps; p.niter = niter; p.ichk = ichk;
		CSVector vb = make_vec(n, b), x0(n), norm(n), sol(n);
		norm.SetSVect(1.0);
		std::ofstream fout("/dev/null");
		double t0 = now_s();
		sol.Cg(fout, &m, 0, nullptr, &f, x0, vb, p, norm);
		double t1 = now_s();
		std::memcpy(x, sol.GetVect(), sizeof(double) * n);
		if (stats) { stats[0] = p.nitperf; stats[1] = p.resfin; stats[2] = t1 - t0; }
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

// Whole nonsymmetric driver CSVector::Solver(CSMatrixR&) (Bslib/solvers.cpp:1339):
// CombineLU + ILU2 + preconditioned Lanczos (Bslib/lanczos.cpp:34), natural
// ordering.  stats as ref_solve_symm.
int ref_solver(int n, const int *ia, const int *ja, const double *a, const double *b, double *x,
               double tau1, double tau2, double theta, double memory, double sclmin, double pivmin,
               int sttype, double eps, int niter, int ichk, double *stats) {
	try {
		CSMatrixR m = make_csr(n, ia, ja, a);
		CSlvParam p;
		p.msglev = 0; p.ordtype = 0; p.ittype = 1;
		p.tau1 = tau1; p.tau2 = tau2; p.theta = theta; p.memory = memory;
		p.sclmin = sclmin; p.pivmin = pivmin;
		p.sttype = sttype; p.eps = eps; p.niter = niter; p.ichk = ichk;
		CSVector vb = make_vec(n, b), norm(n), sol(n);
		norm.SetSVect(1.0);
		std::ofstream fout("/dev/null");
		double t0 = now_s();
		sol.Solver(fout, m, vb, p, norm);
		double t1 = now_s();
		std::memcpy(x, sol.GetVect(), sizeof(double) * n);
		if (stats) {
			stats[0] = p.nitperf; stats[1] = p.resfin; stats[2] = p.timefct; stats[3] = p.timeitr;
			stats[4] = p.density; stats[5] = p.density2; stats[6] = t1 - t0;
		}
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

// CombineLU of a block matrix (Bslib/smatrixrs.cpp:1645): upper blocks as
// they are, lower blocks transposed, both patterns extended to their union.
int ref_combine_lu_block(int nsup, int bs, const int *ia, const int *ja, const double *a, int **ia_s, int **ja_s,
                         double **al, double **au) {
	try {
		RSBuild m(nsup, bs, ia, ja, a);
		CSMatrixRS l, u;
		m.CombineLU(l, u);
		int *ial, *jal;
		RSBuild::export_rs(l, bs, &ial, &jal, al);
		RSBuild::export_rs(u, bs, ia_s, ja_s, au);
		std::free(ial);
		std::free(jal);
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

// CombineLU + block ILU2 (Bslib/ilu2rs.cpp:1458) of a full-stored block
// matrix; L and U come back with the same pattern (diagonal block first).
int ref_ilu2_block(int nsup, int bs, const int *ia, const int *ja, const double *a, double tau1, double tau2,
                   double theta, double memory, double sclmin, double pivmin, int **ia_f, int **ja_f, double **a_l,
                   double **a_u, double *stats) {
	try {
		RSBuild m(nsup, bs, ia, ja, a);
		CSlvParam p;
		p.msglev = 0; p.tau1 = tau1; p.tau2 = tau2; p.theta = theta; p.memory = memory;
		p.sclmin = sclmin; p.pivmin = pivmin;
		CSMatrixRS al, au, l, u, dummy;
		m.CombineLU(al, au);
		std::ofstream fout("/dev/null");
		double t0 = now_s();
		dummy.Ilu2(fout, p, al, au, l, u);
		double t1 = now_s();
		int *ial, *jal;
		RSBuild::export_rs(l, bs, &ial, &jal, a_l);
		RSBuild::export_rs(u, bs, ia_f, ja_f, a_u);
		std::free(ial);
		std::free(jal);
		if (stats) { stats[0] = p.density; stats[1] = p.density2; stats[2] = t1 - t0; }
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

// Block triangular solves with a block factor (CSMatrixRS::SolveL,
// Bslib/mvm.cpp:3140; SolveU, :3410).
int ref_solve_l_block(int nsup, int bs, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	RSBuild m(nsup, bs, ia, ja, a);
	CSVector vx = make_vec(nsup * bs, x), vy(nsup * bs);
	m.SolveL(vx, vy);
	std::memcpy(y, vy.GetVect(), sizeof(double) * nsup * bs);
	return 0;
}
int ref_solve_u_block(int nsup, int bs, const int *ia, const int *ja, const double *a, const double *x, double *y) {
	RSBuild m(nsup, bs, ia, ja, a);
	CSVector vx = make_vec(nsup * bs, x), vy(nsup * bs);
	m.SolveU(vx, vy);
	std::memcpy(y, vy.GetVect(), sizeof(double) * nsup * bs);
	return 0;
}

// Block IC2 (CSMatrixRS::Ich2, Bslib/ich2rs.cpp:1075) of an upper-stored
// symmetric block matrix; U comes back (L = U^T).
int ref_ich2_block(int nsup, int bs, const int *ia, const int *ja, const double *a, double tau1, double tau2,
                   double theta, double memory, int **ia_f, int **ja_f, double **a_u, double *stats) {
	try {
		RSBuild m(nsup, bs, ia, ja, a);
		CSlvParam p;
		p.msglev = 0; p.tau1 = tau1; p.tau2 = tau2; p.theta = theta; p.memory = memory;
		std::ofstream fout("/dev/null");
		// CSMatrixRS::Ich2 prints its histograms and statistics to cout and to
		// the log stream whatever msglev says (Bslib/ich2rs.cpp:244-245,
		// :1276-1297); failed streams format nothing
		fout.setstate(std::ios::badbit);
		const std::ios::iostate cst = std::cout.rdstate();
		std::cout.setstate(std::ios::badbit);
		double t0 = now_s();
		CSMatrixRS u;
		try {
			u = m.Ich2(fout, p);
		} catch (...) {
			std::cout.clear(cst);
			throw;
		}
		double t1 = now_s();
		std::cout.clear(cst);
		RSBuild::export_rs(u, bs, ia_f, ja_f, a_u);
		if (stats) { stats[0] = p.density; stats[1] = p.density2; stats[2] = t1 - t0; }
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

// Whole symmetric block driver CSVector::SolveSymm(CSMatrixRS&)
// (Bslib/solvers.cpp:4452) with natural ordering: block IC2, then PCG, one
// right-hand side per call as the reference takes them (Bslib/cg.cpp:375-377);
// nrhs load cases solved one after another from x = 0.  a: upper-stored
// blocks, column-major.  stats[4 * k + 0..3] per case: iterations, resfin,
// wall seconds, density.
int ref_solve_symm_block(int nsup, int bs, const int *ia, const int *ja, const double *a, int nrhs, const double *b,
                         double *x, double tau1, double tau2, double theta, double memory, int ittype, double eps,
                         int niter, double *stats) {
	const std::ios::iostate cst = std::cout.rdstate();
	try {
		const int n = nsup * bs;
		std::ofstream fout("/dev/null");
		fout.setstate(std::ios::badbit);
		std::cout.setstate(std::ios::badbit);
		for (int k = 0; k < nrhs; k++) {
			RSBuild m(nsup, bs, ia, ja, a);
			CSlvParam p;
			p.msglev = 0; p.ordtype = 0;
			p.tau1 = tau1; p.tau2 = tau2; p.theta = theta; p.memory = memory;
			p.ittype = ittype; p.eps = eps; p.niter = niter; p.ichk = 1;
			CSVector vb = make_vec(n, b + (size_t)k * n), norm(n), sol(n);
			norm.SetSVect(1.0);
			sol.SetSVect(0.0);
			double t0 = now_s();
			sol.SolveSymm(fout, m, vb, p, norm);
			double t1 = now_s();
			std::memcpy(x + (size_t)k * n, sol.GetVect(), sizeof(double) * n);
			if (stats) {
				stats[4 * k + 0] = p.nitperf; stats[4 * k + 1] = p.resfin; stats[4 * k + 2] = t1 - t0;
				stats[4 * k + 3] = p.density;
			}
		}
		std::cout.clear(cst);
		return 0;
	} catch (const char *e) {
		std::cout.clear(cst);
		return fail(e);
	}
}

// ---- files in the reference's own formats (CSMatrixR::WriteMtrBin / ReadMtrBin,
// Bslib/smatrixr.cpp:3984 / :3852; CSVector::WriteVectBin / ReadVectBin,
// Bslib/svector.cpp:537 / :488; CSMatrixR::ConvertToBinary, :4010).  They print
// to cout; the harness silences it around the calls.

int ref_write_mtr_bin(const char *path, int n, const int *ia, const int *ja, const double *a) {
	QuietCout q;
	CSMatrixR m = make_csr(n, ia, ja, a);
	std::ofstream f(path, std::ios::binary | std::ios::trunc);
	m.WriteMtrBin(f);
	return f ? 0 : fail("write failed");
}

int ref_write_vect_bin(const char *path, int append, int n, const double *v) {
	QuietCout q;
	CSVector vv = make_vec(n, v);
	std::ofstream f(path, std::ios::binary | (append ? std::ios::app : std::ios::trunc));
	vv.WriteVectBin(f);
	return f ? 0 : fail("write failed");
}

// A binary file holding a matrix and then nvec vectors, read with the
// reference's readers: ia / ja / a are malloc'ed (ref_free), vectors go to
// vecs (nvec * n values, n the matrix size).
int ref_read_system_bin(const char *path, int nvec, int *n_out, int **ia, int **ja, double **a, double *vecs) {
	QuietCout q;
	try {
		std::ifstream f(path, std::ios::binary);
		CSMatrixR m = CSMatrixR::ReadMtrBin(f);
		export_csr(m, ia, ja, a);
		const int n = m.GetNlist();
		*n_out = n;
		CSVector dummy;
		for (int k = 0; k < nvec; k++) {
			CSVector v = dummy.ReadVectBin(f);
			if (vecs) std::memcpy(vecs + (size_t)k * n, v.GetVect(), sizeof(double) * n);
		}
		return f ? 0 : fail("read failed");
	} catch (const char *e) {
		return fail(e);
	}
}

// Block Lanczos of the CSMatrixRS driver (CSVector::BlockLanczosCentral /
// BlockLanczosRight / BlockLanczosLeft, Bslib/lanczos.cpp:2467 / :932 / :1719)
// as CSVector::Solver(CSMatrixRS&) runs them (Bslib/solvers.cpp:1651-1800):
// CombineLU + block ILU2 of a block matrix with uniform block size bs, then
// the variant of ittype (2 central, 3 right, 4 left) on the nrhs columns of B
// at once, x0 = 0.  stats: [0] = wall seconds.
int ref_block_lanczos(int nsup, int bs, const int *ia, const int *ja, const double *a, int ittype, int nrhs,
                      const double *B, double *X, double tau1, double tau2, double theta, double eps, int niter,
                      int ichk, double *stats) {
	QuietCout q;
	try {
		RSBuild m(nsup, bs, ia, ja, a);
		CSlvParam p;
		p.msglev = 0; p.tau1 = tau1; p.tau2 = tau2; p.theta = theta; p.memory = 20.0;
		p.ittype = ittype; p.eps = eps; p.niter = niter; p.ichk = ichk;
		CSMatrixRS al, au, l, u, dummy;
		m.CombineLU(al, au);
		std::ofstream fout("/dev/null");
		fout.setstate(std::ios::badbit);
		dummy.Ilu2(fout, p, al, au, l, u);
		const int n = nsup * bs;
		CSVector vb(n, 1, nrhs), vx(n, 1, nrhs), sol(n, 1, nrhs);
		std::memcpy(vb.GetVect(), B, sizeof(double) * n * nrhs);
		vx.SetSVect(0.0);
		double t0 = now_s();
		if (ittype == 2) sol.BlockLanczosCentral(fout, &m, &l, &u, vx, vb, p);
		else if (ittype == 3) sol.BlockLanczosRight(fout, &m, &l, &u, vx, vb, p);
		else sol.BlockLanczosLeft(fout, &m, &l, &u, vx, vb, p);
		double t1 = now_s();
		std::memcpy(X, sol.GetVect(), sizeof(double) * n * nrhs);
		if (stats) stats[0] = t1 - t0;
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

// IC(0) of an upper-stored SPD matrix (CSMatrixR::Ich, Bslib/ich2r.cpp:1821):
// U by rows, inverse pivots first.
int ref_ich0(int n, const int *ia, const int *ja, const double *a, int **ia_u, int **ja_u, double **a_u) {
	QuietCout q;
	try {
		CSMatrixR m = make_csr(n, ia, ja, a);
		CSMatrixR u = m.Ich();
		export_csr(u, ia_u, ja_u, a_u);
		return 0;
	} catch (const char *e) {
		return fail(e);
	}
}

} // extern "C"
