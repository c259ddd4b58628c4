// Synthetic linear systems for the Bslib solver path: the seeded heat and
// Lame elasticity problems that the tests and the benchmark solve.
//
// The reference ships only analytic stencil generators (e.g. the 3-D 7-point
// CSMatrixR(nx,ny,nz,dshft,dunsy) constructor, Bslib/smatrixr.cpp:282-315);
// these generators produce the same storage layouts with physical
// coefficients:
//   * point CSR, 0-based, each row's diagonal entry first and the remaining
//     columns ascending (the "diagonal first" rule that Bslib/ich2r.cpp:182-190
//     relies on);
//   * 3x3 block CSR in the CSMatrixRS layout (Bslib/smatrix.h:1040-1048):
//     block j of the row list starts at a[9*j] and is stored column-major,
//     element (r,c) at a[9*j + 3*c + r]; the diagonal block comes first.
// Symmetric solvers want the upper triangle only (Bslib/mvm.cpp:2637-2652);
// bsgp_upper() extracts it.
//
// Random numbers: std::mt19937_64 with the problem's seed; a uniform double is
// (x >> 11) * 2^-53, a standard normal is Box-Muller on two such uniforms
// (cos branch only), lognormal(sigma) = exp(sigma * normal).  All values are
// drawn in cell / unknown order as documented per generator.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>
#include <algorithm>
#include <new>

namespace {

struct Rng {
	std::mt19937_64 g;
	explicit Rng(uint64_t seed) : g(seed) {}
	double uniform() { return (double)(g() >> 11) * 0x1.0p-53; }           // [0,1)
	double uniform_open() { return ((double)(g() >> 11) + 1.0) * 0x1.0p-53; } // (0,1]
	double normal() {
		double u1 = uniform_open(), u2 = uniform();
		return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
	}
	double lognormal(double sigma) { return std::exp(sigma * normal()); }
	double sym() { return 2.0 * uniform() - 1.0; } // [-1,1)
};

struct Problem {
	int n = 0;       // rows (point) or block rows (block)
	int bs = 1;      // block size
	int nrhs = 1;
	std::vector<int> ia, ja;
	std::vector<double> a;   // bs*bs per entry, column-major blocks
	std::vector<double> rhs; // n*bs*nrhs, right-hand side r stored at rhs[r*n*bs ...]
	std::vector<int> parts;  // independent sub-problem row offsets (batched problems)
	double info[8] = {0};    // generator-specific statistics
};

// Build CSR from per-row column maps (diagonal first, rest ascending).
struct RowBuilder {
	int n, bs;
	std::vector<std::vector<std::pair<int, int>>> rows; // (col, slot)
	std::vector<std::vector<double>> vals;
	RowBuilder(int n_, int bs_) : n(n_), bs(bs_), rows(n_), vals(n_) {}
	double *entry(int i, int j) {
		auto &r = rows[i];
		for (auto &p : r)
			if (p.first == j) return &vals[i][(size_t)p.second * bs * bs];
		int slot = (int)r.size();
		r.push_back({j, slot});
		vals[i].resize((size_t)(slot + 1) * bs * bs, 0.0);
		return &vals[i][(size_t)slot * bs * bs];
	}
	void finish(Problem &p) {
		p.n = n; p.bs = bs;
		p.ia.assign(n + 1, 0);
		for (int i = 0; i < n; i++) p.ia[i + 1] = p.ia[i] + (int)rows[i].size();
		p.ja.resize(p.ia[n]);
		p.a.resize((size_t)p.ia[n] * bs * bs);
		for (int i = 0; i < n; i++) {
			auto r = rows[i];
			std::sort(r.begin(), r.end(), [i](const std::pair<int, int> &x, const std::pair<int, int> &y) {
				if ((x.first == i) != (y.first == i)) return x.first == i;
				return x.first < y.first;
			});
			int k = p.ia[i];
			for (auto &e : r) {
				p.ja[k] = e.first;
				std::memcpy(&p.a[(size_t)k * bs * bs], &vals[i][(size_t)e.second * bs * bs], sizeof(double) * bs * bs);
				k++;
			}
			std::vector<std::pair<int, int>>().swap(rows[i]);
			std::vector<double>().swap(vals[i]);
		}
	}
};

inline double harmonic(double x, double y) { return 2.0 * x * y / (x + y); }

// Cell-centred finite-volume diffusion, -div(k grad u) = f with u = 0 on a
// ghost layer outside the box (h = 1): face conductance is the harmonic mean
// of the two cells, a boundary face contributes k_i to the diagonal.  With
// k == 1 this is the classic 7-point (5-point in 2-D) Laplacian, diagonal 6
// (4), off-diagonals -1.  Conductivities are drawn first (cell order
// x fastest), then the right-hand side uniform[-1,1] (same order).
void heat_grid(Problem &p, int nx, int ny, int nz, double sigma, Rng &rng, int row0,
               std::vector<int> &ia, std::vector<int> &ja, std::vector<double> &a, std::vector<double> &rhs) {
	const int n = nx * ny * nz;
	std::vector<double> k(n, 1.0);
	if (sigma > 0.0)
		for (int i = 0; i < n; i++) k[i] = rng.lognormal(sigma);
	auto id = [&](int x, int y, int z) { return x + nx * (y + ny * z); };
	for (int z = 0; z < nz; z++)
		for (int y = 0; y < ny; y++)
			for (int x = 0; x < nx; x++) {
				int i = id(x, y, z);
				double diag = 0.0;
				int nb[6];
				int cnt = 0;
				const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
				double off[6];
				for (int d = 0; d < 6; d++) {
					if (nz == 1 && d >= 4) continue;
					int xx = x + dx[d], yy = y + dy[d], zz = z + dz[d];
					if (xx < 0 || xx >= nx || yy < 0 || yy >= ny || zz < 0 || zz >= nz) {
						diag += k[i];
						continue;
					}
					int j = id(xx, yy, zz);
					double c = harmonic(k[i], k[j]);
					diag += c;
					nb[cnt] = j;
					off[cnt] = -c;
					cnt++;
				}
				// sort neighbours ascending
				for (int s = 1; s < cnt; s++)
					for (int t = s; t > 0 && nb[t - 1] > nb[t]; t--) {
						std::swap(nb[t - 1], nb[t]);
						std::swap(off[t - 1], off[t]);
					}
				ja.push_back(row0 + i);
				a.push_back(diag);
				for (int s = 0; s < cnt; s++) {
					ja.push_back(row0 + nb[s]);
					a.push_back(off[s]);
				}
				ia.push_back((int)ja.size());
			}
	for (int i = 0; i < n; i++) rhs.push_back(rng.sym());
	(void)p;
}

// ---- trilinear hexahedron (Q1) isotropic elasticity -----------------------
// Local node a = i + 2j + 4k at reference corner (2i-1, 2j-1, 2k-1).  The
// element matrix is integrated with the 2x2x2 Gauss rule; Voigt order
// (xx, yy, zz, yz, xz, xy) with engineering shear strains.
struct HexQ1 {
	double K[24][24];     // stiffness for E = 1, cube side h
	double F[6][24];      // -int B^T C e_m dV for the six unit macro strains, E = 1
	HexQ1(double nu, double h) {
		std::memset(K, 0, sizeof(K));
		std::memset(F, 0, sizeof(F));
		const double lam = nu / ((1 + nu) * (1 - 2 * nu)), mu = 1.0 / (2 * (1 + nu));
		double C[6][6] = {{0}};
		for (int r = 0; r < 3; r++)
			for (int c = 0; c < 3; c++) C[r][c] = lam + (r == c ? 2 * mu : 0.0);
		for (int r = 3; r < 6; r++) C[r][r] = mu;
		const double g = 1.0 / std::sqrt(3.0);
		const double detJ = (h / 2) * (h / 2) * (h / 2);
		for (int q = 0; q < 8; q++) {
			double xi = (q & 1 ? g : -g), eta = (q & 2 ? g : -g), ze = (q & 4 ? g : -g);
			double dN[8][3];
			for (int a = 0; a < 8; a++) {
				double xa = (a & 1) ? 1 : -1, ya = (a & 2) ? 1 : -1, za = (a & 4) ? 1 : -1;
				dN[a][0] = xa * (1 + eta * ya) * (1 + ze * za) / 8 * (2 / h);
				dN[a][1] = ya * (1 + xi * xa) * (1 + ze * za) / 8 * (2 / h);
				dN[a][2] = za * (1 + xi * xa) * (1 + eta * ya) / 8 * (2 / h);
			}
			double B[6][24] = {{0}};
			for (int a = 0; a < 8; a++) {
				B[0][3 * a + 0] = dN[a][0];
				B[1][3 * a + 1] = dN[a][1];
				B[2][3 * a + 2] = dN[a][2];
				B[3][3 * a + 1] = dN[a][2]; B[3][3 * a + 2] = dN[a][1];
				B[4][3 * a + 0] = dN[a][2]; B[4][3 * a + 2] = dN[a][0];
				B[5][3 * a + 0] = dN[a][1]; B[5][3 * a + 1] = dN[a][0];
			}
			double CB[6][24];
			for (int r = 0; r < 6; r++)
				for (int c = 0; c < 24; c++) {
					double s = 0;
					for (int t = 0; t < 6; t++) s += C[r][t] * B[t][c];
					CB[r][c] = s;
				}
			for (int r = 0; r < 24; r++)
				for (int c = 0; c < 24; c++) {
					double s = 0;
					for (int t = 0; t < 6; t++) s += B[t][r] * CB[t][c];
					K[r][c] += s * detJ;
				}
			for (int m = 0; m < 6; m++)
				for (int r = 0; r < 24; r++) F[m][r] -= CB[m][r] * detJ; // (B^T C e_m)_r = (C B)_{m r}
		}
	}
};

void lame_assemble(Problem &p, int nn, bool periodic, double nu, const std::vector<double> &E,
                   const std::vector<char> &fixed, int nload, bool body_load) {
	const int nc = periodic ? nn : nn - 1;
	const double h = 1.0 / nc;
	HexQ1 el(nu, h);
	const int nnode = nn * nn * nn;
	RowBuilder rb(nnode, 3);
	p.nrhs = nload;
	p.rhs.assign((size_t)nnode * 3 * nload, 0.0);
	auto node = [&](int x, int y, int z) {
		if (periodic) { x %= nn; y %= nn; z %= nn; }
		return x + nn * (y + nn * z);
	};
	for (int cz = 0; cz < nc; cz++)
		for (int cy = 0; cy < nc; cy++)
			for (int cx = 0; cx < nc; cx++) {
				int cell = cx + nc * (cy + nc * cz);
				double e = E[cell];
				int g[8];
				for (int a = 0; a < 8; a++) g[a] = node(cx + (a & 1), cy + ((a >> 1) & 1), cz + ((a >> 2) & 1));
				for (int a = 0; a < 8; a++) {
					if (fixed[g[a]]) continue;
					for (int b = 0; b < 8; b++) {
						if (fixed[g[b]]) continue;
						double *blk = rb.entry(g[a], g[b]);
						for (int r = 0; r < 3; r++)
							for (int c = 0; c < 3; c++) blk[3 * c + r] += e * el.K[3 * a + r][3 * b + c];
					}
					for (int m = 0; m < nload; m++) {
						double *f = &p.rhs[(size_t)m * nnode * 3 + (size_t)g[a] * 3];
						if (body_load) {
							f[2] += -h * h * h / 8.0; // unit body force (0,0,-1), consistent Q1 load
						} else {
							for (int r = 0; r < 3; r++) f[r] += e * el.F[m][3 * a + r];
						}
					}
				}
			}
	for (int i = 0; i < nnode; i++)
		if (fixed[i]) {
			double *blk = rb.entry(i, i);
			blk[0] = blk[4] = blk[8] = 1.0;
		}
	rb.finish(p);
}

} // namespace

extern "C" {

// Opaque generated problem.  All arrays stay owned by the handle.
typedef struct bsgp_problem bsgp_problem;

// 3-D heat on an nx*ny*nz cell grid (7-point), conductivity lognormal(sigma)
// per cell (sigma == 0: unit conductivity), RHS uniform[-1,1].
bsgp_problem *bsgp_heat3d(int nx, int ny, int nz, double sigma, unsigned long long seed) {
	Problem *p = new (std::nothrow) Problem();
	if (!p) return nullptr;
	Rng rng(seed);
	p->ia.push_back(0);
	heat_grid(*p, nx, ny, nz, sigma, rng, 0, p->ia, p->ja, p->a, p->rhs);
	p->n = nx * ny * nz;
	p->parts = {0, p->n};
	return (bsgp_problem *)p;
}

// nprob independent 2-D heat problems (5-point) on square grids whose side is
// log-uniform in [smin, smax] (rounded), conductivity lognormal(sigma) per
// cell, RHS uniform[-1,1].  Draw order: all sides, then per problem the
// conductivities and the right-hand side.  The problems are concatenated as
// one block-diagonal CSR; parts[] holds the row offsets.
bsgp_problem *bsgp_heat2d_batch(int nprob, int smin, int smax, double sigma, unsigned long long seed) {
	Problem *p = new (std::nothrow) Problem();
	if (!p) return nullptr;
	Rng rng(seed);
	std::vector<int> side(nprob);
	const double l0 = std::log((double)smin), l1 = std::log((double)smax);
	for (int q = 0; q < nprob; q++) side[q] = (int)std::floor(std::exp(l0 + rng.uniform() * (l1 - l0)) + 0.5);
	p->ia.push_back(0);
	p->parts.push_back(0);
	int row0 = 0;
	for (int q = 0; q < nprob; q++) {
		heat_grid(*p, side[q], side[q], 1, sigma, rng, row0, p->ia, p->ja, p->a, p->rhs);
		row0 += side[q] * side[q];
		p->parts.push_back(row0);
	}
	p->n = row0;
	return (bsgp_problem *)p;
}

// 3-D Lame elasticity, Q1 hexahedra on an nn^3 node grid over the unit cube,
// Poisson ratio nu, Young's modulus lognormal(sigma) per cell (cell order),
// nodes on the z = 0 face clamped (identity block rows, couplings removed),
// unit body load (0,0,-1).  3x3 block CSR, one right-hand side.
bsgp_problem *bsgp_lame3d(int nn, double nu, double sigma, unsigned long long seed) {
	Problem *p = new (std::nothrow) Problem();
	if (!p) return nullptr;
	Rng rng(seed);
	const int nc = nn - 1;
	std::vector<double> E((size_t)nc * nc * nc);
	for (auto &e : E) e = rng.lognormal(sigma);
	std::vector<char> fixed((size_t)nn * nn * nn, 0);
	for (int i = 0; i < nn * nn; i++) fixed[i] = 1; // z == 0 layer
	lame_assemble(*p, nn, false, nu, E, fixed, 1, true);
	p->parts = {0, p->n};
	return (bsgp_problem *)p;
}

// Periodic homogenisation cell: Q1 Lame on an nn^3 periodic node grid (nn^3
// cells), spherical inclusions with radius uniform in [rmin, rmax] cells,
// centres uniform in the cell, non-overlapping in the periodic metric, added
// until the inclusion cell fraction reaches volfrac (or 200000 attempts).
// Young's modulus 1 in the matrix and `contrast` in inclusions, Poisson ratio
// nu.  Node 0 is pinned (identity block row) to remove the rigid translations.
// Six right-hand sides: the unit macro strains in Voigt order.
// info[0] = achieved inclusion fraction, info[1] = number of spheres.
bsgp_problem *bsgp_lame_periodic(int nn, double nu, double rmin, double rmax, double volfrac, double contrast,
                                 unsigned long long seed) {
	Problem *p = new (std::nothrow) Problem();
	if (!p) return nullptr;
	Rng rng(seed);
	struct Sph { double x, y, z, r; };
	std::vector<Sph> sph;
	const int nc = nn;
	std::vector<char> inc((size_t)nc * nc * nc, 0);
	size_t ninc = 0;
	auto pd = [nn](double d) { d = std::fabs(d); return std::min(d, nn - d); };
	for (int attempt = 0; attempt < 200000 && (double)ninc < volfrac * inc.size(); attempt++) {
		Sph s{rng.uniform() * nn, rng.uniform() * nn, rng.uniform() * nn, rmin + rng.uniform() * (rmax - rmin)};
		bool ok = true;
		for (auto &t : sph) {
			double dx = pd(s.x - t.x), dy = pd(s.y - t.y), dz = pd(s.z - t.z);
			if (dx * dx + dy * dy + dz * dz < (s.r + t.r) * (s.r + t.r)) { ok = false; break; }
		}
		if (!ok) continue;
		sph.push_back(s);
		int r = (int)std::ceil(s.r) + 1;
		for (int dz = -r; dz <= r; dz++)
			for (int dy = -r; dy <= r; dy++)
				for (int dx = -r; dx <= r; dx++) {
					int cx = ((int)std::floor(s.x) + dx + nn) % nn, cy = ((int)std::floor(s.y) + dy + nn) % nn,
					    cz = ((int)std::floor(s.z) + dz + nn) % nn;
					double ex = pd(cx + 0.5 - s.x), ey = pd(cy + 0.5 - s.y), ez = pd(cz + 0.5 - s.z);
					if (ex * ex + ey * ey + ez * ez <= s.r * s.r) {
						size_t c = cx + (size_t)nn * (cy + (size_t)nn * cz);
						if (!inc[c]) { inc[c] = 1; ninc++; }
					}
				}
	}
	std::vector<double> E(inc.size());
	for (size_t c = 0; c < inc.size(); c++) E[c] = inc[c] ? contrast : 1.0;
	std::vector<char> fixed((size_t)nn * nn * nn, 0);
	fixed[0] = 1;
	lame_assemble(*p, nn, true, nu, E, fixed, 6, false);
	p->parts = {0, p->n};
	p->info[0] = (double)ninc / (double)inc.size();
	p->info[1] = (double)sph.size();
	return (bsgp_problem *)p;
}

void bsgp_free(bsgp_problem *h) { delete (Problem *)h; }

// Sizes: n (rows or block rows), block size, nonzero entries (blocks),
// right-hand sides, number of independent parts.
void bsgp_sizes(const bsgp_problem *h, int *n, int *bs, int *nnz, int *nrhs, int *nparts) {
	const Problem *p = (const Problem *)h;
	if (n) *n = p->n;
	if (bs) *bs = p->bs;
	if (nnz) *nnz = p->ia.empty() ? 0 : p->ia[p->n];
	if (nrhs) *nrhs = p->nrhs;
	if (nparts) *nparts = (int)p->parts.size() - 1;
}
const int *bsgp_ia(const bsgp_problem *h) { return ((const Problem *)h)->ia.data(); }
const int *bsgp_ja(const bsgp_problem *h) { return ((const Problem *)h)->ja.data(); }
const double *bsgp_a(const bsgp_problem *h) { return ((const Problem *)h)->a.data(); }
const double *bsgp_rhs(const bsgp_problem *h) { return ((const Problem *)h)->rhs.data(); }
const int *bsgp_parts(const bsgp_problem *h) { return ((const Problem *)h)->parts.data(); }
double bsgp_info(const bsgp_problem *h, int k) { return (k >= 0 && k < 8) ? ((const Problem *)h)->info[k] : 0.0; }

} // extern "C"
