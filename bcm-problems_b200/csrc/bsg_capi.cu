// C ABI of libbsg.so (declared in include/bslib_gpu.h): contexts, device
// matrices and factors, and the host-buffer drivers that stand in for
// CSVector::SolveSymm / CSVector::Solver.
#include "bsg_internal.cuh"
#include <cstdio>
#include <cstring>
#include <cmath>
#include <new>
#include <vector>
#include <algorithm>

// The host entry points' CSR checks on device copies, with their messages and
// order (k_format.cu): stage 0 the row pointers (ia[0] == 0 checked by the
// caller), stage 1 the columns, and with upper the upper-storage rule.
int bsg_check_csr_dev(bsg_ctx *c, int n, int nz, const int *d_ia, const int *d_ja, int stage, int upper);
// Device 3x3 block CSR from device input with column-major blocks, expanded
// from the upper triangle when upper; takes over or frees its inputs
// (k_format.cu).
int bsg_bsr3_from_input(bsg_ctx *c, int nb, int *ia, int *ja, double *a, int nz, int upper, int **ia_o, int **ja_o,
                        double **a_o, int *nnz_o);
int bsg_expand_symmetric(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, int nnz_up, int **ia_o,
                         int **ja_o, double **a_o, int *nnz_o);
int bsg_combine_lu(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, int nnz, int **iu_o,
                   int **ju_o, double **al_o, double **au_o, int *nnz_o);
int bsg_strict_transpose(bsg_ctx *c, int n, const int *ia, const int *ja, int nnz, int **it_o, int **jt_o,
                         int **perm_o, int *nnz_o);
int bsg_bsr_to_point(bsg_ctx *c, int nsup, int bs, const int *ia, const int *ja, const double *a, int nnzb, int **pia_o,
                     int **pja_o, double **pa_o);
int bsg_choose_group(double mean_row);
int bsg_spmm_launch(const bsg_mat *m, int nrhs, const double *X, double *Y, long long ld, cudaStream_t s);
int bsg_fct_make_fp32(bsg_fct *f);
int bsg_fill_launch(cudaStream_t s, long long n, double *x, double v);
int bsg_trisolve_sweep_launch(bsg_ctx *c, const bsg_fct *f, int lower, const double *x, const double *yin,
                              double *yout);

static thread_local char g_err[512] = "";
unsigned long long g_bsg_launches = 0;

extern "C" unsigned long long bsg_launch_count(void) { return g_bsg_launches; }

// Stored entries (padding included) of the SELL copies: [0] the matrix,
// [1] strict L rows, [2] strict U rows of the factor (0 where absent);
// [3] / [4] tiles of the tiled L / U form (0: untiled), [5] most staged x
// blocks (32 floats) of one tile over both; [6] / [7] / [8] long rows of the
// matrix / L / U (rows summed outside the slices).  A block factor reports
// its block SELL copies: 9 entries a block, long block rows.
extern "C" int bsg_sell_stats(const bsg_mat *m, const bsg_fct *f, long long *out) {
	if (!out) return bsg_set_error(BSG_ERR_ARG, "bsg_sell_stats: null output");
	out[0] = m ? m->sell.entries : 0;
	// a block factor's copies count 9 entries a block
	out[1] = f ? (f->d_bia ? 9 * f->bsl.blocks : f->sl.entries) : 0;
	out[2] = f ? (f->d_bia ? 9 * f->bsu.blocks : f->su.entries) : 0;
	out[3] = f ? f->sl.ntile : 0;
	out[4] = f ? f->su.ntile : 0;
	out[5] = f ? (f->sl.tmax > f->su.tmax ? f->sl.tmax : f->su.tmax) : 0;
	out[6] = m ? m->sell.nlong : 0;
	out[7] = f ? (f->d_bia ? f->bsl.nlong : f->sl.nlong) : 0;
	out[8] = f ? (f->d_bia ? f->bsu.nlong : f->su.nlong) : 0;
	return BSG_OK;
}

// Average device time of `reps` back-to-back launches of one kernel, timed
// with CUDA events on the context stream (kind 0: SpMV y = A x; kind 1 / 2:
// forward / backward triangular solve in `mode` with `nsweeps`).  The
// buffers are internal, so the call measures the kernel alone.
extern "C" int bsg_time_kernel(bsg_ctx *c, int kind, const bsg_mat *m, const bsg_fct *f, int mode, int nsweeps,
                               int reps, double *ms_per_launch) {
	if (!c || reps < 1 || !ms_per_launch) return bsg_set_error(BSG_ERR_ARG, "bsg_time_kernel: bad argument");
	if (((kind == 0 || kind == 3) && !m) || ((kind == 1 || kind == 2) && !f) || kind < 0 || kind > 3)
		return bsg_set_error(BSG_ERR_ARG, "bsg_time_kernel: missing object");
	if (kind == 3 && (nsweeps < 1 || nsweeps > 64)) return bsg_set_error(BSG_ERR_ARG, "bsg_time_kernel: nrhs 1..64");
	const int nv = kind == 3 ? nsweeps : 1; // vectors
	const size_t N = kind == 0 || kind == 3 ? (size_t)m->n * m->bs : (size_t)f->n;
	double *x, *y, *w;
	BSG_CUDA(cudaMallocAsync(&x, sizeof(double) * N * nv, c->stream));
	BSG_CUDA(cudaMallocAsync(&y, sizeof(double) * N * nv, c->stream));
	BSG_CUDA(cudaMallocAsync(&w, sizeof(double) * N, c->stream));
	int rc = bsg_fill_launch(c->stream, (long long)(N * nv), x, 1.0);
	if (!rc) rc = bsg_fill_launch(c->stream, (long long)N, w, 0.5);
	auto launch = [&]() {
		if (kind == 0 || kind == 3) return bsg_spmm_launch(m, nv, x, y, (long long)N, c->stream);
		if (mode == 1) return bsg_trisolve_sweep_launch(c, f, kind == 1, x, w, y); // one full sweep
		return bsg_trisolve_launch(c, f, kind == 1, mode, nsweeps, x, y, w);
	};
	for (int r = 0; r < 3 && !rc; r++) rc = launch(); // warm-up
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	cudaEventRecord(e0, c->stream);
	for (int r = 0; r < reps && !rc; r++) rc = launch();
	cudaEventRecord(e1, c->stream);
	cudaEventSynchronize(e1);
	float ms = 0;
	cudaEventElapsedTime(&ms, e0, e1);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFreeAsync(x, c->stream);
	cudaFreeAsync(y, c->stream);
	cudaFreeAsync(w, c->stream);
	if (!rc) rc = bsg_check_devstat(c);
	*ms_per_launch = ms / reps;
	return rc;
}

int bsg_set_error(int code, const char *msg) {
	std::snprintf(g_err, sizeof(g_err), "%s", msg ? msg : "");
	return code;
}
int bsg_set_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
	std::snprintf(g_err, sizeof(g_err), "CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e),
	              cudaGetErrorString(e), what, file, line);
	if (e == cudaErrorMemoryAllocation) return BSG_ERR_NOMEM;
	return BSG_ERR_CUDA;
}

extern "C" const char *bsg_last_error(void) { return g_err; }
extern "C" const char *bsg_version(void) { return "bsg 0.1 sm_100a"; }

// Reads the device status word after the work queued so far.
int bsg_check_devstat(bsg_ctx *c) {
	bsg_devstat h;
	cudaError_t e = cudaMemcpyAsync(&h, c->d_stat, sizeof(h), cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
	if (e != cudaSuccess) return bsg_set_cuda_error(e, "device status", __FILE__, __LINE__);
	if (h.code == 0) return BSG_OK;
	char msg[160];
	switch (h.code) {
	case BSG_ERR_PIVOT: std::snprintf(msg, sizeof msg, " Ich2: Diagonal pivot is nonpositive (row %d)", h.where); break;
	case BSG_ERR_WORKSPACE:
		std::snprintf(msg, sizeof msg, " Insufficient workspace in Ich2/Ilu2 (row %d, check %d)", h.where, h.pad[0]);
		break;
	case BSG_ERR_TIMEOUT: std::snprintf(msg, sizeof msg, "device wait limit reached (index %d)", h.where); break;
	case BSG_ERR_ARG: std::snprintf(msg, sizeof msg, "malformed matrix: missing or misplaced diagonal (row %d)", h.where); break;
	default: std::snprintf(msg, sizeof msg, "device error %d at %d", h.code, h.where);
	}
	cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), c->stream);
	return bsg_set_error(h.code, msg);
}

extern "C" void bsg_param_default(bsg_param *p) {
	std::memset(p, 0, sizeof(*p));
	// CSlvParam() (Bslib/slvparam.h:121-214)
	p->msglev = 0;
	p->fcttyp = 1;
	p->ordtype = 1;
	p->memory = 1.0;
	p->tau1 = 1.0e-2;
	p->tau2 = 1.0e-4;
	p->theta = 1.0e-1;
	p->sclmin = 1.0e-8;
	p->pivmin = 1.0e-8;
	p->ittype = 2;
	p->sttype = 2;
	p->niter = 1000;
	p->eps = 1.0e-9;
	p->ichk = 5;
	p->resfin = 1.0e10;
	// GPU-path defaults
	p->precision = 0;
	p->trisolve = 0;
	p->nsweeps = 3;
	p->krylov = 0;
	p->restart = 50;
	p->true_residual = 1;
	p->blockfct = 1;
	p->learned = nullptr;
}

extern "C" int bsg_create(bsg_ctx **out, int device, void *stream) {
	if (!out) return bsg_set_error(BSG_ERR_ARG, "bsg_create: null output");
	*out = nullptr;
	int ndev = 0;
	cudaError_t e = cudaGetDeviceCount(&ndev);
	if (e != cudaSuccess || ndev == 0) return bsg_set_error(BSG_ERR_CUDA, "no CUDA device");
	if (device < 0 || device >= ndev) return bsg_set_error(BSG_ERR_ARG, "bsg_create: bad device");
	BSG_CUDA(cudaSetDevice(device));
	bsg_ctx *c = new (std::nothrow) bsg_ctx();
	if (!c) return bsg_set_error(BSG_ERR_NOMEM, "bsg_create");
	c->device = device;
	if (stream == BSG_OWN_STREAM) {
		BSG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
		c->own_stream = true;
	} else {
		c->stream = (cudaStream_t)stream; // NULL is the device's default stream
		c->own_stream = false;
	}
	c->n_partials = 8192;
	// Keep freed device memory in the stream-ordered pool: factor pools and
	// Krylov bases are reallocated on every solve, and returning them to the
	// driver at each synchronisation would re-map gigabytes per solve.
	{
		cudaMemPool_t pool;
		if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
			unsigned long long keep = ~0ull;
			cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
		}
	}
	BSG_CUDA(cudaMalloc(&c->d_stat, sizeof(bsg_devstat)));
	BSG_CUDA(cudaMalloc(&c->d_scalars, 64 * sizeof(double)));
	BSG_CUDA(cudaMalloc(&c->d_partials, c->n_partials * sizeof(double)));
	BSG_CUDA(cudaMalloc(&c->d_counters, 16 * sizeof(unsigned)));
	BSG_CUDA(cudaMemset(c->d_stat, 0, sizeof(bsg_devstat)));
	BSG_CUDA(cudaMemset(c->d_scalars, 0, 64 * sizeof(double)));
	BSG_CUDA(cudaMemset(c->d_counters, 0, 16 * sizeof(unsigned)));
	BSG_CUDA(cudaMallocHost(&c->h_pinned, 64 * sizeof(double)));
	BSG_CUDA(cudaEventCreate(&c->ev0));
	BSG_CUDA(cudaEventCreate(&c->ev1));
	c->spmv_group = 0;
	*out = c;
	return BSG_OK;
}

extern "C" int bsg_destroy(bsg_ctx *c) {
	if (!c) return BSG_OK;
	cudaSetDevice(c->device);
	cudaStreamSynchronize(c->stream);
	cudaFree(c->d_stat);
	cudaFree(c->d_scalars);
	cudaFree(c->d_partials);
	cudaFree(c->d_counters);
	cudaFreeHost(c->h_pinned);
	cudaEventDestroy(c->ev0);
	cudaEventDestroy(c->ev1);
	if (c->own_stream) cudaStreamDestroy(c->stream);
	delete c;
	return BSG_OK;
}

int bsg_spin_limit_set_fact(unsigned long long ns);
int bsg_spin_limit_set_trsv(unsigned long long ns);
int bsg_spin_limit_set_unet(unsigned long long ns);

extern "C" int bsg_set_spin_limit_ns(bsg_ctx *c, unsigned long long ns) {
	if (!c) return bsg_set_error(BSG_ERR_ARG, "bsg_set_spin_limit_ns: null context");
	if (ns < 1000ull || ns > 600000000000ull)
		return bsg_set_error(BSG_ERR_ARG, "bsg_set_spin_limit_ns: the limit must lie in [1 us, 600 s]");
	BSG_CUDA(cudaSetDevice(c->device));
	BSG_CUDA(cudaStreamSynchronize(c->stream));
	int rc = bsg_spin_limit_set_fact(ns);
	if (!rc) rc = bsg_spin_limit_set_trsv(ns);
	if (!rc) rc = bsg_spin_limit_set_unet(ns);
	if (rc) return bsg_set_error(rc, "bsg_set_spin_limit_ns: cudaMemcpyToSymbol failed");
	BSG_CUDA(cudaDeviceSynchronize());
	return BSG_OK;
}

extern "C" int bsg_sync(bsg_ctx *c) {
	if (!c) return bsg_set_error(BSG_ERR_ARG, "bsg_sync: null context");
	BSG_CUDA(cudaStreamSynchronize(c->stream));
	return bsg_check_devstat(c);
}

// ---- matrices -------------------------------------------------------------

static int check_csr_host(int n, const int *ia, const int *ja, int bs) {
	if (n < 0 || !ia) return bsg_set_error(BSG_ERR_ARG, "bad CSR: n < 0 or ia == NULL");
	if (ia[0] != 0) return bsg_set_error(BSG_ERR_ARG, "bad CSR: ia[0] != 0");
	for (int i = 0; i < n; i++) {
		if (ia[i + 1] < ia[i]) return bsg_set_error(BSG_ERR_ARG, "bad CSR: ia not monotone");
	}
	int nz = ia[n];
	if (nz > 0 && !ja) return bsg_set_error(BSG_ERR_ARG, "bad CSR: ja == NULL");
	for (int k = 0; k < nz; k++)
		if (ja[k] < 0 || ja[k] >= n) return bsg_set_error(BSG_ERR_ARG, "bad CSR: column index out of range");
	(void)bs;
	return BSG_OK;
}

// Symmetric input must hold the upper triangle only, diagonal first.
static int check_upper_host(int n, const int *ia, const int *ja) {
	for (int i = 0; i < n; i++) {
		if (ia[i + 1] == ia[i] || ja[ia[i]] != i)
			return bsg_set_error(BSG_ERR_ARG, "symmetric input: every row must start with its diagonal");
		for (int k = ia[i]; k < ia[i + 1]; k++)
			if (ja[k] < i) return bsg_set_error(BSG_ERR_ARG, "symmetric input: entry below the diagonal");
	}
	return BSG_OK;
}

// Finish a point matrix whose device full storage is set: upper split,
// static contributor lists, SpMV group size.
static int mat_finish_point(bsg_mat *m, const int *d_up_ia, const int *d_up_ja, const double *d_up_a, int nnz_up,
                            bool from_upper) {
	bsg_ctx *c = m->ctx;
	int rc;
	if (from_upper) {
		// the upper input already is the split pattern (al == au)
		BSG_CUDA(cudaMallocAsync(&m->d_iu, sizeof(int) * (m->n + 1), c->stream));
		BSG_CUDA(cudaMallocAsync(&m->d_ju, sizeof(int) * (nnz_up > 0 ? nnz_up : 1), c->stream));
		BSG_CUDA(cudaMallocAsync(&m->d_al, sizeof(double) * (nnz_up > 0 ? nnz_up : 1), c->stream));
		BSG_CUDA(cudaMemcpyAsync(m->d_iu, d_up_ia, sizeof(int) * (m->n + 1), cudaMemcpyDeviceToDevice, c->stream));
		BSG_CUDA(cudaMemcpyAsync(m->d_ju, d_up_ja, sizeof(int) * nnz_up, cudaMemcpyDeviceToDevice, c->stream));
		BSG_CUDA(cudaMemcpyAsync(m->d_al, d_up_a, sizeof(double) * nnz_up, cudaMemcpyDeviceToDevice, c->stream));
		m->d_au = m->d_al;
		m->nnz_up = nnz_up;
	} else {
		rc = bsg_combine_lu(c, m->n, m->d_ia, m->d_ja, m->d_a, m->nnz, &m->d_iu, &m->d_ju, &m->d_al, &m->d_au,
		                    &m->nnz_up);
		if (rc) return rc;
	}
	int nt = 0;
	rc = bsg_strict_transpose(c, m->n, m->d_iu, m->d_ju, m->nnz_up, &m->d_it, &m->d_jt, nullptr, &nt);
	if (rc) return rc;
	rc = bsg_sell_build(c, m->n, m->d_ia, m->d_ja, m->d_a, 0, 0, &m->sell);
	if (rc) return rc;
	m->group = bsg_choose_group(m->n > 0 ? (double)m->nnz / m->n : 1.0);
	BSG_CUDA(cudaStreamSynchronize(c->stream));
	return BSG_OK;
}

static int mat_csr_common(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, int symm_upper,
                          bool host, bsg_mat **out) {
	if (!c || !out) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_csr: null argument");
	*out = nullptr;
	int nz = 0;
	if (host) { // the O(1) checks here, the rest on the device copies below
		if (n < 0 || !ia) return bsg_set_error(BSG_ERR_ARG, "bad CSR: n < 0 or ia == NULL");
		if (ia[0] != 0) return bsg_set_error(BSG_ERR_ARG, "bad CSR: ia[0] != 0");
		nz = ia[n];
		if (nz < 0) return bsg_set_error(BSG_ERR_ARG, "bad CSR: ia not monotone");
	} else {
		BSG_CUDA(cudaMemcpy(&nz, ia + n, sizeof(int), cudaMemcpyDeviceToHost));
	}
	BSG_CUDA(cudaSetDevice(c->device));
	bsg_mat *m = new (std::nothrow) bsg_mat();
	if (!m) return bsg_set_error(BSG_ERR_NOMEM, "bsg_mat_csr");
	m->ctx = c;
	m->n = n;
	m->bs = 1;
	m->symm = symm_upper ? 1 : 0;
	cudaStream_t s = c->stream;
	cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
	int *d_ia, *d_ja;
	double *d_a;
	BSG_CUDA(cudaMallocAsync(&d_ia, sizeof(int) * (n + 1), s));
	BSG_CUDA(cudaMallocAsync(&d_ja, sizeof(int) * (nz > 0 ? nz : 1), s));
	BSG_CUDA(cudaMallocAsync(&d_a, sizeof(double) * (nz > 0 ? nz : 1), s));
	BSG_CUDA(cudaMemcpyAsync(d_ia, ia, sizeof(int) * (n + 1), kind, s));
	int rc = BSG_OK;
	// host input: the row pointers are checked before the columns are read
	if (host) rc = bsg_check_csr_dev(c, n, nz, d_ia, nullptr, 0, 0);
	if (!rc && host && nz > 0 && !ja) rc = bsg_set_error(BSG_ERR_ARG, "bad CSR: ja == NULL");
	if (!rc && nz > 0) {
		BSG_CUDA(cudaMemcpyAsync(d_ja, ja, sizeof(int) * nz, kind, s));
		BSG_CUDA(cudaMemcpyAsync(d_a, a, sizeof(double) * nz, kind, s));
	}
	if (!rc && host) rc = bsg_check_csr_dev(c, n, nz, d_ia, d_ja, 1, symm_upper);
	if (rc) {
		cudaFreeAsync(d_ia, s);
		cudaFreeAsync(d_ja, s);
		cudaFreeAsync(d_a, s);
		delete m;
		return rc;
	}
	if (symm_upper) {
		rc = bsg_expand_symmetric(c, n, d_ia, d_ja, d_a, nz, &m->d_ia, &m->d_ja, &m->d_a, &m->nnz);
		if (!rc) rc = mat_finish_point(m, d_ia, d_ja, d_a, nz, true);
		cudaFreeAsync(d_ia, s);
		cudaFreeAsync(d_ja, s);
		cudaFreeAsync(d_a, s);
	} else {
		m->d_ia = d_ia;
		m->d_ja = d_ja;
		m->d_a = d_a;
		m->nnz = nz;
		rc = mat_finish_point(m, nullptr, nullptr, nullptr, 0, false);
	}
	if (rc) {
		bsg_mat_free(m);
		return rc;
	}
	*out = m;
	return BSG_OK;
}

extern "C" int bsg_mat_csr(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, int symm_upper,
                           bsg_mat **out) {
	return mat_csr_common(c, n, ia, ja, a, symm_upper, true, out);
}
extern "C" int bsg_mat_csr_dev(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, int symm_upper,
                               bsg_mat **out) {
	return mat_csr_common(c, n, ia, ja, a, symm_upper, false, out);
}

// Point CSR of a block matrix with block sizes sprnd[i+1] - sprnd[i]
// (CSMatrixRS with sprndr = sprndc, Bslib/smatrix.h:1040-1048): the blocks of
// block row i follow one another in `a`, each column-major, columns ascending.
// Symmetric (upper) input keeps the upper triangle of each diagonal block, so
// every point row starts with its diagonal; rows come out column-sorted.
static int vbsr_to_point_host(int nsup, const int *sprnd, const int *ia, const int *ja, const double *a,
                              int symm_upper, std::vector<int> &pia, std::vector<int> &pja, std::vector<double> &pa) {
	const int n = sprnd[nsup];
	std::vector<long long> cnt(n + 1, 0);
	size_t off = 0;
	std::vector<size_t> bsa(ia[nsup] + 1, 0);
	for (int i = 0; i < nsup; i++) {
		const int bi = sprnd[i + 1] - sprnd[i];
		for (int k = ia[i]; k < ia[i + 1]; k++) {
			const int j = ja[k], bj = sprnd[j + 1] - sprnd[j];
			bsa[k] = off;
			off += (size_t)bi * bj;
			for (int r = 0; r < bi; r++) {
				const int nr = (symm_upper && j == i) ? bj - r : bj;
				cnt[sprnd[i] + r + 1] += nr;
			}
		}
	}
	for (int r = 0; r < n; r++) cnt[r + 1] += cnt[r];
	if (cnt[n] > 0x7fffffffLL) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_vbsr: more than 2^31 point entries");
	pia.assign(cnt.begin(), cnt.end());
	pja.resize(pia[n]);
	pa.resize(pia[n]);
	std::vector<int> pos(pia.begin(), pia.end() - 1);
	for (int i = 0; i < nsup; i++) {
		const int bi = sprnd[i + 1] - sprnd[i];
		for (int k = ia[i]; k < ia[i + 1]; k++) {
			const int j = ja[k], bj = sprnd[j + 1] - sprnd[j];
			const double *blk = a + bsa[k];
			for (int r = 0; r < bi; r++)
				for (int cc = (symm_upper && j == i) ? r : 0; cc < bj; cc++) {
					const int q = pos[sprnd[i] + r]++;
					pja[q] = sprnd[j] + cc;
					pa[q] = blk[(size_t)cc * bi + r];
				}
		}
	}
	return BSG_OK;
}

extern "C" int bsg_mat_vbsr(bsg_ctx *c, int nsup, const int *sprnd, const int *ia, const int *ja, const double *a,
                            int symm_upper, bsg_mat **out) {
	if (!c || !out || !sprnd) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_vbsr: null argument");
	*out = nullptr;
	const bool force_point = (symm_upper & BSG_VBSR_POINT) != 0;
	symm_upper &= 1;
	int rc = check_csr_host(nsup, ia, ja, 1);
	if (rc) return rc;
	if (sprnd[0] != 0) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_vbsr: sprnd[0] != 0");
	bool all3 = true, all1 = true;
	for (int i = 0; i < nsup; i++) {
		const int b = sprnd[i + 1] - sprnd[i];
		if (b < 1) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_vbsr: empty block");
		all3 = all3 && b == 3;
		all1 = all1 && b == 1;
	}
	for (int i = 0; i < nsup; i++)
		for (int k = ia[i] + 1; k < ia[i + 1]; k++)
			if (ja[k] <= ja[k - 1]) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_vbsr: block columns must ascend");
	if (symm_upper) {
		rc = check_upper_host(nsup, ia, ja);
		if (rc) return rc;
	}
	if (all1) return bsg_mat_csr(c, nsup, ia, ja, a, symm_upper, out);
	if (all3 && !force_point) return bsg_mat_bsr(c, nsup, 3, ia, ja, a, symm_upper, out);
	std::vector<int> pia, pja;
	std::vector<double> pa;
	rc = vbsr_to_point_host(nsup, sprnd, ia, ja, a, symm_upper, pia, pja, pa);
	if (rc) return rc;
	return bsg_mat_csr(c, sprnd[nsup], pia.data(), pja.data(), pa.data(), symm_upper, out);
}

extern "C" int bsg_mat_bsr(bsg_ctx *c, int nsup, int bs, const int *ia, const int *ja, const double *a,
                           int symm_upper, bsg_mat **out) {
	if (!c || !out) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_bsr: null argument");
	if (bs < 1) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_bsr: block size must be positive");
	if (bs == 1) return bsg_mat_csr(c, nsup, ia, ja, a, symm_upper, out);
	if (bs != 3) {
		// other uniform sizes: the point expansion (columns sorted per row first)
		if (nsup < 0 || (long long)nsup * bs > 0x7fffffffLL) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_bsr: too large");
		int rc = check_csr_host(nsup, ia, ja, bs);
		if (rc) return rc;
		std::vector<int> sprnd(nsup + 1), sja(ia[nsup]);
		std::vector<double> sa((size_t)ia[nsup] * bs * bs);
		for (int i = 0; i <= nsup; i++) sprnd[i] = i * bs;
		std::vector<std::pair<int, int>> row;
		for (int i = 0; i < nsup; i++) {
			row.clear();
			for (int k = ia[i]; k < ia[i + 1]; k++) row.push_back({ja[k], k});
			std::sort(row.begin(), row.end());
			for (size_t q = 0; q < row.size(); q++) {
				sja[ia[i] + q] = row[q].first;
				std::copy(a + (size_t)row[q].second * bs * bs, a + (size_t)(row[q].second + 1) * bs * bs,
				          sa.begin() + (size_t)(ia[i] + q) * bs * bs);
			}
		}
		return bsg_mat_vbsr(c, nsup, sprnd.data(), ia, sja.data(), sa.data(), symm_upper, out);
	}
	// the O(1) checks here, the rest on device copies; the symmetric expansion
	// and the row-major blocks on the device
	if (nsup < 0 || !ia) return bsg_set_error(BSG_ERR_ARG, "bad CSR: n < 0 or ia == NULL");
	if (ia[0] != 0) return bsg_set_error(BSG_ERR_ARG, "bad CSR: ia[0] != 0");
	const int nz = ia[nsup];
	if (nz < 0) return bsg_set_error(BSG_ERR_ARG, "bad CSR: ia not monotone");
	BSG_CUDA(cudaSetDevice(c->device));
	cudaStream_t s = c->stream;
	int *d_ia = nullptr, *d_ja = nullptr;
	double *d_a = nullptr;
	BSG_CUDA(cudaMallocAsync(&d_ia, sizeof(int) * (nsup + 1), s));
	BSG_CUDA(cudaMallocAsync(&d_ja, sizeof(int) * (nz > 0 ? nz : 1), s));
	BSG_CUDA(cudaMallocAsync(&d_a, sizeof(double) * 9 * (size_t)(nz > 0 ? nz : 1), s));
	BSG_CUDA(cudaMemcpyAsync(d_ia, ia, sizeof(int) * (nsup + 1), cudaMemcpyHostToDevice, s));
	int rc = bsg_check_csr_dev(c, nsup, nz, d_ia, nullptr, 0, 0);
	if (!rc && nz > 0 && (!ja || !a)) rc = bsg_set_error(BSG_ERR_ARG, "bad CSR: ja == NULL");
	if (!rc && nz > 0) {
		BSG_CUDA(cudaMemcpyAsync(d_ja, ja, sizeof(int) * nz, cudaMemcpyHostToDevice, s));
		BSG_CUDA(cudaMemcpyAsync(d_a, a, sizeof(double) * 9 * (size_t)nz, cudaMemcpyHostToDevice, s));
	}
	if (!rc) rc = bsg_check_csr_dev(c, nsup, nz, d_ia, d_ja, 1, symm_upper);
	bsg_mat *m = rc ? nullptr : new (std::nothrow) bsg_mat();
	if (!rc && !m) rc = bsg_set_error(BSG_ERR_NOMEM, "bsg_mat_bsr");
	if (!rc) {
		m->ctx = c;
		m->n = nsup;
		m->bs = 3;
		m->symm = symm_upper ? 1 : 0;
		rc = bsg_bsr3_from_input(c, nsup, d_ia, d_ja, d_a, nz, symm_upper, &m->d_ia, &m->d_ja, &m->d_a, &m->nnz);
		if (!rc) d_ia = d_ja = nullptr, d_a = nullptr; // taken over or freed
	}
	for (void *q : {(void *)d_ia, (void *)d_ja, (void *)d_a})
		if (q) cudaFreeAsync(q, s);
	if (rc) {
		if (m) bsg_mat_free(m);
		return rc;
	}
	m->group = 32;
	// the factorisations of a block matrix work on its point expansion: keep
	// the point CombineLU split and its static contributor lists
	int *pia = nullptr, *pja = nullptr;
	double *pa = nullptr;
	rc = bsg_bsr_to_point(c, nsup, 3, m->d_ia, m->d_ja, m->d_a, m->nnz, &pia, &pja, &pa);
	if (!rc)
		rc = bsg_combine_lu(c, nsup * 3, pia, pja, pa, m->nnz * 9, &m->d_iu, &m->d_ju, &m->d_al, &m->d_au,
		                    &m->nnz_up);
	for (void *q : {(void *)pia, (void *)pja, (void *)pa})
		if (q) cudaFreeAsync(q, s);
	if (!rc && symm_upper) {
		// IC2 reads the upper values as given (au = A(i,j), j >= i), not
		// the mirrored lower copies of the diagonal blocks
		cudaFreeAsync(m->d_al, s);
		m->d_al = m->d_au;
	}
	int nt = 0;
	if (!rc) rc = bsg_strict_transpose(c, nsup * 3, m->d_iu, m->d_ju, m->nnz_up, &m->d_it, &m->d_jt, nullptr, &nt);
	if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = bsg_set_error(BSG_ERR_CUDA, "bsg_mat_bsr");
	if (rc) {
		bsg_mat_free(m);
		return rc;
	}
	*out = m;
	return BSG_OK;
}

extern "C" int bsg_mat_free(bsg_mat *m) {
	if (!m) return BSG_OK;
	cudaStream_t s = m->ctx->stream;
	bsg_sell_free(&m->sell, s);
	bsg_sell_free(&m->sellT, s);
	if (m->d_au && m->d_au != m->d_al) cudaFreeAsync(m->d_au, s);
	for (void *p : {(void *)m->d_ia, (void *)m->d_ja, (void *)m->d_a, (void *)m->d_iu, (void *)m->d_ju,
	                (void *)m->d_al, (void *)m->d_it, (void *)m->d_jt})
		if (p) cudaFreeAsync(p, s);
	cudaStreamSynchronize(s);
	delete m;
	return BSG_OK;
}

extern "C" int bsg_mat_info(const bsg_mat *m, int *n, int *bs, int *nnz) {
	if (!m) return bsg_set_error(BSG_ERR_ARG, "bsg_mat_info: null matrix");
	if (n) *n = m->n;
	if (bs) *bs = m->bs;
	if (nnz) *nnz = m->nnz;
	return BSG_OK;
}

extern "C" int bsg_mvm_dev(bsg_ctx *c, const bsg_mat *m, const double *x, double *y) {
	if (!c || !m || !x || !y) return bsg_set_error(BSG_ERR_ARG, "bsg_mvm_dev: null argument");
	int rc = bsg_spmm_launch(m, 1, x, y, (long long)m->n * m->bs, c->stream);
	return rc ? bsg_set_error(rc, "SpMV launch failed") : BSG_OK;
}

extern "C" int bsg_mvm_multi_dev(bsg_ctx *c, const bsg_mat *m, int nrhs, const double *X, double *Y) {
	if (!c || !m || !X || !Y || nrhs < 1) return bsg_set_error(BSG_ERR_ARG, "bsg_mvm_multi_dev: bad argument");
	int rc = bsg_spmm_launch(m, nrhs, X, Y, (long long)m->n * m->bs, c->stream);
	return rc ? bsg_set_error(rc, "SpMM launch failed") : BSG_OK;
}

extern "C" int bsg_mvm(bsg_ctx *c, const bsg_mat *m, const double *x, double *y) {
	if (!c || !m || !x || !y) return bsg_set_error(BSG_ERR_ARG, "bsg_mvm: null argument");
	const size_t N = (size_t)m->n * m->bs;
	double *dx, *dy;
	BSG_CUDA(cudaMallocAsync(&dx, sizeof(double) * N, c->stream));
	BSG_CUDA(cudaMallocAsync(&dy, sizeof(double) * N, c->stream));
	BSG_CUDA(cudaMemcpyAsync(dx, x, sizeof(double) * N, cudaMemcpyHostToDevice, c->stream));
	int rc = bsg_mvm_dev(c, m, dx, dy);
	if (!rc) {
		BSG_CUDA(cudaMemcpyAsync(y, dy, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
		BSG_CUDA(cudaStreamSynchronize(c->stream));
	}
	cudaFreeAsync(dx, c->stream);
	cudaFreeAsync(dy, c->stream);
	return rc;
}

// ---- factors --------------------------------------------------------------

int bsg_ic0_run(bsg_ctx *c, bsg_mat *m, bsg_fct **out);

static int fct_common(bsg_ctx *c, bsg_mat *m, bsg_param *p, int kind, bsg_fct **out) {
	if (!c || !m || !p || !out) return bsg_set_error(BSG_ERR_ARG, "factorisation: null argument");
	*out = nullptr;
	if (p->ordtype != 0) return bsg_set_error(BSG_ERR_UNSUPPORTED, "only natural ordering (ordtype = 0) runs on the GPU");
	bsg_fct *f = nullptr;
	// a 3x3 block matrix gets the reference's block factorisations
	// (CSMatrixRS::Ilu2 / CSMatrixRS::Ich2); fcttyp 1 of a symmetric point
	// matrix is IC(0) (CSMatrixR::Ich, SolveSymm's fcttyp 1)
	const bool block = m->bs == 3 && p->blockfct != 0;
	const bool ic0 = kind == 0 && p->fcttyp == 1;
	if (ic0 && (block || m->bs != 1 || !m->symm))
		return bsg_set_error(BSG_ERR_UNSUPPORTED, "fcttyp = 1 (IC(0)) needs a symmetric point matrix (upper input)");
	int rc = ic0 ? bsg_ic0_run(c, m, &f) : block ? bsg_bfact_run(c, m, kind == 0, p, &f) : bsg_fact_run(c, m, kind, p, &f);
	if (rc) return rc;
	float ms = 0;
	cudaEventElapsedTime(&ms, c->ev0, c->ev1);
	p->timefct = ms * 1e-3;
	p->density = f->density;
	p->density2 = f->density2;
	if (p->precision == 1) {
		rc = block ? bsg_bfact_make_fp32(f) : bsg_fct_make_fp32(f);
		if (rc) { bsg_fct_free(f); return rc; }
	}
	*out = f;
	return BSG_OK;
}

extern "C" int bsg_fct_ich2(bsg_ctx *c, bsg_mat *m, bsg_param *p, bsg_fct **out) { return fct_common(c, m, p, 0, out); }
extern "C" int bsg_fct_ilu2(bsg_ctx *c, bsg_mat *m, bsg_param *p, bsg_fct **out) { return fct_common(c, m, p, 1, out); }
extern "C" int bsg_fct_to_fp32(bsg_fct *f) {
	if (!f) return bsg_set_error(BSG_ERR_ARG, "bsg_fct_to_fp32: null factor");
	return f->d_bia ? bsg_bfact_make_fp32(f) : bsg_fct_make_fp32(f);
}

extern "C" int bsg_fct_export(const bsg_fct *f, int *nnz, int *iu, int *ju, double *l, double *u) {
	if (!f) return bsg_set_error(BSG_ERR_ARG, "bsg_fct_export: null factor");
	if (f->d_bia) return bsg_set_error(BSG_ERR_ARG, "bsg_fct_export: block factor (use bsg_fct_export_block)");
	if (nnz) *nnz = f->nnz;
	cudaStream_t s = f->ctx->stream;
	if (iu) BSG_CUDA(cudaMemcpyAsync(iu, f->d_iu, sizeof(int) * (f->n + 1), cudaMemcpyDeviceToHost, s));
	if (ju) BSG_CUDA(cudaMemcpyAsync(ju, f->d_ju, sizeof(int) * f->nnz, cudaMemcpyDeviceToHost, s));
	if (l) BSG_CUDA(cudaMemcpyAsync(l, f->d_l, sizeof(double) * f->nnz, cudaMemcpyDeviceToHost, s));
	if (u) BSG_CUDA(cudaMemcpyAsync(u, f->d_u, sizeof(double) * f->nnz, cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	return BSG_OK;
}

extern "C" int bsg_fct_export_block(const bsg_fct *f, int *nb, int *nnzb, int *ia, int *ja, double *l, double *u) {
	if (!f) return bsg_set_error(BSG_ERR_ARG, "bsg_fct_export_block: null factor");
	if (!f->d_bia) return bsg_set_error(BSG_ERR_ARG, "bsg_fct_export_block: point factor (use bsg_fct_export)");
	if (nb) *nb = f->nb;
	if (nnzb) *nnzb = f->nnz;
	cudaStream_t s = f->ctx->stream;
	if (ia) BSG_CUDA(cudaMemcpyAsync(ia, f->d_bia, sizeof(int) * (f->nb + 1), cudaMemcpyDeviceToHost, s));
	if (ja) BSG_CUDA(cudaMemcpyAsync(ja, f->d_bja, sizeof(int) * f->nnz, cudaMemcpyDeviceToHost, s));
	if (l) BSG_CUDA(cudaMemcpyAsync(l, f->d_bl, sizeof(double) * 9 * (size_t)f->nnz, cudaMemcpyDeviceToHost, s));
	if (u) BSG_CUDA(cudaMemcpyAsync(u, f->d_bu, sizeof(double) * 9 * (size_t)f->nnz, cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	return BSG_OK;
}

extern "C" int bsg_fct_info(const bsg_fct *f, int *n, int *nnz, int *levels_l, int *levels_u, double *density,
                            double *density2) {
	if (!f) return bsg_set_error(BSG_ERR_ARG, "bsg_fct_info: null factor");
	if (n) *n = f->n;
	if (nnz) *nnz = f->nnz;
	if (levels_l) *levels_l = f->levels_l;
	if (levels_u) *levels_u = f->levels_u;
	if (density) *density = f->density;
	if (density2) *density2 = f->density2;
	return BSG_OK;
}

extern "C" int bsg_fct_free(bsg_fct *f) {
	if (!f) return BSG_OK;
	cudaStream_t s = f->ctx->stream;
	bsg_sell_free(&f->sl, s);
	bsg_sell_free(&f->su, s);
	bsg_sell_free(&f->slt, s);
	bsg_sell_free(&f->sut, s);
	bsg_bsell_free(&f->bsl, s);
	bsg_bsell_free(&f->bsu, s);
	if (f->d_swscr) cudaFreeAsync(f->d_swscr, s);
	for (void *q : {(void *)f->d_utr_v, (void *)f->d_utr_f, (void *)f->d_l_f})
		if (q) cudaFreeAsync(q, s);
	if (f->d_l && f->d_l != f->d_u) cudaFreeAsync(f->d_l, s);
	for (void *p : {(void *)f->d_iu, (void *)f->d_ju, (void *)f->d_u, (void *)f->d_dinv_l, (void *)f->d_dinv_u,
	                (void *)f->d_lr_i, (void *)f->d_lr_j, (void *)f->d_lr_v, (void *)f->d_ur_f, (void *)f->d_lr_f,
	                (void *)f->d_perm})
		if (p) cudaFreeAsync(p, s);
	if (f->d_bia) // block factor: its strict U rows are separate arrays
		for (void *p : {(void *)f->d_bia, (void *)f->d_bja, (void *)f->d_bl, (void *)f->d_bu, (void *)f->d_bdl,
		                (void *)f->d_bdu, (void *)f->d_ones, (void *)f->d_ur_i, (void *)f->d_ur_j, (void *)f->d_ur_v})
			if (p) cudaFreeAsync(p, s);
	cudaStreamSynchronize(s);
	delete f;
	return BSG_OK;
}

extern "C" int bsg_solve_l_dev(bsg_ctx *c, const bsg_fct *f, int mode, int nsweeps, const double *x, double *y) {
	if (!c || !f || !x || !y || x == y) return bsg_set_error(BSG_ERR_ARG, "bsg_solve_l_dev: bad argument");
	double *work = nullptr;
	if (mode == 1 && nsweeps > 1) BSG_CUDA(cudaMallocAsync(&work, sizeof(double) * f->n, c->stream));
	int rc = bsg_trisolve_launch(c, f, 1, mode, nsweeps, x, y, work);
	if (work) cudaFreeAsync(work, c->stream);
	if (!rc) rc = bsg_check_devstat(c);
	return rc;
}
extern "C" int bsg_solve_t_dev(bsg_ctx *c, bsg_fct *f, int which, int mode, int nsweeps, const double *x, double *y) {
	if (!c || !f || !x || !y || x == y || (which != 0 && which != 1))
		return bsg_set_error(BSG_ERR_ARG, "bsg_solve_t_dev: bad argument");
	double *work = nullptr;
	if (mode == 1 && nsweeps > 1) BSG_CUDA(cudaMallocAsync(&work, sizeof(double) * f->n, c->stream));
	int rc = bsg_trisolve_t_launch(c, f, which, mode, nsweeps, x, y, work);
	if (work) cudaFreeAsync(work, c->stream);
	if (!rc) rc = bsg_check_devstat(c);
	return rc;
}
extern "C" int bsg_solve_u_dev(bsg_ctx *c, const bsg_fct *f, int mode, int nsweeps, const double *x, double *y) {
	if (!c || !f || !x || !y || x == y) return bsg_set_error(BSG_ERR_ARG, "bsg_solve_u_dev: bad argument");
	double *work = nullptr;
	if (mode == 1 && nsweeps > 1) BSG_CUDA(cudaMallocAsync(&work, sizeof(double) * f->n, c->stream));
	int rc = bsg_trisolve_launch(c, f, 0, mode, nsweeps, x, y, work);
	if (work) cudaFreeAsync(work, c->stream);
	if (!rc) rc = bsg_check_devstat(c);
	return rc;
}

extern "C" int bsg_solve_multi_dev(bsg_ctx *c, const bsg_fct *f, int lower, int mode, int nsweeps, int nrhs,
                                   const double *x, double *y) {
	if (!c || !f || !x || !y || x == y || nrhs < 1)
		return bsg_set_error(BSG_ERR_ARG, "bsg_solve_multi_dev: bad argument");
	double *work = nullptr;
	if (mode == 1 && nsweeps > 1) BSG_CUDA(cudaMallocAsync(&work, sizeof(double) * f->n * (size_t)nrhs, c->stream));
	int rc = bsg_trisolve_multi(c, f, lower ? 1 : 0, mode, nsweeps, nrhs, x, y, work);
	if (work) cudaFreeAsync(work, c->stream);
	if (!rc) rc = bsg_check_devstat(c);
	return rc;
}

// ---- host-buffer drivers ----------------------------------------------------

static int drive(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, const double *b, double *x,
                 bsg_param *p, int symm) {
	if (!c || !p || !b || !x) return bsg_set_error(BSG_ERR_ARG, "driver: null argument");
	bsg_mat *m = nullptr;
	bsg_fct *f = nullptr;
	int rc = bsg_mat_csr(c, n, ia, ja, a, symm, &m);
	if (rc) return rc;
	rc = symm ? bsg_fct_ich2(c, m, p, &f) : bsg_fct_ilu2(c, m, p, &f);
	if (rc) { bsg_mat_free(m); return rc; }
	double *db = nullptr, *dx = nullptr;
	cudaStream_t s = c->stream;
	if (cudaMallocAsync(&db, sizeof(double) * n, s) != cudaSuccess || cudaMallocAsync(&dx, sizeof(double) * n, s) != cudaSuccess) {
		bsg_fct_free(f); bsg_mat_free(m);
		return bsg_set_error(BSG_ERR_NOMEM, "driver vectors");
	}
	cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyHostToDevice, s);
	cudaMemsetAsync(dx, 0, sizeof(double) * n, s);
	if (p->krylov != 0) rc = bsg_gmres_dev(c, m, f, db, dx, p);
	else if (symm) rc = bsg_pcg_dev(c, m, f, db, dx, p);  // SolveSymm: Cg
	else rc = bsg_lanczos_dev(c, m, f, db, dx, p);        // Solver: Lanczos
	int rc2 = (int)cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
	cudaStreamSynchronize(s);
	cudaFreeAsync(db, s);
	cudaFreeAsync(dx, s);
	bsg_fct_free(f);
	bsg_mat_free(m);
	if (!rc && rc2) rc = bsg_set_error(BSG_ERR_CUDA, "copy of the solution failed");
	return rc;
}

extern "C" int bsg_solve_lu(bsg_ctx *c, const bsg_fct *f, int which, int mode, int nsweeps, const double *x,
                            double *y) {
	if (!c || !f || !x || !y || which < 0 || which > 2 || mode < 0 || mode > 1)
		return bsg_set_error(BSG_ERR_ARG, "bsg_solve_lu: bad argument");
	const size_t n = (size_t)f->n * (f->d_bia ? 3 : 1);
	cudaStream_t s = c->stream;
	double *dx = nullptr, *dy = nullptr, *dt = nullptr, *work = nullptr;
	int rc = BSG_OK;
	if (cudaMallocAsync(&dx, sizeof(double) * (n ? n : 1), s) != cudaSuccess ||
	    cudaMallocAsync(&dy, sizeof(double) * (n ? n : 1), s) != cudaSuccess ||
	    cudaMallocAsync(&dt, sizeof(double) * (n ? n : 1), s) != cudaSuccess ||
	    cudaMallocAsync(&work, sizeof(double) * (n ? n : 1), s) != cudaSuccess)
		rc = bsg_set_error(BSG_ERR_NOMEM, "bsg_solve_lu: vectors");
	if (!rc && cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
		rc = bsg_set_error(BSG_ERR_CUDA, "bsg_solve_lu: copy to the device failed");
	// which 0: SolveL then SolveU (the preconditioner), 1: SolveL, 2: SolveU
	if (!rc && which != 2) rc = bsg_trisolve_launch(c, f, 1, mode, nsweeps, dx, which == 0 ? dt : dy, work);
	if (!rc && which != 1) rc = bsg_trisolve_launch(c, f, 0, mode, nsweeps, which == 0 ? dt : dx, dy, work);
	if (!rc && cudaMemcpyAsync(y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost, s) != cudaSuccess)
		rc = bsg_set_error(BSG_ERR_CUDA, "bsg_solve_lu: copy of the result failed");
	cudaStreamSynchronize(s);
	for (double *q : {dx, dy, dt, work})
		if (q) cudaFreeAsync(q, s);
	if (!rc) rc = bsg_check_devstat(c);
	return rc;
}

extern "C" int bsg_solve(bsg_ctx *c, const bsg_mat *m, const bsg_fct *f, const double *b, double *x, bsg_param *p) {
	if (!c || !m || !f || !p || !b || !x) return bsg_set_error(BSG_ERR_ARG, "bsg_solve: null argument");
	const size_t n = (size_t)m->n * m->bs;
	double *db = nullptr, *dx = nullptr;
	cudaStream_t s = c->stream;
	if (cudaMallocAsync(&db, sizeof(double) * (n ? n : 1), s) != cudaSuccess ||
	    cudaMallocAsync(&dx, sizeof(double) * (n ? n : 1), s) != cudaSuccess) {
		if (db) cudaFreeAsync(db, s);
		return bsg_set_error(BSG_ERR_NOMEM, "bsg_solve: vectors");
	}
	int rc = BSG_OK;
	if (cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
	    cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
		rc = bsg_set_error(BSG_ERR_CUDA, "bsg_solve: copy to the device failed");
	if (!rc) {
		const bool point = m->bs == 1 && !f->d_bia;
		if (p->krylov != 0) rc = bsg_gmres_dev(c, m, f, db, dx, p);
		else if (m->symm) rc = bsg_pcg_dev(c, m, f, db, dx, p);              // CSVector::Cg
		else if (point && p->ittype >= 2 && p->ittype <= 4)                   // block Lanczos variants
			rc = bsg_block_lanczos_dev(c, m, f, p->ittype, 1, db, dx, p, nullptr);
		else if (point) rc = bsg_lanczos_dev(c, m, f, db, dx, p);            // CSVector::Lanczos
		else rc = bsg_gmres_dev(c, m, f, db, dx, p);
	}
	// the last iterate comes back also when the iteration limit was reached
	if (rc == BSG_OK || rc == BSG_ERR_NOCONV) {
		if (cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s) != cudaSuccess && rc == BSG_OK)
			rc = bsg_set_error(BSG_ERR_CUDA, "bsg_solve: copy of the solution failed");
	}
	cudaStreamSynchronize(s);
	cudaFreeAsync(db, s);
	cudaFreeAsync(dx, s);
	return rc;
}

extern "C" int bsg_solve_symm_csr(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, const double *b,
                                  double *x, bsg_param *p) {
	return drive(c, n, ia, ja, a, b, x, p, 1);
}
extern "C" int bsg_solver_csr(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, const double *b,
                              double *x, bsg_param *p) {
	return drive(c, n, ia, ja, a, b, x, p, 0);
}
