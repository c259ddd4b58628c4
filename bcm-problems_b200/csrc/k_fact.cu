// Second-order threshold incomplete factorisation on the GPU: IC2
// (CSMatrixR::Ich2, Bslib/ich2r.cpp:956-1195) and ILU2 (CSMatrixR::Ilu2,
// Bslib/ilu2r.cpp:1122-1395), numeric phase with the pattern decided on the
// fly exactly as the reference decides it (tau1 / tau2 / theta rules).
//
// Parallel schedule ("sync-free rows").  One warp factors one row; warps
// claim rows in increasing order from an atomic counter, so every row a warp
// waits for is held by a running warp and the schedule cannot deadlock.
// Row i needs every earlier row k whose row mask contains column i
// (C(i) = {k < i : i in mask(k)}); the rows that update i (i stored in k)
// and the rows whose dropped entry at i compensates i's diagonal.  C(i) is
// not known in advance, but it closes over finished rows: a column i enters
// mask(k) only through A(k,i) != 0 or through an earlier row m in C(i) that
// stores both k and i (unless both are R entries, the R x R skip of
// Ich2InitMask, Bslib/ich2r.cpp:202-222).  So the warp seeds C(i) with the
// rows of A's column i, and for each finished member m that stores i it adds
// the stored columns of m lying between m and i.  Each wait is on a row of
// lower index with a bounded spin (globaltimer limit).
//
// Arithmetic order (deterministic, identical to oracle/bsl_oracle.c):
// compensations into the diagonal in ascending contributor order, then the
// updates of ascending contributors, each as fma(-l, g, f), then the row's own
// theta compensations in ascending column order.  The reference uses its
// linked-list order instead, which changes results only at rounding level.
//
// Output: a pool of finished rows (diagonal first, then every mask column
// ascending, flagged U / R / dropped) from which the U part is compacted into
// the reference layout (Ich2StoreScaleU, Bslib/ich2r.cpp:910-954).
#include "bsg_internal.cuh"
#include <cub/device/device_scan.cuh>

#define F_U 0u
#define F_R 1u
#define F_D 2u
#define CF_COL(x) ((int)((x) & 0x3fffffffu))
#define CF_FLAG(x) ((x) >> 30)

#define FACT_WARPS 4
#define CMAX 256   // contributors per row
#define HCAP 512   // distinct mask columns per row (power of two)

namespace {

struct FactArgs {
	int n, kind;
	const int *iu, *ju;          // upper pattern, diagonal first
	const double *al, *au;       // values (al == au for IC2)
	const int *it, *jt;          // static contributors: rows k < i with (k,i) stored
	const double *scll, *sclu, *diag0;
	double tau1, tau2, theta, pivmin;
	unsigned int *pool_cf;       // col | flag << 30
	double *pool_l, *pool_u;
	long long pool_cap;
	unsigned long long *pool_len;
	long long *row_off;
	int *row_len, *done;
	unsigned int *claim;
	bsg_devstat *st;
};

struct WarpShared {
	int W[CMAX];           // contributors (unsorted, then sorted)
	int Wp[CMAX];          // pool index of column i in that row
	unsigned char Wf[CMAX];
	int Ws[CMAX];
	int Wps[CMAX];
	unsigned char Wfs[CMAX];
	int wset[CMAX * 2];    // membership hash of W (keys)
	int hkey[HCAP];        // column accumulator
	double hl[HCAP], hu[HCAP];
	int lst[HCAP];         // extracted slots, then sorted
	int lsts[HCAP];
	int nW, nl;
};

__device__ __forceinline__ unsigned hash_u(int k) { return (unsigned)k * 2654435761u; }

// Find or insert column c; returns slot or -1 if full.
__device__ int hfind_insert(WarpShared &s, int c) {
	unsigned h = hash_u(c) & (HCAP - 1);
	for (int probe = 0; probe < HCAP; probe++) {
		int k = s.hkey[h];
		if (k == c) return (int)h;
		if (k == -1) {
			int old = atomicCAS(&s.hkey[h], -1, c);
			if (old == -1) {
				s.hl[h] = 0.0;
				s.hu[h] = 0.0;
				return (int)h;
			}
			if (old == c) return (int)h;
		}
		h = (h + 1) & (HCAP - 1);
	}
	return -1;
}

// Insert row k into the contributor set; returns 1 if new, 0 if present, -1 if full.
__device__ int wset_insert(WarpShared &s, int k) {
	unsigned h = hash_u(k) & (2 * CMAX - 1);
	for (int probe = 0; probe < 2 * CMAX; probe++) {
		int old = atomicCAS(&s.wset[h], -1, k);
		if (old == -1) return 1;
		if (old == k) return 0;
		h = (h + 1) & (2 * CMAX - 1);
	}
	return -1;
}

// Bounded wait for row m; returns 1 when finished, 0 on abort/timeout.
__device__ int wait_row(const FactArgs &A, int m) {
	int v = ld_acquire(A.done + m);
	if (v == 1) return 1;
	if (v == 2) return 0;
	unsigned long long t0 = globaltimer_ns();
	for (unsigned it = 1;; it++) {
		__nanosleep(100);
		v = ld_acquire(A.done + m);
		if (v == 1) return 1;
		if (v == 2) return 0;
		if ((it & 63) == 0) {
			if (*(volatile int *)&A.st->code != 0) return 0;
			if (globaltimer_ns() - t0 > BSG_SPIN_LIMIT_NS) {
				devstat_fail(A.st, BSG_ERR_TIMEOUT, m);
				return 0;
			}
		}
	}
}

__global__ void __launch_bounds__(FACT_WARPS * 32) k_fact_rows(FactArgs A) {
	extern __shared__ unsigned char smem_raw[];
	WarpShared &s = reinterpret_cast<WarpShared *>(smem_raw)[threadIdx.x >> 5];
	const int lane = threadIdx.x & 31;
	const bool ilu = A.kind == 1;

	for (;;) {
		int i = 0;
		if (lane == 0) i = (int)atomicAdd(A.claim, 1u);
		i = __shfl_sync(0xffffffffu, i, 0);
		if (i >= A.n) return;
		if (*(volatile int *)&A.st->code != 0) return;

		// ---- reset per-row shared state
		for (int t = lane; t < 2 * CMAX; t += 32) s.wset[t] = -1;
		for (int t = lane; t < HCAP; t += 32) s.hkey[t] = -1;
		__syncwarp();

		// ---- seed contributors with A's column i
		const int tb = A.it[i], te = A.it[i + 1];
		int err = 0;
		if (te - tb > CMAX) err = BSG_ERR_WORKSPACE;
		if (!err) {
			for (int t = tb + lane; t < te; t += 32) {
				int k = A.jt[t];
				s.W[t - tb] = k;
				wset_insert(s, k);
			}
		}
		if (lane == 0) s.nW = te - tb;
		__syncwarp();

		// ---- close C(i) over finished rows
		for (int idx = 0; !err && idx < s.nW; idx++) {
			const int m = s.W[idx];
			int ok = 1;
			if (lane == 0) ok = wait_row(A, m);
			ok = __shfl_sync(0xffffffffu, ok, 0);
			__syncwarp();
			if (!ok) { err = -100; break; }
			const long long off = __ldcg(A.row_off + m);
			const int len = __ldcg(A.row_len + m);
			// binary search column i among the mask columns of row m (entries 1..len-1)
			int pos = -1;
			unsigned fi = 0;
			if (lane == 0) {
				int lo = 1, hi = len - 1;
				while (lo <= hi) {
					int mid = (lo + hi) >> 1;
					int c = CF_COL(__ldcg(A.pool_cf + off + mid));
					if (c == i) { pos = mid; break; }
					if (c < i) lo = mid + 1; else hi = mid - 1;
				}
				if (pos >= 0) fi = CF_FLAG(__ldcg(A.pool_cf + off + pos));
			}
			pos = __shfl_sync(0xffffffffu, pos, 0);
			fi = __shfl_sync(0xffffffffu, fi, 0);
			if (pos < 0) { err = BSG_ERR_ARG; break; }
			if (lane == 0) { s.Wp[idx] = (int)(off + pos); s.Wf[idx] = (unsigned char)fi; }
			if (fi != F_D) {
				for (int e0 = 1; e0 < pos; e0 += 32) {
					const int e = e0 + lane;
					bool cand = false;
					int k = 0;
					if (e < pos) {
						unsigned cf = __ldcg(A.pool_cf + off + e);
						unsigned fe = CF_FLAG(cf);
						cand = fe != F_D && !(fi == F_R && fe == F_R);
						k = CF_COL(cf);
					}
					int isnew = 0;
					if (cand) isnew = wset_insert(s, k);
					if (isnew < 0) err = BSG_ERR_WORKSPACE;
					unsigned b = __ballot_sync(0xffffffffu, isnew == 1);
					int base = s.nW;
					__syncwarp();
					if (isnew == 1) {
						int slot = base + __popc(b & ((1u << lane) - 1));
						if (slot < CMAX) s.W[slot] = k; else err = BSG_ERR_WORKSPACE;
					}
					__syncwarp();
					if (lane == 0) s.nW = min(base + __popc(b), CMAX);
					__syncwarp();
				}
				err = __reduce_min_sync(0xffffffffu, err);
			}
			__syncwarp();
		}
		if (err) {
			if (err != -100 && lane == 0) devstat_fail(A.st, err, i);
			if (lane == 0) st_release(A.done + i, 2);
			return;
		}
		const int nW = s.nW;

		// ---- sort contributors ascending (rank sort; rows are distinct)
		for (int t = lane; t < nW; t += 32) {
			int k = s.W[t], r = 0;
			for (int u = 0; u < nW; u++) r += s.W[u] < k;
			s.Ws[r] = k; s.Wps[r] = s.Wp[t]; s.Wfs[r] = s.Wf[t];
		}
		__syncwarp();

		// ---- diagonal: initial scaled value plus earlier rows' compensations
		double dsum = 0.0;
		if (lane == 0) {
			dsum = A.diag0[i];
			for (int t = 0; t < nW; t++)
				if (s.Wfs[t] == F_D) dsum += __ldcg(A.pool_l + s.Wps[t]);
		}
		dsum = __shfl_sync(0xffffffffu, dsum, 0);

		// ---- init the scaled row (Ich2InitRow / Ilu2InitRow)
		const int ab = A.iu[i], ae = A.iu[i + 1];
		{
			int slot = -1;
			if (lane == 0) {
				slot = hfind_insert(s, i);
				s.hl[slot] = dsum;
				s.hu[slot] = dsum;
			}
			__syncwarp();
			const double si_l = A.scll[i], si_u = A.sclu[i];
			for (int k = ab + 1 + lane; k < ae; k += 32) {
				int j = A.ju[k];
				int sl = hfind_insert(s, j);
				if (sl < 0) { err = BSG_ERR_WORKSPACE; continue; }
				if (ilu) {
					s.hl[sl] = A.al[k] * si_u * A.scll[j];
					s.hu[sl] = A.au[k] * si_l * A.sclu[j];
				} else {
					double v = A.al[k] * si_l * A.scll[j];
					s.hl[sl] = v;
					s.hu[sl] = v;
				}
			}
			__syncwarp();
		}

		// ---- updates from stored contributors, ascending
		for (int t = 0; t < nW && !err; t++) {
			const unsigned fi = s.Wfs[t];
			if (fi == F_D) continue;
			const int m = s.Ws[t];
			const long long p0 = s.Wps[t];
			const long long end = __ldcg(A.row_off + m) + __ldcg(A.row_len + m);
			const double lel = __ldcg(A.pool_l + p0);
			const double uel = ilu ? __ldcg(A.pool_u + p0) : lel;
			for (long long e = p0 + lane; e < end; e += 32) {
				unsigned cf = __ldcg(A.pool_cf + e);
				unsigned fe = CF_FLAG(cf);
				if (fe == F_D || (fi == F_R && fe == F_R)) continue;
				int sl = hfind_insert(s, CF_COL(cf));
				if (sl < 0) { err = BSG_ERR_WORKSPACE; continue; }
				if (ilu) {
					s.hl[sl] = fma(-uel, __ldcg(A.pool_l + e), s.hl[sl]);
					s.hu[sl] = fma(-lel, __ldcg(A.pool_u + e), s.hu[sl]);
				} else {
					double v = fma(-lel, __ldcg(A.pool_l + e), s.hl[sl]);
					s.hl[sl] = v;
					s.hu[sl] = v;
				}
			}
			__syncwarp();
			err = __reduce_min_sync(0xffffffffu, err);
		}
		err = __reduce_min_sync(0xffffffffu, err);
		if (err) {
			if (lane == 0) { devstat_fail(A.st, err, i); st_release(A.done + i, 2); }
			return;
		}

		// ---- extract the off-diagonal mask columns and sort them ascending
		if (lane == 0) s.nl = 0;
		__syncwarp();
		for (int h = lane; h < HCAP; h += 32) {
			int c = s.hkey[h];
			bool take = c >= 0 && c != i;
			unsigned b = __ballot_sync(0xffffffffu, take);
			int base = s.nl;
			if (take) s.lst[base + __popc(b & ((1u << lane) - 1))] = h;
			__syncwarp();
			if (lane == 0) s.nl = base + __popc(b);
			__syncwarp();
		}
		const int nl = s.nl;
		for (int t = lane; t < nl; t += 32) {
			int c = s.hkey[s.lst[t]], r = 0;
			for (int u = 0; u < nl; u++) r += s.hkey[s.lst[u]] < c;
			s.lsts[r] = s.lst[t];
		}
		__syncwarp();
		const int di = hfind_insert(s, i); // existing slot of the diagonal

		// ---- filter by tau2 with theta compensation (ascending columns)
		if (lane == 0) {
			double dl = s.hl[di], du = s.hu[di];
			for (int t = 0; t < nl; t++) {
				int h = s.lsts[t];
				double v = fabs(s.hl[h]);
				if (ilu) v = fmax(v, fabs(s.hu[h]));
				if (!(v >= A.tau2)) {
					v *= A.theta;
					dl += v;
					du += v;
				}
			}
			s.hl[di] = dl;
			s.hu[di] = du;
		}
		__syncwarp();

		// ---- pivot (Ich2PivScaleRow / Ilu2PivScaleRow)
		const double fd = s.hl[di];
		double deleml, delemu;
		if (!ilu) {
			if (!(fd > 0.0)) {
				if (lane == 0) { devstat_fail(A.st, BSG_ERR_PIVOT, i); st_release(A.done + i, 2); }
				return;
			}
			deleml = delemu = 1.0 / sqrt(fd);
		} else {
			double m = fabs(fd);
			if (m < A.pivmin) m = A.pivmin;
			deleml = 1.0 / sqrt(m);
			delemu = fd < 0.0 ? -deleml : deleml;
		}

		// ---- store the row: diagonal, then every mask column ascending
		long long off = 0;
		if (lane == 0) {
			off = (long long)atomicAdd(A.pool_len, (unsigned long long)(nl + 1));
		}
		off = __shfl_sync(0xffffffffu, off, 0);
		if (off + nl + 1 > A.pool_cap) {
			if (lane == 0) { devstat_fail(A.st, BSG_ERR_WORKSPACE, i); st_release(A.done + i, 2); }
			return;
		}
		if (lane == 0) {
			A.pool_cf[off] = (unsigned)i | (F_U << 30);
			A.pool_l[off] = deleml;
			if (ilu) A.pool_u[off] = delemu;
		}
		for (int t = lane; t < nl; t += 32) {
			int h = s.lsts[t];
			int c = s.hkey[h];
			double l = s.hl[h], u = s.hu[h];
			double v = fabs(l);
			if (ilu) v = fmax(v, fabs(u));
			unsigned flag;
			if (!(v >= A.tau2)) {
				flag = F_D;
				l = v * A.theta; // compensation handed to row c
				u = l;
			} else {
				if (ilu) { l *= delemu; u *= deleml; } else { l *= deleml; u = l; }
				double w = fabs(l);
				if (ilu) w = fmax(w, fabs(u));
				flag = (w >= A.tau1) ? F_U : F_R;
			}
			A.pool_cf[off + 1 + t] = (unsigned)c | (flag << 30);
			A.pool_l[off + 1 + t] = l;
			if (ilu) A.pool_u[off + 1 + t] = u;
		}
		if (lane == 0) {
			A.row_off[i] = off;
			A.row_len[i] = nl + 1;
		}
		__threadfence();
		__syncwarp();
		if (lane == 0) st_release(A.done + i, 1);
	}
}

// Scaling (Ich2AllocScale, Bslib/ich2r.cpp:62-97; Ilu2AllocScale,
// Bslib/ilu2r.cpp:28-66).  Missing or misplaced diagonal -> BSG_ERR_ARG.
__global__ void k_fact_scale(int n, int kind, const int *iu, const int *ju, const double *al, double sclmin,
                             double *scll, double *sclu, double *diag0, bsg_devstat *st) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	if (iu[i] >= iu[i + 1] || ju[iu[i]] != i) {
		devstat_fail(st, BSG_ERR_ARG, i);
		return;
	}
	double d = al[iu[i]];
	if (kind == 0) {
		double s = 1.0 / sqrt(d);
		scll[i] = s;
		sclu[i] = s;
		diag0[i] = d * s * s;
	} else {
		double m = fabs(d);
		if (m < sclmin) m = sclmin;
		m = 1.0 / sqrt(m);
		scll[i] = m;
		sclu[i] = d < 0.0 ? m : -m;
		diag0[i] = d * scll[i] * sclu[i];
	}
}

__global__ void k_count_u(int n, const long long *row_off, const int *row_len, const unsigned *cf, int *cnt, int *cntr) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	long long off = row_off[i];
	int len = row_len[i], c = 0, r = 0;
	for (long long e = off; e < off + len; e++) {
		unsigned f = CF_FLAG(cf[e]);
		c += f == F_U;
		r += f == F_R;
	}
	cnt[i] = c;
	cntr[i] = r;
}

__global__ void k_emit_u(int n, int kind, const long long *row_off, const int *row_len, const unsigned *cf,
                         const double *pl, const double *pu, const double *scll, const double *sclu,
                         const int *iu_out, int *ju, double *l, double *u) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	long long off = row_off[i];
	int len = row_len[i];
	int z = iu_out[i];
	for (long long e = off; e < off + len; e++) {
		unsigned x = cf[e];
		if (CF_FLAG(x) != F_U) continue;
		int j = CF_COL(x);
		ju[z] = j;
		if (j == i) {
			l[z] = pl[e] * scll[i];
			u[z] = (kind == 1 ? pu[e] : pl[e]) * sclu[i];
		} else {
			l[z] = pl[e] / scll[j];
			u[z] = (kind == 1 ? pu[e] : pl[e]) / sclu[j];
		}
		z++;
	}
}

inline int nb(long long n, int t) { return (int)((n + t - 1) / t); }

} // namespace

int bsg_strict_transpose(bsg_ctx *c, int n, const int *ia, const int *ja, int nnz, int **it_o, int **jt_o,
                         int **perm_o, int *nnz_o);
int bsg_fct_finish(bsg_ctx *c, bsg_fct *f);

// Runs the factorisation of m (whose upper split d_iu/d_ju/d_al/d_au and
// static contributor lists d_it/d_jt are prepared) and builds the factor.
int bsg_fact_run(bsg_ctx *c, bsg_mat *m, int kind, const bsg_param *p, bsg_fct **out) {
	const int n = m->n;
	cudaStream_t st = c->stream;
	double mem = p->memory < 0 ? -p->memory : p->memory;
	if (mem < 8.0) mem = 8.0;
	// the pool holds U + R + dropped entries (the reference's `memory` counts
	// U + R only), so it is sized at 3x the requested multiple of nnz(A)
	long long cap = (long long)(mem * 3.0 * (double)m->nnz_up) + 4LL * n + 1024;
	if (cap > 0x7ffffff0LL) cap = 0x7ffffff0LL; // pool indices are 32-bit
	double *scll, *sclu, *diag0, *pl, *pu = nullptr;
	unsigned *cf;
	long long *row_off;
	int *row_len, *done;
	unsigned long long *pool_len;
	unsigned *claim;
	BSG_CUDA(cudaMallocAsync(&scll, sizeof(double) * n, st));
	BSG_CUDA(cudaMallocAsync(&sclu, sizeof(double) * n, st));
	BSG_CUDA(cudaMallocAsync(&diag0, sizeof(double) * n, st));
	if (cudaMallocAsync(&cf, sizeof(unsigned) * cap, st) != cudaSuccess) return bsg_set_error(BSG_ERR_NOMEM, "factor pool");
	if (cudaMallocAsync(&pl, sizeof(double) * cap, st) != cudaSuccess) return bsg_set_error(BSG_ERR_NOMEM, "factor pool");
	if (kind == 1 && cudaMallocAsync(&pu, sizeof(double) * cap, st) != cudaSuccess)
		return bsg_set_error(BSG_ERR_NOMEM, "factor pool");
	BSG_CUDA(cudaMallocAsync(&row_off, sizeof(long long) * n, st));
	BSG_CUDA(cudaMallocAsync(&row_len, sizeof(int) * n, st));
	BSG_CUDA(cudaMallocAsync(&done, sizeof(int) * n, st));
	BSG_CUDA(cudaMallocAsync(&pool_len, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMallocAsync(&claim, sizeof(unsigned), st));
	BSG_CUDA(cudaMemsetAsync(done, 0, sizeof(int) * n, st));
	BSG_CUDA(cudaMemsetAsync(pool_len, 0, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMemsetAsync(claim, 0, sizeof(unsigned), st));
	BSG_CUDA(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), st));

	cudaEventRecord(c->ev0, st);
	k_fact_scale<<<nb(n, 256), 256, 0, st>>>(n, kind, m->d_iu, m->d_ju, m->d_al, p->sclmin, scll, sclu, diag0, c->d_stat);
	FactArgs A;
	A.n = n; A.kind = kind;
	A.iu = m->d_iu; A.ju = m->d_ju; A.al = m->d_al; A.au = m->d_au;
	A.it = m->d_it; A.jt = m->d_jt;
	A.scll = scll; A.sclu = sclu; A.diag0 = diag0;
	A.tau1 = p->tau1; A.tau2 = p->tau2; A.theta = p->theta; A.pivmin = p->pivmin;
	A.pool_cf = cf; A.pool_l = pl; A.pool_u = pu; A.pool_cap = cap; A.pool_len = pool_len;
	A.row_off = row_off; A.row_len = row_len; A.done = done; A.claim = claim; A.st = c->d_stat;
	size_t smem = sizeof(WarpShared) * FACT_WARPS;
	BSG_CUDA(cudaFuncSetAttribute(k_fact_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	int per_sm = 0;
	BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fact_rows, FACT_WARPS * 32, smem));
	if (per_sm < 1) per_sm = 1;
	int grid = per_sm * BSG_SMS;
	int need = (n + FACT_WARPS - 1) / FACT_WARPS;
	if (grid > need) grid = need;
	if (grid < 1) grid = 1;
	k_fact_rows<<<grid, FACT_WARPS * 32, smem, st>>>(A);
	BSG_CUDA(cudaGetLastError());
	int rc = bsg_check_devstat(c);
	if (rc) {
		cudaFreeAsync(scll, st); cudaFreeAsync(sclu, st); cudaFreeAsync(diag0, st); cudaFreeAsync(cf, st);
		cudaFreeAsync(pl, st); if (pu) cudaFreeAsync(pu, st); cudaFreeAsync(row_off, st); cudaFreeAsync(row_len, st);
		cudaFreeAsync(done, st); cudaFreeAsync(pool_len, st); cudaFreeAsync(claim, st);
		return rc;
	}

	// ---- compact U into the reference layout
	bsg_fct *f = new bsg_fct();
	f->ctx = c; f->n = n; f->bs = 1; f->kind = kind;
	int *cnt, *cntr, *iu;
	BSG_CUDA(cudaMallocAsync(&cnt, sizeof(int) * (n + 1), st));
	BSG_CUDA(cudaMallocAsync(&cntr, sizeof(int) * (n + 1), st));
	BSG_CUDA(cudaMallocAsync(&iu, sizeof(int) * (n + 1), st));
	BSG_CUDA(cudaMemsetAsync(cnt + n, 0, sizeof(int), st));
	BSG_CUDA(cudaMemsetAsync(cntr + n, 0, sizeof(int), st));
	k_count_u<<<nb(n, 256), 256, 0, st>>>(n, row_off, row_len, cf, cnt, cntr);
	size_t tmp = 0;
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, iu, n + 1, st));
	void *d_tmp;
	BSG_CUDA(cudaMallocAsync(&d_tmp, tmp, st));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, cnt, iu, n + 1, st));
	int nzu = 0;
	BSG_CUDA(cudaMemcpyAsync(&nzu, iu + n, sizeof(int), cudaMemcpyDeviceToHost, st));
	// R count (density2)
	int *iur;
	BSG_CUDA(cudaMallocAsync(&iur, sizeof(int) * (n + 1), st));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, cntr, iur, n + 1, st));
	int nzr = 0;
	BSG_CUDA(cudaMemcpyAsync(&nzr, iur + n, sizeof(int), cudaMemcpyDeviceToHost, st));
	BSG_CUDA(cudaStreamSynchronize(st));
	f->nnz = nzu;
	f->d_iu = iu;
	BSG_CUDA(cudaMallocAsync(&f->d_ju, sizeof(int) * nzu, st));
	BSG_CUDA(cudaMallocAsync(&f->d_l, sizeof(double) * nzu, st));
	BSG_CUDA(cudaMallocAsync(&f->d_u, sizeof(double) * nzu, st));
	k_emit_u<<<nb(n, 256), 256, 0, st>>>(n, kind, row_off, row_len, cf, pl, pu, scll, sclu, iu, f->d_ju, f->d_l, f->d_u);
	BSG_CUDA(cudaGetLastError());
	cudaEventRecord(c->ev1, st);
	f->density = (double)nzu / (double)m->nnz_up;
	f->density2 = (double)nzr / (double)m->nnz_up;
	cudaFreeAsync(cnt, st); cudaFreeAsync(cntr, st); cudaFreeAsync(iur, st); cudaFreeAsync(d_tmp, st);
	cudaFreeAsync(scll, st); cudaFreeAsync(sclu, st); cudaFreeAsync(diag0, st); cudaFreeAsync(cf, st);
	cudaFreeAsync(pl, st); if (pu) cudaFreeAsync(pu, st); cudaFreeAsync(row_off, st); cudaFreeAsync(row_len, st);
	cudaFreeAsync(done, st); cudaFreeAsync(pool_len, st); cudaFreeAsync(claim, st);
	rc = bsg_fct_finish(c, f);
	if (rc) return rc;
	*out = f;
	return BSG_OK;
}
