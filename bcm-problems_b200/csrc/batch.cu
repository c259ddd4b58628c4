// Batched PCG: many independent SPD systems in one solve.  A system is one
// (right-hand side, segment) pair: nrhs right-hand sides of one matrix (the
// load cases of a homogenisation cell) times nseg diagonal blocks of that
// matrix that nothing couples (a batch of independent problems assembled as
// one block-diagonal matrix).  Every system runs CSVector::Cg's recurrence
// (Bslib/cg.cpp:31-350) with its own scalars and its own stopping test; the
// reference solves one right-hand side of one problem at a time
// (Bslib/cg.cpp:375-377), this solves them together with one SpMM, one
// preconditioner pass per right-hand side and segmented reductions per
// iteration.
//
// Vectors are [nrhs][n] with leading dimension n.  Reductions are split into
// fixed chunks (a block per chunk, then one warp per system adding its chunks
// in order), so every system's scalars are deterministic.  A converged
// system takes zero steps while the others continue.  The iterations are
// captured once in a CUDA graph of `graph_iters` iterations and the graph is
// replayed; the host reads the number of active systems once per replay.
// The chunk length of the reductions and, for point matrices with several
// right-hand sides, the sub-warp group of the SpMM are chosen on first use by
// timing the candidates (autotune), and kept for the shape.
#include "bsg_internal.cuh"
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

int bsg_spmm_launch(const bsg_mat *m, int nrhs, const double *X, double *Y, long long ld, cudaStream_t s);
int bsg_precond_apply_multi(bsg_ctx *c, const bsg_fct *f, const bsg_param *p, int nr, const double *r, double *z,
                            double *tmp, double *work);

namespace {

// per-system scalars (doubles, SC_N per system)
enum { SC_GAM = 0, SC_GAMOLD, SC_PAP, SC_RR, SC_RR0, SC_ALPHA, SC_BETA, SC_BB, SC_N = 8 };
// per-system ints
enum { SI_ACTIVE = 0, SI_ITERS, SI_FIRST, SI_BREAK, SI_N = 4 };

struct Chunks {
	int nchunk = 0;
	int *sys = nullptr;        // system of each chunk
	long long *beg = nullptr;  // element range inside the [nrhs][n] vector
	long long *end = nullptr;
	int *first = nullptr;      // first chunk of each system (nsys + 1)
};

// partial[c*Q + q] = sum over chunk c of x_q . y_q
template <int Q>
__global__ void __launch_bounds__(256) k_bdots(int nchunk, const long long *beg, const long long *end, const double *x0,
                                               const double *y0, const double *x1, const double *y1, double *part) {
	__shared__ double sh[Q][8];
	for (int c = blockIdx.x; c < nchunk; c += gridDim.x) {
		double a[Q];
#pragma unroll
		for (int q = 0; q < Q; q++) a[q] = 0.0;
		for (long long e = beg[c] + threadIdx.x; e < end[c]; e += blockDim.x) {
			a[0] = fma(x0[e], y0[e], a[0]);
			if (Q > 1) a[Q - 1] = fma(x1[e], y1[e], a[Q - 1]);
		}
#pragma unroll
		for (int q = 0; q < Q; q++) {
			double v = warp_sum(a[q]);
			if ((threadIdx.x & 31) == 0) sh[q][threadIdx.x >> 5] = v;
		}
		__syncthreads();
		if (threadIdx.x < Q) {
			double t = 0.0;
			for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[threadIdx.x][w];
			part[(size_t)c * Q + threadIdx.x] = t;
		}
		__syncthreads();
	}
}

// out[s*SC_N + slot_q] = sum of the chunks of system s, in chunk order (one
// warp per system: lane-strided sums, then a fixed shuffle tree)
template <int Q>
__global__ void k_bfinal(int nsys, const int *first, const double *part, double *sc, int slot0, int slot1) {
	const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	const int lane = threadIdx.x & 31;
	if (s >= nsys) return;
	double a[Q];
#pragma unroll
	for (int q = 0; q < Q; q++) a[q] = 0.0;
	for (int c = first[s] + lane; c < first[s + 1]; c += 32)
#pragma unroll
		for (int q = 0; q < Q; q++) a[q] += part[(size_t)c * Q + q];
#pragma unroll
	for (int q = 0; q < Q; q++) a[q] = warp_sum(a[q]);
	if (lane == 0) {
		sc[(size_t)s * SC_N + slot0] = a[0];
		if (Q > 1) sc[(size_t)s * SC_N + slot1] = a[Q - 1];
	}
}

// alpha = gamma / (p . A p) for active systems (Bslib/cg.cpp:262-278; a
// non-positive p . A p is a breakdown: the system stops)
__global__ void k_balpha(int nsys, double *sc, int *si) {
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= nsys) return;
	double *d = sc + (size_t)s * SC_N;
	int *k = si + (size_t)s * SI_N;
	double alpha = 0.0;
	if (k[SI_ACTIVE]) {
		if (!(d[SC_PAP] > 0.0)) {
			k[SI_ACTIVE] = 0;
			k[SI_BREAK] = 1;
		} else {
			alpha = d[SC_GAM] / d[SC_PAP];
		}
	}
	d[SC_ALPHA] = alpha;
}

// after z = M^{-1} r and the dots (r.r, r.z): stopping test on the recursive
// residual relative to the initial one (ittype 0), then beta
__global__ void k_bbeta(int nsys, double eps2, int niter, double *sc, int *si, int *nactive) {
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= nsys) return;
	double *d = sc + (size_t)s * SC_N;
	int *k = si + (size_t)s * SI_N;
	double beta = 0.0;
	if (k[SI_ACTIVE]) {
		k[SI_ITERS]++;
		if (d[SC_RR] <= eps2 * d[SC_RR0] || k[SI_ITERS] >= niter) {
			k[SI_ACTIVE] = 0;
		} else {
			beta = k[SI_FIRST] ? 0.0 : d[SC_GAM] / d[SC_GAMOLD];
			k[SI_FIRST] = 0;
			d[SC_GAMOLD] = d[SC_GAM];
			atomicAdd(nactive, 1);
		}
	}
	d[SC_BETA] = beta;
}

// End of one pass of the loop body: continue while a system is active and
// the pass limit is not reached; clear the active count for the next pass.
__global__ void k_bcontinue(cudaGraphConditionalHandle h, int *cnt, int max_passes) {
	const int passes = ++cnt[2];
	const bool go = cnt[0] > 0 && passes < max_passes;
	cnt[0] = 0;
	cudaGraphSetConditional(h, go ? 1u : 0u);
}

// system of element e of the [nrhs][n] vectors
__device__ __forceinline__ int sys_of(long long e, long long n, int nseg, const int *segid) {
	const int rhs = (int)(e / n);
	return rhs * nseg + segid[e - (long long)rhs * n];
}

// p = z + beta p for active systems
__global__ void k_bp(long long N, long long n, int nseg, const int *segid, const double *sc, const int *si,
                     const double *z, double *p) {
	for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
		const int s = sys_of(e, n, nseg, segid);
		if (si[(size_t)s * SI_N + SI_ACTIVE]) p[e] = fma(sc[(size_t)s * SC_N + SC_BETA], p[e], z[e]);
	}
}

// x += alpha p, r -= alpha q (alpha = 0 for stopped systems)
__global__ void k_bxr(long long N, long long n, int nseg, const int *segid, const double *sc, const double *p,
                      const double *q, double *r, double *x) {
	for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
		const double a = sc[(size_t)sys_of(e, n, nseg, segid) * SC_N + SC_ALPHA];
		if (a != 0.0) {
			x[e] = fma(a, p[e], x[e]);
			r[e] = fma(-a, q[e], r[e]);
		}
	}
}

// r = b - t
__global__ void k_bres(long long N, const double *b, const double *t, double *r) {
	for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x)
		r[e] = b[e] - t[e];
}

// segment id of every row; and a check that no matrix entry couples two
// segments (the systems would not be independent)
__global__ void k_segid(int nrow, int nseg, const int *off, int *segid) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow; i += gridDim.x * blockDim.x) {
		int lo = 0, hi = nseg - 1;
		while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (off[mid] <= i) lo = mid; else hi = mid - 1; }
		segid[i] = lo;
	}
}
__global__ void k_segcheck(int nbrow, int bs, const int *ia, const int *ja, const int *segid, int *bad) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbrow; i += gridDim.x * blockDim.x) {
		const int si = segid[(long long)i * bs];
		for (int k = ia[i]; k < ia[i + 1]; k++)
			if (segid[(long long)ja[k] * bs] != si) { atomicExch(bad, 1); break; }
	}
}

__global__ void k_binit(int nsys, double *sc, int *si) {
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= nsys) return;
	double *d = sc + (size_t)s * SC_N;
	int *k = si + (size_t)s * SI_N;
	d[SC_RR0] = d[SC_RR];
	d[SC_GAMOLD] = d[SC_GAM];
	k[SI_ACTIVE] = d[SC_RR] > 0.0 ? 1 : 0;
	k[SI_ITERS] = 0;
	k[SI_FIRST] = 1;
	k[SI_BREAK] = 0;
	d[SC_BETA] = 0.0;
}
// restart a system from its true residual (FP32 drift): active again, p = z
__global__ void k_brestart(int nsys, double eps2, double *sc, int *si, int *nrestart) {
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= nsys) return;
	double *d = sc + (size_t)s * SC_N;
	int *k = si + (size_t)s * SI_N;
	// SC_BB holds the true residual r.r here
	if (!k[SI_BREAK] && d[SC_BB] > eps2 * d[SC_RR0]) {
		k[SI_ACTIVE] = 1;
		k[SI_FIRST] = 1;
		atomicAdd(nrestart, 1);
	}
}

inline int ew(long long n) {
	long long b = (n + 255) / 256;
	return (int)(b < BSG_SMS * 16 ? (b > 0 ? b : 1) : BSG_SMS * 16);
}

// stream-ordered device buffer, freed on scope exit (move-only)
struct DevBuf {
	void *p = nullptr;
	cudaStream_t s = nullptr;
	DevBuf() = default;
	DevBuf(const DevBuf &) = delete;
	DevBuf &operator=(const DevBuf &) = delete;
	DevBuf(DevBuf &&o) noexcept : p(o.p), s(o.s) { o.p = nullptr; }
	~DevBuf() { if (p) cudaFreeAsync(p, s); }
};

int build_chunks(cudaStream_t st, int nrhs, int nseg, const std::vector<long long> &off, long long n, long long chunk,
                 Chunks &ch, std::vector<DevBuf> &keep) {
	std::vector<int> sys, first;
	std::vector<long long> b, e;
	for (int r = 0; r < nrhs; r++)
		for (int g = 0; g < nseg; g++) {
			first.push_back((int)sys.size());
			const long long s0 = off[g], s1 = off[g + 1];
			for (long long a = s0; a < s1; a += chunk) {
				sys.push_back(r * nseg + g);
				b.push_back(r * n + a);
				e.push_back(r * n + (a + chunk < s1 ? a + chunk : s1));
			}
		}
	first.push_back((int)sys.size());
	ch.nchunk = (int)sys.size();
	keep.resize(keep.size() + 4);
	DevBuf *d = &keep[keep.size() - 4];
	for (int k = 0; k < 4; k++) d[k].s = st;
	BSG_CUDA(cudaMallocAsync(&d[0].p, sizeof(int) * (sys.size() + 1), st));
	BSG_CUDA(cudaMallocAsync(&d[1].p, sizeof(long long) * (b.size() + 1), st));
	BSG_CUDA(cudaMallocAsync(&d[2].p, sizeof(long long) * (e.size() + 1), st));
	BSG_CUDA(cudaMallocAsync(&d[3].p, sizeof(int) * first.size(), st));
	BSG_CUDA(cudaMemcpyAsync(d[0].p, sys.data(), sizeof(int) * sys.size(), cudaMemcpyHostToDevice, st));
	BSG_CUDA(cudaMemcpyAsync(d[1].p, b.data(), sizeof(long long) * b.size(), cudaMemcpyHostToDevice, st));
	BSG_CUDA(cudaMemcpyAsync(d[2].p, e.data(), sizeof(long long) * e.size(), cudaMemcpyHostToDevice, st));
	BSG_CUDA(cudaMemcpyAsync(d[3].p, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice, st));
	BSG_CUDA(cudaStreamSynchronize(st)); // the host vectors go out of scope
	ch.sys = (int *)d[0].p;
	ch.beg = (long long *)d[1].p;
	ch.end = (long long *)d[2].p;
	ch.first = (int *)d[3].p;
	return BSG_OK;
}

// tuned shapes, per (rows, block size, nrhs, nseg)
struct Tuned {
	long long chunk;
	int group;
};
std::map<std::tuple<long long, int, int, int>, Tuned> g_tuned;

} // namespace

extern "C" int bsg_pcg_batch_dev(bsg_ctx *c, const bsg_mat *m, const bsg_fct *f, int nrhs, int nseg,
                                 const int *seg_off, const double *d_B, double *d_X, bsg_param *p, int *iters,
                                 double *res, int *tuned) {
	if (!c || !m || !f || !d_B || !d_X || !p || nrhs < 1 || nseg < 1 || (nseg > 1 && !seg_off))
		return bsg_set_error(BSG_ERR_ARG, "bsg_pcg_batch_dev: bad argument");
	const long long n = (long long)m->n * m->bs;
	const long long N = n * nrhs;
	const int nsys = nrhs * nseg;
	if (f->n != n) return bsg_set_error(BSG_ERR_ARG, "bsg_pcg_batch_dev: factor and matrix sizes differ");
	std::vector<long long> off(nseg + 1);
	if (nseg == 1) {
		off[0] = 0; off[1] = n;
	} else {
		for (int g = 0; g <= nseg; g++) off[g] = seg_off[g];
		if (off[0] != 0 || off[nseg] != n) return bsg_set_error(BSG_ERR_ARG, "bsg_pcg_batch_dev: segments must cover 0..n");
		for (int g = 0; g < nseg; g++)
			if (off[g + 1] <= off[g] || off[g] % m->bs)
				return bsg_set_error(BSG_ERR_ARG, "bsg_pcg_batch_dev: segment offsets must increase by whole block rows");
	}
	// the iterations run on a stream that can be captured: the context's
	// own, or a private one ordered after it when the context uses the
	// legacy default stream
	cudaStream_t caller = c->stream;
	cudaStream_t st = caller;
	bool priv = false;
	if (caller == nullptr || caller == cudaStreamLegacy) {
		BSG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
		priv = true;
		cudaEvent_t e;
		BSG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
		cudaEventRecord(e, caller);
		cudaStreamWaitEvent(st, e, 0);
		cudaEventDestroy(e);
	}
	c->stream = st; // library launches below go to st
	// device buffers of this call, released in restore() before the
	// private stream they are ordered on goes away
	std::vector<DevBuf> keep;
	keep.reserve(32);
	auto restore = [&](int rc) {
		keep.clear();
		if (priv) {
			cudaEvent_t e;
			if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) {
				cudaEventRecord(e, st);
				cudaStreamWaitEvent(caller, e, 0);
				cudaEventDestroy(e);
			}
			cudaStreamSynchronize(st);
			cudaStreamDestroy(st);
		}
		c->stream = caller;
		return rc;
	};

	// CUDA errors after this point restore the context's stream first
#define BCHK(call)                                                                          \
	do {                                                                                    \
		cudaError_t e_ = (call);                                                            \
		if (e_ != cudaSuccess) return restore(bsg_set_cuda_error(e_, #call, __FILE__, __LINE__)); \
	} while (0)
	auto alloc = [&](void **ptr, size_t bytes) -> int {
		keep.emplace_back();
		keep.back().s = st;
		if (cudaMallocAsync(&keep.back().p, bytes > 0 ? bytes : 1, st) != cudaSuccess)
			return bsg_set_error(BSG_ERR_NOMEM, "batched PCG buffers");
		*ptr = keep.back().p;
		return BSG_OK;
	};
	double *r = nullptr, *z = nullptr, *pp = nullptr, *q = nullptr, *t = nullptr, *w = nullptr, *sc = nullptr,
	       *part = nullptr;
	int *si = nullptr, *segid = nullptr, *dseg = nullptr, *cnt = nullptr;
	int rc = BSG_OK;
	if (!rc) rc = alloc((void **)&r, sizeof(double) * N);
	if (!rc) rc = alloc((void **)&z, sizeof(double) * N);
	if (!rc) rc = alloc((void **)&pp, sizeof(double) * N);
	if (!rc) rc = alloc((void **)&q, sizeof(double) * N);
	if (!rc) rc = alloc((void **)&t, sizeof(double) * N);
	if (!rc) rc = alloc((void **)&w, sizeof(double) * N);
	if (!rc) rc = alloc((void **)&sc, sizeof(double) * SC_N * nsys);
	if (!rc) rc = alloc((void **)&si, sizeof(int) * SI_N * nsys);
	if (!rc) rc = alloc((void **)&segid, sizeof(int) * n);
	if (!rc) rc = alloc((void **)&dseg, sizeof(int) * (nseg + 1));
	if (!rc) rc = alloc((void **)&cnt, sizeof(int) * 4);
	if (rc) return restore(rc);
	{
		std::vector<int> o32(nseg + 1);
		for (int g = 0; g <= nseg; g++) o32[g] = (int)off[g];
		BCHK(cudaMemcpyAsync(dseg, o32.data(), sizeof(int) * (nseg + 1), cudaMemcpyHostToDevice, st));
		BCHK(cudaMemsetAsync(cnt, 0, sizeof(int) * 4, st));
		BSG_COUNT(2);
		k_segid<<<ew(n), 256, 0, st>>>((int)n, nseg, dseg, segid);
		k_segcheck<<<ew(m->n), 256, 0, st>>>(m->n, m->bs, m->d_ia, m->d_ja, segid, cnt + 3);
		int bad = 0;
		BCHK(cudaMemcpyAsync(&bad, cnt + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
		BCHK(cudaStreamSynchronize(st));
		if (bad) return restore(bsg_set_error(BSG_ERR_ARG, "bsg_pcg_batch_dev: the matrix couples two segments"));
	}

	// ---- autotune on first use of this shape: reduction chunk, SpMM group
	const auto key = std::make_tuple(n, m->bs, nrhs, nseg);
	Tuned tune;
	auto it = g_tuned.find(key);
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	if (it != g_tuned.end()) {
		tune = it->second;
	} else {
		tune.chunk = 16384;
		tune.group = m->group;
		float best = 1e30f;
		const long long cands[3] = {4096, 16384, 65536};
		for (long long cand : cands) {
			Chunks ch;
			std::vector<DevBuf> kk;
			if ((rc = build_chunks(st, nrhs, nseg, off, n, cand, ch, kk))) break;
			DevBuf pb;
			pb.s = st;
			if (cudaMallocAsync(&pb.p, sizeof(double) * 2 * ch.nchunk, st) != cudaSuccess) { rc = BSG_ERR_NOMEM; break; }
			float ms = 0;
			for (int rep = 0; rep < 4; rep++) {
				if (rep == 1) cudaEventRecord(e0, st);
				k_bdots<2><<<ch.nchunk < 65535 ? ch.nchunk : 65535, 256, 0, st>>>(ch.nchunk, ch.beg, ch.end, d_B, d_B, d_X,
				                                                                  d_X, (double *)pb.p);
				k_bfinal<2><<<(nsys + 7) / 8, 256, 0, st>>>(nsys, ch.first, (double *)pb.p, sc, SC_RR, SC_GAM);
			}
			cudaEventRecord(e1, st);
			cudaEventSynchronize(e1);
			cudaEventElapsedTime(&ms, e0, e1);
			BSG_COUNT(8);
			if (ms < best) { best = ms; tune.chunk = cand; }
		}
		if (!rc && m->bs == 1 && nrhs > 1) {
			bsg_mat *mm = const_cast<bsg_mat *>(m);
			const int g0 = mm->group;
			float bestg = 1e30f;
			const int groups[4] = {4, 8, 16, 32};
			for (int G : groups) {
				mm->group = G;
				for (int rep = 0; rep < 3 && !rc; rep++) {
					if (rep == 1) cudaEventRecord(e0, st);
					rc = bsg_spmm_launch(mm, nrhs, d_B, q, n, st);
				}
				cudaEventRecord(e1, st);
				cudaEventSynchronize(e1);
				float ms = 0;
				cudaEventElapsedTime(&ms, e0, e1);
				if (ms < bestg) { bestg = ms; tune.group = G; }
			}
			mm->group = rc ? g0 : tune.group;
		}
		if (!rc) g_tuned[key] = tune;
	}
	if (!rc && m->bs == 1 && nrhs > 1) const_cast<bsg_mat *>(m)->group = tune.group;
	if (rc) {
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		return restore(rc);
	}
	if (tuned) { tuned[0] = (int)tune.chunk; tuned[1] = tune.group; }

	Chunks ch;
	if ((rc = build_chunks(st, nrhs, nseg, off, n, tune.chunk, ch, keep))) return restore(rc);
	if ((rc = alloc((void **)&part, sizeof(double) * 2 * ch.nchunk))) return restore(rc);
	const int dgrid = ch.nchunk < 65535 ? ch.nchunk : 65535;
	const int fgrid = (nsys + 7) / 8, sgrid = (nsys + 255) / 256;
	const double eps2 = p->eps * p->eps;

	auto dots2 = [&](const double *x0, const double *y0, const double *x1, const double *y1, int s0, int s1) {
		BSG_COUNT(2);
		k_bdots<2><<<dgrid, 256, 0, st>>>(ch.nchunk, ch.beg, ch.end, x0, y0, x1, y1, part);
		k_bfinal<2><<<fgrid, 256, 0, st>>>(nsys, ch.first, part, sc, s0, s1);
	};
	auto dots1 = [&](const double *x0, const double *y0, int s0) {
		BSG_COUNT(2);
		k_bdots<1><<<dgrid, 256, 0, st>>>(ch.nchunk, ch.beg, ch.end, x0, y0, nullptr, nullptr, part);
		k_bfinal<1><<<fgrid, 256, 0, st>>>(nsys, ch.first, part, sc, s0, s0);
	};
	// every right-hand side in one pass over the factor per sweep
	auto precond_all = [&](const double *src, double *dst) {
		return bsg_precond_apply_multi(c, f, p, nrhs, src, dst, t, w);
	};

	BCHK(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), st));
	BCHK(cudaMemsetAsync(pp, 0, sizeof(double) * N, st)); // p = z + 0 * p on the first step
	cudaEventRecord(e0, st);
	// r = b - A x; z = M^{-1} r; (r.r, r.z); per-system start
	if (!rc) rc = bsg_spmm_launch(m, nrhs, d_X, q, n, st);
	BSG_COUNT(1);
	k_bres<<<ew(N), 256, 0, st>>>(N, d_B, q, r);
	if (!rc) rc = precond_all(r, z);
	if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return restore(bsg_set_error(rc, "batched PCG start")); }
	dots2(r, r, r, z, SC_RR, SC_GAM);
	BSG_COUNT(1);
	k_binit<<<sgrid, 256, 0, st>>>(nsys, sc, si);

	// ---- one iteration, as launched into the graph
	const int K = 8; // iterations per graph
	auto iteration = [&]() -> int {
		BSG_COUNT(1);
		k_bp<<<ew(N), 256, 0, st>>>(N, n, nseg, segid, sc, si, z, pp);
		int e = bsg_spmm_launch(m, nrhs, pp, q, n, st);
		if (e) return e;
		dots1(pp, q, SC_PAP);
		BSG_COUNT(2);
		k_balpha<<<sgrid, 256, 0, st>>>(nsys, sc, si);
		k_bxr<<<ew(N), 256, 0, st>>>(N, n, nseg, segid, sc, pp, q, r, d_X);
		if ((e = precond_all(r, z))) return e;
		dots2(r, r, r, z, SC_RR, SC_GAM);
		BSG_COUNT(1);
		k_bbeta<<<sgrid, 256, 0, st>>>(nsys, eps2, p->niter, sc, si, cnt);
		return 0;
	};
	// The whole iteration loop is one graph: a conditional WHILE node whose
	// body is K captured iterations followed by k_bcontinue, which decides on
	// the device whether another pass runs.  The host launches the graph once
	// per solve (and once more per true-residual restart) and reads nothing
	// in between.
	cudaGraph_t graph = nullptr, body = nullptr;
	cudaGraphExec_t exec = nullptr;
	cudaGraphConditionalHandle hcond = 0;
	cudaGraphNode_t wnode = nullptr;
	const int max_replays = (p->niter + K - 1) / K + 8;
	const unsigned long long l0 = g_bsg_launches;
	cudaError_t ce = cudaGraphCreate(&graph, 0);
	if (ce == cudaSuccess) ce = cudaGraphConditionalHandleCreate(&hcond, graph, 1, cudaGraphCondAssignDefault);
	if (ce == cudaSuccess) {
		cudaGraphNodeParams cp = {};
		cp.type = cudaGraphNodeTypeConditional;
		cp.conditional.handle = hcond;
		cp.conditional.type = cudaGraphCondTypeWhile;
		cp.conditional.size = 1;
		ce = cudaGraphAddNode(&wnode, graph, nullptr, 0, &cp);
		if (ce == cudaSuccess) body = cp.conditional.phGraph_out[0];
	}
	if (ce == cudaSuccess) ce = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
	if (ce == cudaSuccess) {
		for (int k = 0; k < K && !rc; k++) rc = iteration();
		BSG_COUNT(1);
		k_bcontinue<<<1, 1, 0, st>>>(hcond, cnt, max_replays);
		cudaGraph_t captured = nullptr;
		ce = cudaStreamEndCapture(st, &captured);
	}
	const unsigned long long per_pass = g_bsg_launches - l0;
	g_bsg_launches = l0;
	if (rc || ce != cudaSuccess || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
		if (graph) cudaGraphDestroy(graph);
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		return restore(bsg_set_error(rc ? rc : BSG_ERR_CUDA, "batched PCG: graph construction failed"));
	}
	int *h_cnt = nullptr;
	BCHK(cudaMallocHost(&h_cnt, sizeof(int) * 4));
	int replays = 0, restarts = 0, status = BSG_OK;
	BCHK(cudaMemsetAsync(cnt, 0, sizeof(int) * 3, st));
	for (;;) {
		BCHK(cudaGraphLaunch(exec, st));
		BCHK(cudaMemcpyAsync(h_cnt, cnt, sizeof(int) * 3, cudaMemcpyDeviceToHost, st));
		BCHK(cudaStreamSynchronize(st));
		g_bsg_launches += per_pass * (unsigned long long)(h_cnt[2] - replays);
		replays = h_cnt[2];
		// all stopped: confirm on the FP64 true residuals, restart drifted systems
		if ((rc = bsg_spmm_launch(m, nrhs, d_X, q, n, st))) break;
		BSG_COUNT(1);
		k_bres<<<ew(N), 256, 0, st>>>(N, d_B, q, q); // q = b - A x, all right-hand sides
		dots1(q, q, SC_BB);
		BCHK(cudaMemsetAsync(cnt + 1, 0, sizeof(int), st));
		BSG_COUNT(1);
		k_brestart<<<sgrid, 256, 0, st>>>(nsys, eps2, sc, si, cnt + 1);
		BCHK(cudaMemcpyAsync(h_cnt + 1, cnt + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
		BCHK(cudaStreamSynchronize(st));
		if (h_cnt[1] == 0 || restarts >= 5 || replays >= max_replays) {
			if (h_cnt[1] != 0) status = BSG_ERR_NOCONV;
			break;
		}
		restarts++;
		// restarted systems continue from their true residual (others keep r,
		// which their zero steps leave unchanged)
		BCHK(cudaMemcpyAsync(r, q, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
		if ((rc = precond_all(r, z))) break;
		dots2(r, r, r, z, SC_RR, SC_GAM);
	}
	cudaEventRecord(e1, st);
	cudaGraphExecDestroy(exec);
	cudaGraphDestroy(graph);
	// per-system results: iterations and FP64 true relative residuals
	std::vector<double> hsc((size_t)SC_N * nsys);
	std::vector<int> hsi((size_t)SI_N * nsys);
	if (!rc) {
		if ((rc = bsg_spmm_launch(m, nrhs, d_X, q, n, st)) == 0) {
			BSG_COUNT(1);
			k_bres<<<ew(N), 256, 0, st>>>(N, d_B, q, q);
			dots2(q, q, d_B, d_B, SC_BB, SC_PAP);
			cudaMemcpyAsync(hsc.data(), sc, sizeof(double) * hsc.size(), cudaMemcpyDeviceToHost, st);
			cudaMemcpyAsync(hsi.data(), si, sizeof(int) * hsi.size(), cudaMemcpyDeviceToHost, st);
			if (cudaStreamSynchronize(st) != cudaSuccess) rc = BSG_ERR_CUDA;
		}
	}
	cudaFreeHost(h_cnt);
	float ms = 0;
	cudaEventElapsedTime(&ms, e0, e1);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (rc) return restore(bsg_set_error(rc, "batched PCG failed"));
	int maxit = 0, brk = 0;
	double maxres = 0.0;
	for (int s = 0; s < nsys; s++) {
		const double rr = hsc[(size_t)s * SC_N + SC_BB], bb = hsc[(size_t)s * SC_N + SC_PAP];
		const double rs = bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
		const int itn = hsi[(size_t)s * SI_N + SI_ITERS];
		if (iters) iters[s] = itn;
		if (res) res[s] = rs;
		if (itn > maxit) maxit = itn;
		if (rs > maxres) maxres = rs;
		brk |= hsi[(size_t)s * SI_N + SI_BREAK];
	}
	p->nitperf = maxit;
	p->resfin = maxres;
	p->timeitr = ms * 1e-3;
	if (tuned) { tuned[2] = K; tuned[3] = replays; }
	rc = restore(BSG_OK);
	if (brk) return bsg_set_error(BSG_ERR_BREAKDOWN, " Matrix is not positive definite");
	if (status) return bsg_set_error(status, "iteration limit reached");
	return rc;
}
#undef BCHK
