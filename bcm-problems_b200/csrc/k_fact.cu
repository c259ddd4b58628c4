// Second-order threshold incomplete factorisation on the GPU: IC2
// (CSMatrixR::Ich2, Bslib/ich2r.cpp:956-1195) and ILU2 (CSMatrixR::Ilu2,
// Bslib/ilu2r.cpp:1122-1395), numeric phase with the pattern decided on the
// fly exactly as the reference decides it (tau1 / tau2 / theta rules).
//
// Dependencies.  Row i needs every earlier row k whose row mask contains
// column i, C(i) = {k < i : i in mask(k)}: the rows that update i (i stored
// in k, as U or R) and the rows that dropped i (their theta compensation goes
// to i's diagonal).  C(i) is not known in advance, but it closes over
// finished rows: column i enters mask(k) only through A(k,i) != 0, or through
// an earlier row m in C(i) that stores both k and i (unless both are R
// entries -- the R x R skip of Ich2InitMask, Bslib/ich2r.cpp:202-222).  So
// C(i) is the closure of A's column i under "add the stored columns of m
// between m and i", and a member that does not store i has dropped it.
//
// Schedule (dynamic, deadlock-free).  A row enters a global FIFO queue when
// all rows of A's column i are finished (a counter per row, decremented by
// each finishing row).  A warp pops a row and tries it: it builds C(i) over
// finished rows (one member per lane, rows read with 16-byte loads); if it
// meets an unfinished member m it parks the row on m's waiter list and moves
// on; m re-queues its waiters when it finishes.  The smallest unfinished row
// always has all its dependencies finished and is queued or being tried, so
// the factorisation always progresses, and the queue order follows the
// dependency levels, so the GPU works on a whole wavefront of rows at once.
// Every spin (an empty queue slot) is bounded by globaltimer.
//
// Storage.  A finished row keeps only its stored part: the diagonal (inverse
// pivot) and the U / R entries sorted by column, in a pool, published by one
// 64-bit release store of (done | offset | length).  Dropped entries are not
// kept: their theta compensations are pushed at once into a per-row 64-bit
// fixed-point accumulator (scale set by tau2 * theta, bsg_comp_scale), whose
// integer sum does not depend on the order of the pushes.
//
// Arithmetic order (deterministic, identical to oracle/bsl_oracle.c):
// diagonal = scaled a_ii + (fixed-point sum of compensations received);
// then the updates of ascending contributors, each as fma(-l, g, f); then the
// row's own theta compensations in ascending column order.  The result does
// not depend on the schedule.  (The reference sums in its linked-list order
// instead; that changes results only at rounding level.)
//
// Output: the U part compacted into the reference layout (Ich2StoreScaleU,
// Bslib/ich2r.cpp:910-954) and each row's depth in the forward-solve
// dependency graph (the level schedule of the triangular solves).
#include "bsg_internal.cuh"
#include <cub/device/device_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#define F_U 0u
#define F_R 1u
#define F_D 2u
#define CF_COL(x) ((int)((x) & 0x3fffffffu))
#define CF_FLAG(x) ((x) >> 30)

#define FACT_WARPS 4
#define CMAX 256   // members of C(i)
#define HCAP 512   // distinct mask columns per row (power of two)
#define PFCAP 1024 // prefetched contributor entries per row
// capacities of the global-memory workspace that takes the rows that do not
// fit the shared one (about 0.7 MB per warp)
#define CMAX_BIG 8192
#define HCAP_BIG 8192
#define PFCAP_BIG 8192
#define W_EMPTY (-1)
#define W_CLOSED (-2)

// row record: bit 63 done | bits 32..62 pool offset | bits 0..15 stored length
#define REC_DONE (1ull << 63)
#define REC_OFF(r) ((long long)(((r) >> 32) & 0x7fffffffull))
#define REC_LEN(r) ((int)((r) & 0xffffull))

namespace {

struct FactArgs {
	int n, kind;
	const int *iu, *ju;          // upper pattern, diagonal first
	const double *al, *au;       // values (al == au for IC2)
	const int *it, *jt;          // static contributors: rows k < i with (k,i) stored
	const double *scll, *sclu, *diag0;
	double tau1, tau2, theta, pivmin;
	unsigned int *pool_cf;       // col | flag << 30; rows start on 4-entry boundaries
	double *pool_l, *pool_u;
	long long pool_cap;
	unsigned long long *pool_len;
	unsigned long long *rec;     // per-row record (see REC_*)
	unsigned long long *acc;     // per-row fixed-point compensation sum
	double acc_scale, acc_inv_scale;
	int *lev;
	int *nstat, *whead, *wnext;
	int *queue;
	long long qcap;
	unsigned long long *qhead, *qtail;
	int *done_count;
	bsg_devstat *st;
	unsigned long long *stats; // FACT_NSTAT counters (see bsg_fact_stats)
	unsigned char *big_ws;     // GlobWS::bytes per warp of the launch
};

// Scheduler / phase counters summed over all warps of the last factorisation.
enum { FS_TRY = 0, FS_PARK, FS_CYC_POP, FS_CYC_CLOSE, FS_CYC_BLOCKED, FS_CYC_PREF, FS_CYC_UPD, FS_CYC_FIN,
       FS_CONTRIB, FS_MASK, FS_ROUNDS, FS_CYC_PF, FS_CYC_PA, FS_CYC_PB, FS_BIG, FACT_NSTAT = 16 };
struct PhaseClock {
	unsigned long long v[FACT_NSTAT];
};

// Per-warp workspace of one row.  Rows first run in shared memory (SmemWS);
// a row whose member set, mask or a contributor segment does not fit is
// tried again by the same warp in a larger workspace in global memory
// (GlobWS), so any row up to the big capacities factors.  Both expose the
// same members; sc[] = {members, mask columns, kept columns, blocking row}.
struct SmemWS {
	static constexpr bool big = false;
	static constexpr int cmax = CMAX, hcap = HCAP, pfcap = PFCAP;
	int W[CMAX];           // members (discovery order, then sorted)
	int Wp[CMAX];          // pool index of column i in that row (stored members)
	int We[CMAX];          // pool end of that row
	unsigned char Wf[CMAX];
	int Ws[CMAX], Wps[CMAX], Wes[CMAX];
	unsigned char Wfs[CMAX];
	int Wb[CMAX + 1];      // prefetch segment bases (sorted order)
	int wset[CMAX * 2];    // membership hash of W (keys)
	int hkey[HCAP];        // column accumulator
	double hl[HCAP], hu[HCAP];
	int lst[HCAP];         // extracted slots, then sorted
	int lsts[HCAP];
	unsigned pf_cf[PFCAP]; // prefetched contributor segments
	short pf_slot[PFCAP];
	double pf_l[PFCAP], pf_u[PFCAP];
	int sc[4];
};

struct GlobWS {
	static constexpr bool big = true;
	static constexpr int cmax = CMAX_BIG, hcap = HCAP_BIG, pfcap = PFCAP_BIG;
	static constexpr size_t bytes = 8 * (2 * (size_t)HCAP_BIG + 2 * (size_t)PFCAP_BIG) +
	                                4 * (6 * (size_t)CMAX_BIG + (CMAX_BIG + 4) + 2 * (size_t)CMAX_BIG +
	                                     3 * (size_t)HCAP_BIG + PFCAP_BIG + 4) +
	                                2 * (size_t)PFCAP_BIG + 2 * (size_t)CMAX_BIG;
	double *hl, *hu, *pf_l, *pf_u;
	int *W, *Wp, *We, *Ws, *Wps, *Wes, *Wb, *wset, *hkey, *lst, *lsts, *sc;
	unsigned *pf_cf;
	short *pf_slot;
	unsigned char *Wf, *Wfs;
	__device__ explicit GlobWS(unsigned char *p) {
		hl = reinterpret_cast<double *>(p); hu = hl + HCAP_BIG;
		pf_l = hu + HCAP_BIG; pf_u = pf_l + PFCAP_BIG;
		W = reinterpret_cast<int *>(pf_u + PFCAP_BIG);
		Wp = W + CMAX_BIG; We = Wp + CMAX_BIG; Ws = We + CMAX_BIG; Wps = Ws + CMAX_BIG; Wes = Wps + CMAX_BIG;
		Wb = Wes + CMAX_BIG; wset = Wb + CMAX_BIG + 4;
		hkey = wset + 2 * CMAX_BIG; lst = hkey + HCAP_BIG; lsts = lst + HCAP_BIG;
		pf_cf = reinterpret_cast<unsigned *>(lsts + HCAP_BIG);
		sc = reinterpret_cast<int *>(pf_cf + PFCAP_BIG);
		pf_slot = reinterpret_cast<short *>(sc + 4);
		Wf = reinterpret_cast<unsigned char *>(pf_slot + PFCAP_BIG); Wfs = Wf + CMAX_BIG;
	}
};

__device__ __forceinline__ unsigned hash_u(int k) { return (unsigned)k * 2654435761u; }

// Find or insert column c; returns slot or -1 if full.
template <class WS>
__device__ int hfind_insert(WS &s, int c) {
	unsigned h = hash_u(c) & (s.hcap - 1);
	for (int probe = 0; probe < s.hcap; probe++) {
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
		h = (h + 1) & (s.hcap - 1);
	}
	return -1;
}

// Insert row k into the member set; 1 if new, 0 if present, -1 if full.
// Most candidates are already members: probe with plain reads, CAS only
// into an empty slot.
template <class WS>
__device__ int wset_insert(WS &s, int k) {
	unsigned h = hash_u(k) & (2 * s.cmax - 1);
	for (int probe = 0; probe < 2 * s.cmax; probe++) {
		int cur = s.wset[h];
		if (cur == k) return 0;
		if (cur == -1) {
			int old = atomicCAS(&s.wset[h], -1, k);
			if (old == -1) return 1;
			if (old == k) return 0;
		}
		h = (h + 1) & (2 * s.cmax - 1);
	}
	return -1;
}

// Add a nonnegative compensation to row j's 64-bit fixed-point accumulator
// (value * 2^scale_bits, truncated): integer addition makes the sum exact and
// independent of the order of the adds, and a reduction without return value
// costs no round trip.  scale_bits leaves room for 2^12 maximal terms.
__device__ void acc_push(unsigned long long *acc, int j, double comp, double scale) {
	atomicAdd(acc + j, (unsigned long long)(comp * scale));
}
__device__ double acc_value(const unsigned long long *acc, int j, double inv_scale) {
	return __dmul_rn((double)__ldcg(acc + j), inv_scale);
}

__device__ void q_push(const FactArgs &A, int row) {
	unsigned long long t = atomicAdd(A.qtail, 1ull);
	if ((long long)t >= A.qcap) {
		devstat_fail(A.st, BSG_ERR_WORKSPACE, row, 1);
		return;
	}
	atomicExch(A.queue + t, row);
}

// Pop the next queued row; -1 when the factorisation is finished or failed.
__device__ int q_pop(const FactArgs &A) {
	unsigned long long h = atomicAdd(A.qhead, 1ull);
	if ((long long)h >= A.qcap) return -1;
	int v = *(volatile int *)(A.queue + h);
	if (v >= 0) return v;
	unsigned long long t0 = globaltimer_ns();
	for (unsigned it = 1;; it++) {
		__nanosleep(64);
		v = *(volatile int *)(A.queue + h);
		if (v >= 0) return v;
		if ((it & 31) == 0) {
			if (*(volatile int *)A.done_count >= A.n) return -1;
			if (*(volatile int *)&A.st->code != 0) return -1;
			if (globaltimer_ns() - t0 > BSG_SPIN_LIMIT_NS) {
				devstat_fail(A.st, BSG_ERR_TIMEOUT, (int)h);
				return -1;
			}
		}
	}
}

// Park row i on unfinished row m (lane 0).
__device__ void park(const FactArgs &A, int i, int m) {
	for (;;) {
		int old = *(volatile int *)(A.whead + m);
		if (old == W_CLOSED) { q_push(A, i); return; }
		A.wnext[i] = old;
		__threadfence();
		if (atomicCAS(A.whead + m, old, i) == old) return;
	}
}

// Examine member m of C(i) (one lane): classify it and add its candidates.
// Returns 0, or a BSG_ERR_* code.
template <class WS>
__device__ int close_member(const FactArgs &A, WS &s, int i, int t, int m, unsigned long long rec,
                           int &levmax) {
	const long long off = REC_OFF(rec);
	const int len = REC_LEN(rec);
	const uint4 *row4 = reinterpret_cast<const uint4 *>(A.pool_cf + off);
	// pass 1: find column i among the stored entries 1..len-1 (sorted); the
	// first 32 entries stay in registers for pass 2
	uint4 v0[8];
#pragma unroll
	for (int r = 0; r < 8; r++) {
		v0[r] = make_uint4(0x3fffffffu, 0x3fffffffu, 0x3fffffffu, 0x3fffffffu);
		if (4 * r < len) v0[r] = __ldcg(row4 + r);
	}
	int pos = -1;
	unsigned fi = 0;
	bool past = false;
#pragma unroll
	for (int r = 0; r < 8; r++) {
		unsigned e4[4] = {v0[r].x, v0[r].y, v0[r].z, v0[r].w};
#pragma unroll
		for (int c4 = 0; c4 < 4; c4++) {
			const int e = 4 * r + c4;
			if (e < 1 || e >= len || past || pos >= 0) continue;
			const int c = CF_COL(e4[c4]);
			if (c == i) { pos = e; fi = CF_FLAG(e4[c4]); }
			else if (c > i) past = true;
		}
	}
	for (int q0 = 8; pos < 0 && !past && 4 * q0 < len; q0 += 8) {
		uint4 v[8];
#pragma unroll
		for (int r = 0; r < 8; r++) {
			v[r] = make_uint4(0x3fffffffu, 0x3fffffffu, 0x3fffffffu, 0x3fffffffu);
			if (4 * (q0 + r) < len) v[r] = __ldcg(row4 + q0 + r);
		}
#pragma unroll
		for (int r = 0; r < 8; r++) {
			unsigned e4[4] = {v[r].x, v[r].y, v[r].z, v[r].w};
#pragma unroll
			for (int c4 = 0; c4 < 4; c4++) {
				const int e = 4 * (q0 + r) + c4;
				if (e >= len || past || pos >= 0) continue;
				const int c = CF_COL(e4[c4]);
				if (c == i) { pos = e; fi = CF_FLAG(e4[c4]); }
				else if (c > i) past = true;
			}
		}
	}
	if (pos < 0) { // m dropped column i: compensation only, no expansion
		s.Wf[t] = (unsigned char)F_D;
		return 0;
	}
	s.Wp[t] = (int)(off + pos);
	s.We[t] = (int)(off + len);
	s.Wf[t] = (unsigned char)fi;
	if (fi == F_U) levmax = max(levmax, __ldcg(A.lev + m) + 1);
	// pass 2: the stored columns of m between m and i are members, except
	// R entries when i is R too (R x R skip)
	int err = 0;
#pragma unroll
	for (int r = 0; r < 8; r++) {
		unsigned e4[4] = {v0[r].x, v0[r].y, v0[r].z, v0[r].w};
#pragma unroll
		for (int c4 = 0; c4 < 4; c4++) {
			const int e = 4 * r + c4;
			if (e < 1 || e >= pos || err) continue;
			if (fi == F_R && CF_FLAG(e4[c4]) == F_R) continue;
			const int c = CF_COL(e4[c4]);
			const int isnew = wset_insert(s, c);
			if (isnew < 0) { err = BSG_ERR_WORKSPACE; continue; }
			if (isnew == 1) {
				int slot = atomicAdd(&s.sc[0], 1);
				if (slot < s.cmax) s.W[slot] = c; else err = BSG_ERR_WORKSPACE;
			}
		}
	}
	for (int e = 32; e < pos && !err; e++) {
		const unsigned cf = __ldcg(A.pool_cf + off + e);
		if (fi == F_R && CF_FLAG(cf) == F_R) continue;
		const int c = CF_COL(cf);
		const int isnew = wset_insert(s, c);
		if (isnew < 0) { err = BSG_ERR_WORKSPACE; continue; }
		if (isnew == 1) {
			int slot = atomicAdd(&s.sc[0], 1);
			if (slot < s.cmax) s.W[slot] = c; else err = BSG_ERR_WORKSPACE;
		}
	}
	return err;
}

// Factor row i.  Returns -1 when done, the unfinished row it waits for
// (>= 0), -2 on error (reported through the status word), or -3 when the
// row does not fit a shared-memory workspace (nothing was published yet, so
// the caller retries it in the global one).
template <class WS>
__device__ int try_row(const FactArgs &A, WS &s, int i, int lane, PhaseClock &pc) {
	const bool ilu = A.kind == 1;
	const long long c0 = clock64();
	for (int t = lane; t < 2 * s.cmax; t += 32) s.wset[t] = -1;
	for (int t = lane; t < s.hcap; t += 32) s.hkey[t] = -1;
	if (lane == 0) { s.sc[3] = -1; s.sc[0] = 0; }
	__syncwarp();

	// ---- seed with A's column i (all finished: the row was queued)
	const int tb = A.it[i], te = A.it[i + 1];
	if (te - tb > s.cmax) {
		if (!WS::big) return -3;
		if (lane == 0) devstat_fail(A.st, BSG_ERR_WORKSPACE, i, 2);
		return -2;
	}
	for (int t = tb + lane; t < te; t += 32) {
		int k = A.jt[t];
		s.W[t - tb] = k;
		wset_insert(s, k);
	}
	if (lane == 0) s.sc[0] = te - tb;
	__syncwarp();

	// ---- close C(i): rounds over the newest members, one member per lane
	int err = 0, levmax = 0;
	for (int lo = 0; lo < s.sc[0] && !err;) {
		pc.v[FS_ROUNDS]++;
		const int hi = min(s.sc[0], s.cmax);
		for (int base = lo; base < hi; base += 32) {
			const int t = base + lane;
			int m = -1;
			unsigned long long rec = 0;
			if (t < hi) {
				m = s.W[t];
				rec = ld_acquire_u64(A.rec + m);
				if (!(rec & REC_DONE)) { atomicCAS(&s.sc[3], -1, m); m = -1; }
			}
			__syncwarp();
			if (s.sc[3] >= 0) {
				pc.v[FS_CYC_BLOCKED] += clock64() - c0;
				return s.sc[3];
			}
			if (m >= 0) {
				int e2 = close_member(A, s, i, t, m, rec, levmax);
				if (e2) err = e2;
			}
			__syncwarp();
		}
		err = __reduce_min_sync(0xffffffffu, err);
		lo = hi;
		__syncwarp();
	}
	if (err) {
		if (!WS::big) return -3;
		if (lane == 0) devstat_fail(A.st, err, i, 3);
		return -2;
	}
	levmax = __reduce_max_sync(0xffffffffu, levmax);
	const int nW = s.sc[0];
	const long long c1 = clock64();
	pc.v[FS_CYC_CLOSE] += c1 - c0;
	pc.v[FS_CONTRIB] += nW;

	// ---- sort members ascending (rank sort; rows are distinct)
	for (int t = lane; t < nW; t += 32) {
		int k = s.W[t], r = 0;
		for (int u = 0; u < nW; u++) r += s.W[u] < k;
		s.Ws[r] = k; s.Wps[r] = s.Wp[t]; s.Wes[r] = s.We[t]; s.Wfs[r] = s.Wf[t];
	}
	__syncwarp();

	// ---- segment bases: stored member t contributes its entries [pos, end)
	if (lane == 0) {
		int b = 0;
		for (int t = 0; t < nW; t++) {
			s.Wb[t] = b;
			if (s.Wfs[t] != F_D) b += s.Wes[t] - s.Wps[t];
		}
		s.Wb[nW] = b;
	}
	const double comp = acc_value(A.acc, i, A.acc_inv_scale);
	__syncwarp();
	const long long c2 = clock64();
	pc.v[FS_CYC_PREF] += c2 - c1;

	// ---- init the scaled row (Ich2InitRow / Ilu2InitRow); the diagonal gets
	//      the compensations of the rows that dropped column i
	const int ab = A.iu[i], ae = A.iu[i + 1];
	if (lane == 0) {
		int slot = hfind_insert(s, i);
		const double d = __dadd_rn(A.diag0[i], comp);
		s.hl[slot] = d;
		s.hu[slot] = d;
	}
	__syncwarp();
	{
		const double si_l = A.scll[i], si_u = A.sclu[i];
		for (int k = ab + 1 + lane; k < ae; k += 32) {
			int j = A.ju[k];
			int sl = hfind_insert(s, j);
			if (sl < 0) { err = BSG_ERR_WORKSPACE; continue; }
			if (ilu) {
				s.hl[sl] = __dmul_rn(__dmul_rn(A.al[k], si_u), A.scll[j]);
				s.hu[sl] = __dmul_rn(__dmul_rn(A.au[k], si_l), A.sclu[j]);
			} else {
				double v = __dmul_rn(__dmul_rn(A.al[k], si_l), A.scll[j]);
				s.hl[sl] = v;
				s.hu[sl] = v;
			}
		}
		err = __reduce_min_sync(0xffffffffu, err);
		__syncwarp();
	}

	// ---- updates from the stored members in ascending order, in groups of
	//      consecutive members whose segments fit the shared prefetch buffer
	for (int t0 = 0; t0 < nW && !err;) {
		int t1 = t0;
		while (t1 < nW && s.Wb[t1 + 1] - s.Wb[t0] <= s.pfcap) t1++;
		if (t1 == t0) { // one segment longer than the buffer
			if (!WS::big) return -3;
			if (lane == 0) devstat_fail(A.st, BSG_ERR_WORKSPACE, i, 5);
			return -2;
		}
		const int gb = s.Wb[t0], npf = s.Wb[t1] - gb;
		long long g0 = clock64();
		// prefetch: 4 independent loads per lane in flight
		for (int f0 = 0; f0 < npf; f0 += 128) {
			unsigned c4[4];
			double l4[4], u4[4];
#pragma unroll
			for (int r = 0; r < 4; r++) {
				const int f = f0 + r * 32 + lane;
				c4[r] = 0; l4[r] = 0; u4[r] = 0;
				if (f < npf) {
					// owner: the last member with Wb <= entry (dropped members have empty segments)
					int lo = t0, hi = t1 - 1;
					while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (s.Wb[mid] <= gb + f) lo = mid; else hi = mid - 1; }
					const long long g = (long long)s.Wps[lo] + (gb + f - s.Wb[lo]);
					c4[r] = __ldcg(A.pool_cf + g);
					l4[r] = __ldcg(A.pool_l + g);
					if (ilu) u4[r] = __ldcg(A.pool_u + g);
				}
			}
#pragma unroll
			for (int r = 0; r < 4; r++) {
				const int f = f0 + r * 32 + lane;
				if (f < npf) { s.pf_cf[f] = c4[r]; s.pf_l[f] = l4[r]; s.pf_u[f] = u4[r]; }
			}
		}
		__syncwarp();
		long long g1 = clock64();
		pc.v[FS_CYC_PF] += g1 - g0;
		// phase A: accumulator slot of every entry, in parallel (R x R gets none)
		for (int f = lane; f < npf; f += 32) {
			int lo = t0, hi = t1 - 1;
			while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (s.Wb[mid] <= gb + f) lo = mid; else hi = mid - 1; }
			const unsigned cf = s.pf_cf[f];
			short sl = -1;
			if (!(s.Wfs[lo] == F_R && CF_FLAG(cf) == F_R)) {
				int h = hfind_insert(s, CF_COL(cf));
				if (h < 0) err = BSG_ERR_WORKSPACE; else sl = (short)h;
			}
			s.pf_slot[f] = sl;
		}
		err = __reduce_min_sync(0xffffffffu, err);
		__syncwarp();
		long long g2 = clock64();
		pc.v[FS_CYC_PA] += g2 - g1;
		// phase B: ascending members, fma(-l, g, f) per column
		for (int t = t0; t < t1 && !err; t++) {
			if (s.Wfs[t] == F_D) continue;
			const int b = s.Wb[t] - gb, seg = s.Wb[t + 1] - s.Wb[t];
			const double lel = s.pf_l[b];
			const double uel = ilu ? s.pf_u[b] : lel;
			for (int e = lane; e < seg; e += 32) {
				const int sl = s.pf_slot[b + e];
				if (sl < 0) continue;
				if (ilu) {
					s.hl[sl] = fma(-uel, s.pf_l[b + e], s.hl[sl]);
					s.hu[sl] = fma(-lel, s.pf_u[b + e], s.hu[sl]);
				} else {
					double v = fma(-lel, s.pf_l[b + e], s.hl[sl]);
					s.hl[sl] = v;
					s.hu[sl] = v;
				}
			}
			__syncwarp();
		}
		pc.v[FS_CYC_PB] += clock64() - g2;
		t0 = t1;
		__syncwarp();
	}
	err = __reduce_min_sync(0xffffffffu, err);
	if (err) {
		if (!WS::big) return -3;
		if (lane == 0) devstat_fail(A.st, err, i, 4);
		return -2;
	}
	const long long c3 = clock64();
	pc.v[FS_CYC_UPD] += c3 - c2;

	// ---- extract the off-diagonal mask columns and sort them ascending
	if (lane == 0) s.sc[1] = 0;
	__syncwarp();
	for (int h = lane; h < s.hcap; h += 32) {
		int c = s.hkey[h];
		bool take = c >= 0 && c != i;
		unsigned b = __ballot_sync(0xffffffffu, take);
		int base = s.sc[1];
		if (take) s.lst[base + __popc(b & ((1u << lane) - 1))] = h;
		__syncwarp();
		if (lane == 0) s.sc[1] = base + __popc(b);
		__syncwarp();
	}
	const int nl = s.sc[1];
	for (int t = lane; t < nl; t += 32) {
		int c = s.hkey[s.lst[t]], r = 0;
		for (int u = 0; u < nl; u++) r += s.hkey[s.lst[u]] < c;
		s.lsts[r] = s.lst[t];
	}
	__syncwarp();
	const int di = hfind_insert(s, i); // existing slot of the diagonal

	// ---- filter by tau2 with theta compensation (ascending columns); the
	//      kept columns are listed in lst[] in ascending order
	if (lane == 0) {
		double dl = s.hl[di], du = s.hu[di];
		int nk = 0;
		for (int t = 0; t < nl; t++) {
			int h = s.lsts[t];
			double v = fabs(s.hl[h]);
			if (ilu) v = fmax(v, fabs(s.hu[h]));
			if (!(v >= A.tau2)) {
				v = __dmul_rn(v, A.theta);
				dl = __dadd_rn(dl, v);
				du = __dadd_rn(du, v);
			} else {
				s.lst[nk++] = h;
			}
		}
		s.hl[di] = dl;
		s.hu[di] = du;
		s.sc[2] = nk;
	}
	__syncwarp();
	const int nk = s.sc[2];

	// ---- pivot (Ich2PivScaleRow / Ilu2PivScaleRow)
	const double fd = s.hl[di];
	double deleml, delemu;
	if (!ilu) {
		if (!(fd > 0.0)) {
			if (lane == 0) devstat_fail(A.st, BSG_ERR_PIVOT, i);
			return -2;
		}
		deleml = delemu = 1.0 / sqrt(fd);
	} else {
		double m = fabs(fd);
		if (m < A.pivmin) m = A.pivmin;
		deleml = 1.0 / sqrt(m);
		delemu = fd < 0.0 ? -deleml : deleml;
	}

	// ---- store the stored part: diagonal, then the kept columns ascending
	const int len = nk + 1;
	const int alloc = (len + 3) & ~3;
	long long off = 0;
	if (lane == 0) off = (long long)atomicAdd(A.pool_len, (unsigned long long)alloc);
	off = __shfl_sync(0xffffffffu, off, 0);
	if (off + alloc > A.pool_cap || len > 0xffff) {
		if (lane == 0) devstat_fail(A.st, BSG_ERR_WORKSPACE, i, 6);
		return -2;
	}
	if (lane == 0) {
		A.pool_cf[off] = (unsigned)i | (F_U << 30);
		A.pool_l[off] = deleml;
		if (ilu) A.pool_u[off] = delemu;
	}
	for (int t = lane; t < nk; t += 32) {
		const int h = s.lst[t];
		double l = s.hl[h], u = s.hu[h];
		if (ilu) { l = __dmul_rn(l, delemu); u = __dmul_rn(u, deleml); } else { l = __dmul_rn(l, deleml); u = l; }
		double w = fabs(l);
		if (ilu) w = fmax(w, fabs(u));
		const unsigned flag = (w >= A.tau1) ? F_U : F_R;
		A.pool_cf[off + 1 + t] = (unsigned)s.hkey[h] | (flag << 30);
		A.pool_l[off + 1 + t] = l;
		if (ilu) A.pool_u[off + 1 + t] = u;
	}
	// ---- hand the dropped entries' compensations to their rows
	for (int t = lane; t < nl; t += 32) {
		const int h = s.lsts[t];
		double v = fabs(s.hl[h]);
		if (ilu) v = fmax(v, fabs(s.hu[h]));
		if (!(v >= A.tau2)) acc_push(A.acc, s.hkey[h], __dmul_rn(v, A.theta), A.acc_scale);
	}
	if (lane == 0) A.lev[i] = levmax;
	__threadfence();
	__syncwarp();
	if (lane == 0) st_release_u64(A.rec + i, REC_DONE | ((unsigned long long)off << 32) | (unsigned long long)len);
	__syncwarp();

	// ---- wake parked rows, release A-successors, count
	if (lane == 0) {
		__threadfence();
		int w = atomicExch(A.whead + i, W_CLOSED);
		while (w >= 0) {
			int nx = *(volatile int *)(A.wnext + w);
			q_push(A, w);
			w = nx;
		}
	}
	for (int k = ab + 1 + lane; k < ae; k += 32) {
		int j = A.ju[k];
		if (atomicSub(A.nstat + j, 1) == 1) q_push(A, j);
	}
	__syncwarp();
	if (lane == 0) {
		__threadfence();
		atomicAdd(A.done_count, 1);
	}
	pc.v[FS_CYC_FIN] += clock64() - c3;
	pc.v[FS_MASK] += nl;
	return -1;
}

__global__ void __launch_bounds__(FACT_WARPS * 32) k_fact_rows(FactArgs A) {
	extern __shared__ unsigned char smem_raw[];
	const int warp = threadIdx.x >> 5;
	SmemWS &s = reinterpret_cast<SmemWS *>(smem_raw)[warp];
	GlobWS g(A.big_ws + (size_t)(blockIdx.x * FACT_WARPS + warp) * GlobWS::bytes);
	const int lane = threadIdx.x & 31;
	PhaseClock pc;
#pragma unroll
	for (int k = 0; k < FACT_NSTAT; k++) pc.v[k] = 0;
	for (;;) {
		int i = 0;
		const long long t0 = clock64();
		if (lane == 0) i = q_pop(A);
		i = __shfl_sync(0xffffffffu, i, 0);
		pc.v[FS_CYC_POP] += clock64() - t0;
		if (i < 0) break;
		pc.v[FS_TRY]++;
		int r = try_row(A, s, i, lane, pc);
		if (r == -3) {
			pc.v[FS_BIG]++;
			__syncwarp();
			r = try_row(A, g, i, lane, pc);
		}
		if (r == -2) break;
		if (r >= 0) {
			pc.v[FS_PARK]++;
			if (lane == 0) park(A, i, r);
		}
		__syncwarp();
	}
	if (lane == 0 && A.stats) {
#pragma unroll
		for (int k = 0; k < FACT_NSTAT; k++)
			if (pc.v[k]) atomicAdd(A.stats + k, pc.v[k]);
	}
}

// Per-row scheduler state (counts of unfinished rows of A's column i).
__global__ void k_fact_init(int n, const int *it, int *nstat, int *whead, unsigned long long *rec,
                            unsigned long long *acc, int *lev) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	nstat[i] = it[i + 1] - it[i];
	whead[i] = W_EMPTY;
	rec[i] = 0;
	acc[i] = 0;
	lev[i] = 0;
}
// Initial queue: the rows with no static contributor.
__global__ void k_fact_seed(FactArgs A) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < A.n && A.it[i + 1] == A.it[i]) q_push(A, i);
}
__global__ void k_fill_int(long long n, int *p, int v) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		p[i] = v;
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
		diag0[i] = __dmul_rn(__dmul_rn(d, s), s);
	} else {
		double m = fabs(d);
		if (m < sclmin) m = sclmin;
		m = 1.0 / sqrt(m);
		scll[i] = m;
		sclu[i] = d < 0.0 ? m : -m;
		diag0[i] = __dmul_rn(__dmul_rn(d, scll[i]), sclu[i]);
	}
}

__global__ void k_count_u(int n, const unsigned long long *rec, const unsigned *cf, int *cnt, int *cntr) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const long long off = REC_OFF(rec[i]);
	const int len = REC_LEN(rec[i]);
	int c = 0, r = 0;
	for (long long e = off; e < off + len; e++) {
		unsigned f = CF_FLAG(cf[e]);
		c += f == F_U;
		r += f == F_R;
	}
	cnt[i] = c;
	cntr[i] = r;
}

__global__ void k_emit_u(int n, int kind, const unsigned long long *rec, const unsigned *cf, const double *pl,
                         const double *pu, const double *scll, const double *sclu, const int *iu_out, int *ju,
                         double *l, double *u) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const long long off = REC_OFF(rec[i]);
	const int len = REC_LEN(rec[i]);
	int z = iu_out[i];
	for (long long e = off; e < off + len; e++) {
		unsigned x = cf[e];
		if (CF_FLAG(x) != F_U) continue;
		int j = CF_COL(x);
		ju[z] = j;
		if (j == i) {
			l[z] = __dmul_rn(pl[e], scll[i]);
			u[z] = __dmul_rn(kind == 1 ? pu[e] : pl[e], sclu[i]);
		} else {
			l[z] = __ddiv_rn(pl[e], scll[j]);
			u[z] = __ddiv_rn(kind == 1 ? pu[e] : pl[e], sclu[j]);
		}
		z++;
	}
}

__global__ void k_level_keys(int n, const int *lev, unsigned long long *keys, int *vals) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	keys[i] = ((unsigned long long)(unsigned)lev[i] << 32) | (unsigned)i;
	vals[i] = i;
}

inline int nb(long long n, int t) { return n > 0 ? (int)((n + t - 1) / t) : 1; }

} // namespace

int bsg_fct_finish(bsg_ctx *c, bsg_fct *f);

// Scale of the fixed-point compensation sums: a compensation is below
// tau2 * theta < 2^e, so 2^(51 - e) leaves room for 2^12 maximal terms in 63
// bits; the rule is exact (frexp) so the oracle derives the same scale.
void bsg_comp_scale(double tau2, double theta, double *scale, double *inv_scale) {
	int e = -13;
	double maxterm = tau2 * theta;
	if (maxterm > 0.0) frexp(maxterm, &e);
	int bits = 51 - e;
	if (bits > 1000) bits = 1000;
	*scale = ldexp(1.0, bits);
	*inv_scale = ldexp(1.0, -bits);
}

static unsigned long long g_fact_stats[FACT_NSTAT];

// Counters of the last factorisation in this process: [0] row tries,
// [1] parks, [2..7] SM cycles summed over warps in queue wait, closure,
// blocked closures, prefetch, updates, finish; [8] members of C(i),
// [9] mask columns, [10] closure rounds, [11..13] SM cycles in prefetch,
// slot resolution and fma phases, [14] rows retried in the global-memory
// workspace, [15] warps launched.
extern "C" int bsg_fact_stats(unsigned long long *out, int nout) {
	for (int k = 0; k < nout && k < FACT_NSTAT; k++) out[k] = g_fact_stats[k];
	return BSG_OK;
}

// Runs the factorisation of m (whose upper split d_iu/d_ju/d_al/d_au and
// static contributor lists d_it/d_jt are prepared) and builds the factor.
int bsg_fact_run(bsg_ctx *c, bsg_mat *m, int kind, const bsg_param *p, bsg_fct **out) {
	const int n = m->n * m->bs; // point rows (block matrices factor their point expansion)
	cudaStream_t st = c->stream;
	double mem = p->memory < 0 ? -p->memory : p->memory;
	if (mem < 8.0) mem = 8.0;
	// the pool holds U + R entries padded to 4-entry rows
	long long cap = (long long)(mem * 2.0 * (double)m->nnz_up) + 8LL * n + 1024;
	if (cap > 0x7ffffff0LL) cap = 0x7ffffff0LL; // pool offsets are 31-bit
	const long long qcap = 8LL * n + 65536;
	double *scll, *sclu, *diag0, *pl, *pu = nullptr;
	unsigned *cf;
	unsigned long long *rec, *acc;
	int *lev, *nstat, *whead, *wnext, *queue, *done_count;
	unsigned long long *pool_len, *qhead, *qtail;
	BSG_CUDA(cudaMallocAsync(&scll, sizeof(double) * n, st));
	BSG_CUDA(cudaMallocAsync(&sclu, sizeof(double) * n, st));
	BSG_CUDA(cudaMallocAsync(&diag0, sizeof(double) * n, st));
	if (cudaMallocAsync(&cf, sizeof(unsigned) * cap, st) != cudaSuccess) return bsg_set_error(BSG_ERR_NOMEM, "factor pool");
	if (cudaMallocAsync(&pl, sizeof(double) * cap, st) != cudaSuccess) return bsg_set_error(BSG_ERR_NOMEM, "factor pool");
	if (kind == 1 && cudaMallocAsync(&pu, sizeof(double) * cap, st) != cudaSuccess)
		return bsg_set_error(BSG_ERR_NOMEM, "factor pool");
	BSG_CUDA(cudaMallocAsync(&rec, sizeof(unsigned long long) * n, st));
	BSG_CUDA(cudaMallocAsync(&acc, sizeof(unsigned long long) * n, st));
	BSG_CUDA(cudaMallocAsync(&lev, sizeof(int) * n, st));
	BSG_CUDA(cudaMallocAsync(&nstat, sizeof(int) * n, st));
	BSG_CUDA(cudaMallocAsync(&whead, sizeof(int) * n, st));
	BSG_CUDA(cudaMallocAsync(&wnext, sizeof(int) * n, st));
	BSG_CUDA(cudaMallocAsync(&queue, sizeof(int) * qcap, st));
	BSG_CUDA(cudaMallocAsync(&done_count, sizeof(int), st));
	BSG_CUDA(cudaMallocAsync(&pool_len, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMallocAsync(&qhead, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMallocAsync(&qtail, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMemsetAsync(pool_len, 0, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMemsetAsync(qhead, 0, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMemsetAsync(qtail, 0, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMemsetAsync(done_count, 0, sizeof(int), st));
	BSG_CUDA(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), st));

	cudaEventRecord(c->ev0, st);
	// scale, init, queue fill, seed, rows, count, emit, level keys (+ CUB scans/sorts)
	BSG_COUNT(8);
	k_fact_scale<<<nb(n, 256), 256, 0, st>>>(n, kind, m->d_iu, m->d_ju, m->d_al, p->sclmin, scll, sclu, diag0, c->d_stat);
	k_fact_init<<<nb(n, 256), 256, 0, st>>>(n, m->d_it, nstat, whead, rec, acc, lev);
	k_fill_int<<<BSG_SMS * 4, 256, 0, st>>>(qcap, queue, -1);
	FactArgs A;
	A.n = n; A.kind = kind;
	A.iu = m->d_iu; A.ju = m->d_ju; A.al = m->d_al; A.au = m->d_au;
	A.it = m->d_it; A.jt = m->d_jt;
	A.scll = scll; A.sclu = sclu; A.diag0 = diag0;
	A.tau1 = p->tau1; A.tau2 = p->tau2; A.theta = p->theta; A.pivmin = p->pivmin;
	A.pool_cf = cf; A.pool_l = pl; A.pool_u = pu; A.pool_cap = cap; A.pool_len = pool_len;
	A.rec = rec; A.acc = acc; A.lev = lev;
	bsg_comp_scale(p->tau2, p->theta, &A.acc_scale, &A.acc_inv_scale);
	A.nstat = nstat; A.whead = whead; A.wnext = wnext; A.queue = queue; A.qcap = qcap;
	A.qhead = qhead; A.qtail = qtail; A.done_count = done_count; A.st = c->d_stat;
	BSG_CUDA(cudaMallocAsync(&A.stats, sizeof(unsigned long long) * FACT_NSTAT, st));
	BSG_CUDA(cudaMemsetAsync(A.stats, 0, sizeof(unsigned long long) * FACT_NSTAT, st));
	k_fact_seed<<<nb(n, 256), 256, 0, st>>>(A);
	size_t smem = sizeof(SmemWS) * FACT_WARPS;
	BSG_CUDA(cudaFuncSetAttribute(k_fact_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	int per_sm = 0;
	BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fact_rows, FACT_WARPS * 32, smem));
	if (per_sm < 1) per_sm = 1;
	int grid = per_sm * BSG_SMS;
	int need = (n + FACT_WARPS - 1) / FACT_WARPS;
	if (grid > need) grid = need;
	if (grid < 1) grid = 1;
	if (cudaMallocAsync(&A.big_ws, GlobWS::bytes * (size_t)grid * FACT_WARPS, st) != cudaSuccess)
		return bsg_set_error(BSG_ERR_NOMEM, "factor row workspace");
	k_fact_rows<<<grid, FACT_WARPS * 32, smem, st>>>(A);
	BSG_CUDA(cudaGetLastError());
	int rc = bsg_check_devstat(c);
	cudaMemcpyAsync(g_fact_stats, A.stats, sizeof(g_fact_stats), cudaMemcpyDeviceToHost, st);
	cudaStreamSynchronize(st);
	g_fact_stats[FACT_NSTAT - 1] = (unsigned long long)grid * FACT_WARPS; // warps launched
	cudaFreeAsync(A.stats, st);
	cudaFreeAsync(A.big_ws, st);
	int ndone = 0;
	if (!rc) {
		BSG_CUDA(cudaMemcpy(&ndone, done_count, sizeof(int), cudaMemcpyDeviceToHost));
		if (ndone != n) rc = bsg_set_error(BSG_ERR_TIMEOUT, "factorisation scheduler stopped early");
	}
	auto release = [&]() {
		for (void *q : {(void *)scll, (void *)sclu, (void *)diag0, (void *)cf, (void *)pl, (void *)pu, (void *)rec,
		                (void *)acc, (void *)lev, (void *)nstat, (void *)whead, (void *)wnext, (void *)queue,
		                (void *)done_count, (void *)pool_len, (void *)qhead, (void *)qtail})
			if (q) cudaFreeAsync(q, st);
	};
	if (rc) {
		release();
		return rc;
	}

	// ---- compact U into the reference layout
	bsg_fct *f = new bsg_fct();
	f->ctx = c; f->n = n; f->bs = 1; f->kind = kind;
	int *cnt, *cntr, *iu, *iur;
	BSG_CUDA(cudaMallocAsync(&cnt, sizeof(int) * (n + 1), st));
	BSG_CUDA(cudaMallocAsync(&cntr, sizeof(int) * (n + 1), st));
	BSG_CUDA(cudaMallocAsync(&iu, sizeof(int) * (n + 1), st));
	BSG_CUDA(cudaMallocAsync(&iur, sizeof(int) * (n + 1), st));
	BSG_CUDA(cudaMemsetAsync(cnt + n, 0, sizeof(int), st));
	BSG_CUDA(cudaMemsetAsync(cntr + n, 0, sizeof(int), st));
	k_count_u<<<nb(n, 256), 256, 0, st>>>(n, rec, cf, cnt, cntr);
	size_t tmp = 0;
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, iu, n + 1, st));
	void *d_tmp;
	BSG_CUDA(cudaMallocAsync(&d_tmp, tmp, st));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, cnt, iu, n + 1, st));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, cntr, iur, n + 1, st));
	int nzu = 0, nzr = 0;
	BSG_CUDA(cudaMemcpyAsync(&nzu, iu + n, sizeof(int), cudaMemcpyDeviceToHost, st));
	BSG_CUDA(cudaMemcpyAsync(&nzr, iur + n, sizeof(int), cudaMemcpyDeviceToHost, st));
	BSG_CUDA(cudaStreamSynchronize(st));
	f->nnz = nzu;
	f->d_iu = iu;
	BSG_CUDA(cudaMallocAsync(&f->d_ju, sizeof(int) * nzu, st));
	BSG_CUDA(cudaMallocAsync(&f->d_l, sizeof(double) * nzu, st));
	BSG_CUDA(cudaMallocAsync(&f->d_u, sizeof(double) * nzu, st));
	k_emit_u<<<nb(n, 256), 256, 0, st>>>(n, kind, rec, cf, pl, pu, scll, sclu, iu, f->d_ju, f->d_l, f->d_u);
	BSG_CUDA(cudaGetLastError());
	// level schedule of the triangular solves: rows by (forward level, index)
	{
		unsigned long long *keys, *k2;
		int *vals;
		BSG_CUDA(cudaMallocAsync(&keys, sizeof(unsigned long long) * n, st));
		BSG_CUDA(cudaMallocAsync(&k2, sizeof(unsigned long long) * n, st));
		BSG_CUDA(cudaMallocAsync(&vals, sizeof(int) * n, st));
		BSG_CUDA(cudaMallocAsync(&f->d_perm, sizeof(int) * n, st));
		k_level_keys<<<nb(n, 256), 256, 0, st>>>(n, lev, keys, vals);
		size_t t2 = 0;
		BSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t2, keys, k2, vals, f->d_perm, n, 0, 64, st));
		void *d_t2;
		BSG_CUDA(cudaMallocAsync(&d_t2, t2 > 0 ? t2 : 1, st));
		BSG_CUDA(cub::DeviceRadixSort::SortPairs(d_t2, t2, keys, k2, vals, f->d_perm, n, 0, 64, st));
		unsigned long long last = 0;
		if (n > 0) BSG_CUDA(cudaMemcpyAsync(&last, k2 + n - 1, sizeof(last), cudaMemcpyDeviceToHost, st));
		BSG_CUDA(cudaStreamSynchronize(st));
		f->levels_l = f->levels_u = n > 0 ? (int)(last >> 32) + 1 : 0;
		cudaFreeAsync(keys, st); cudaFreeAsync(vals, st); cudaFreeAsync(k2, st); cudaFreeAsync(d_t2, st);
	}
	cudaEventRecord(c->ev1, st);
	f->density = (double)nzu / (double)m->nnz_up;
	f->density2 = (double)nzr / (double)m->nnz_up;
	cudaFreeAsync(cnt, st); cudaFreeAsync(cntr, st); cudaFreeAsync(iur, st); cudaFreeAsync(d_tmp, st);
	release();
	rc = bsg_fct_finish(c, f);
	if (rc) return rc;
	*out = f;
	return BSG_OK;
}
