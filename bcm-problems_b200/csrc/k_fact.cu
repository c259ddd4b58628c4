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
// every row of A's column i has been claimed by a warp (a counter per row,
// decremented when such a row is first claimed).  A warp pops a row and tries it: it builds C(i) over
// finished rows (one member per lane, rows read with 16-byte loads).  An
// unfinished member m that another warp is computing is waited for; a member
// nobody is computing parks the row on m's waiter list and the warp moves on;
// m re-queues its waiters when it finishes.  Waits only go from a row to a
// smaller row that a running warp holds, so every chain of waits ends at a
// warp that is computing; the smallest unfinished row always has all its
// dependencies finished and is queued or being computed, so the
// factorisation always progresses, and the queue order follows the
// dependency levels, so the GPU works on a whole wavefront of rows at once.
// Every spin (an empty queue slot, a member being computed) is bounded by
// globaltimer.
//
// Storage.  A finished row keeps only its stored part: the diagonal (inverse
// pivot; the column field of that entry holds the row's forward-solve depth)
// and the U / R entries sorted by column, in a pool, published by one
// 64-bit release store of (done | offset | length).  Dropped entries are not
// kept: their theta compensations are pushed at once into a per-row 64-bit
// fixed-point accumulator (scale set by tau2 * theta, bsg_comp_scale), whose
// integer sum does not depend on the order of the pushes.
//
// Arithmetic order (deterministic, identical to oracle/bsl_oracle.c): the
// scaled row, then the updates of ascending contributors, each as
// fma(-l, g, f); then the diagonal gets the fixed-point sum of the
// compensations received; then the row's own theta compensations in
// ascending column order.  The result does
// not depend on the schedule.  (The reference sums in its linked-list order
// instead; that changes results only at rounding level.)
//
// Output: the U part compacted into the reference layout (Ich2StoreScaleU,
// Bslib/ich2r.cpp:910-954) and each row's depth in the forward-solve
// dependency graph (the level schedule of the triangular solves).
#include "bsg_internal.cuh"
#include "bsg_blk3.cuh"
#include <cub/device/device_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#define F_U 0u
#define F_R 1u
#define F_D 2u
#define CF_COL(x) ((int)((x) & 0x3fffffffu))
#define CF_FLAG(x) ((x) >> 30)

#ifndef FACT_WARPS
#define FACT_WARPS 4
#endif
#ifndef FACT_MINB
#define FACT_MINB 2 // blocks per SM the registers must allow
#endif
#define CMAX 128   // members of C(i)
#define HCAP 256   // distinct mask columns per row (power of two)
#ifndef PFCAP
#define PFCAP 256  // prefetched contributor entries per row
#endif
// capacities of the global-memory workspaces that take the rows that do not
// fit the shared one (about 0.7 MB each), and how many there are
#define BIG_SLOTS 64
#define CMAX_BIG 8192
#define HCAP_BIG 8192
#define PFCAP_BIG 8192
// members within MWIN rows below the row are kept in a bitmap (one shared
// atomic per test-and-set), farther ones in the hash
#ifndef MWIN
#define MWIN 16384
#endif
#ifndef WSETCAP
#define WSETCAP 128 // far members (hash slots, a power of two)
#endif
// block rows (3 x 3 blocks): mask columns of the shared workspace, member
// bitmap window
#define HCAP_BLK 256
#define CMAX_BLK 256
#define MWIN_BLK 8192
#define FACT_WARPS_BLK 2 // warps of a CTA in block mode (larger workspaces)
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
	int *inprog;                 // 1 while a warp is computing the row
	int *queue;
	long long qcap;
	unsigned long long *qhead, *qtail;
	int *done_count;
	bsg_devstat *st;
	unsigned long long *stats; // FACT_NSTAT counters (see bsg_fact_stats)
	unsigned char *big_ws;     // BIG_SLOTS workspaces of GlobWS<>::bytes
	int *big_owner;            // 1 while a warp holds that workspace
	int *nhold;                // warps holding their row for a member nobody computes
	int hold_max;              // at most this many (half the warps)
};

// Scheduler / phase counters summed over all warps of the last factorisation.
enum { FS_TRY = 0, FS_PARK, FS_CYC_POP, FS_CYC_CLOSE, FS_CYC_BLOCKED, FS_CYC_TAIL, FS_CYC_UPD, FS_CYC_FIN,
       FS_CONTRIB, FS_MASK, FS_ROUNDS, FS_CYC_PF, FS_CYC_PA, FS_CYC_PB, FS_BIG, FS_WARPS,
       FS_CYC_PLOAD, FS_CYC_PCLOSE, FS_CYC_TOPUB, FS_CYC_POSTPUB, FS_BATCHES, FS_CLOSED, FS_CYC_TCLOSE,
       FS_CYC_FPRE, FACT_NSTAT = 24 };
struct PhaseClock {
	unsigned long long v[FACT_NSTAT];
};

// Per-warp workspace of one row.  Rows first run in shared memory (SmemWS);
// a row whose member set, mask or a contributor segment does not fit is
// tried again by the same warp in a larger workspace in global memory
// (GlobWS), so any row up to the big capacities factors.  Both expose the
// same members; sc[] = {members, mask columns, kept columns, blocking row}.
// IC2 (ILU false) keeps one value per column: its shared workspace has no
// U-side arrays, so more warps fit on an SM.  Block rows (BLK) keep 9
// values per column (U side; ILU: then the L side at 9 (hcap + slot)) in hl
// and read their members' blocks straight from the pool.
template <bool ILU, bool BLK = false>
struct SmemWS {
	static constexpr bool big = false, ilu = ILU, blk = BLK;
	static constexpr int cmax = BLK ? CMAX_BLK : CMAX, hcap = BLK ? HCAP_BLK : HCAP, pfcap = PFCAP,
	                     wcap = WSETCAP, mwin = BLK ? MWIN_BLK : MWIN;
	int W[cmax];           // members (discovery order, then sorted)
	int Wp[cmax];          // pool index of column i in that row (stored members)
	int We[cmax];          // pool end of that row
	unsigned char Wf[cmax];
	int Ws[cmax], Wps[cmax], Wes[cmax];
	unsigned char Wfs[cmax];
	int Wb[cmax + 1];      // prefetch segment bases (sorted order)
	unsigned char Wst[cmax]; // member state: 0 not closed, 1 closed, 2 applied
	int wset[WSETCAP];     // membership hash of W (keys), members below i - mwin
	unsigned wbits[mwin > 0 ? mwin / 32 : 1]; // membership bitmap: bit i - 1 - k for member k
	int hkey[hcap];        // column accumulator
	double hl[BLK ? hcap * (ILU ? 18 : 9) : HCAP], hu[ILU && !BLK ? HCAP : 1];
	int lsts[hcap];        // selected members (updates); sorted slots (finish)
	// the updates' prefetch buffers and the finish's slot lists are never
	// live at once; Wlv (depth of a closed member) lives in a closure pass
	union {
		struct {
			unsigned pf_cf[BLK ? 1 : PFCAP]; // prefetched contributor segments
			short pf_slot[BLK ? 1 : PFCAP];
		};
		struct {
			int lst[hcap];         // extracted slots, then sorted
			int lkey[hcap];        // columns of the extracted slots
		};
		int Wlv[cmax];
	};
	double pf_l[BLK ? 1 : PFCAP], pf_u[ILU && !BLK ? PFCAP : 1];
	int sc[4];
	int slots[1];          // (the global workspace lists its slots; this one scans them)
};

template <bool ILU, bool BLK = false>
struct GlobWS {
	static constexpr bool big = true, ilu = ILU, blk = BLK;
	static constexpr int cmax = CMAX_BIG, hcap = HCAP_BIG, pfcap = PFCAP_BIG, wcap = 2 * CMAX_BIG,
	                     mwin = BLK ? MWIN_BLK : MWIN;
	static constexpr size_t nval = BLK ? 18 * (size_t)HCAP_BIG : (size_t)HCAP_BIG; // hl doubles
	static constexpr size_t bytes = 8 * (nval + (size_t)HCAP_BIG + 2 * (size_t)PFCAP_BIG) +
	                                4 * (7 * (size_t)CMAX_BIG + (CMAX_BIG + 4) + 2 * (size_t)CMAX_BIG +
	                                     4 * (size_t)HCAP_BIG + PFCAP_BIG + 4) +
	                                2 * (size_t)PFCAP_BIG + 3 * (size_t)CMAX_BIG + mwin / 8 + 4 * (size_t)HCAP_BIG;
	double *hl, *hu, *pf_l, *pf_u;
	int *W, *Wp, *We, *Ws, *Wps, *Wes, *Wlv, *Wb, *wset, *hkey, *lst, *lsts, *lkey, *sc;
	unsigned *pf_cf, *wbits;
	int *slots;            // the accumulator slots in use, in insertion order
	short *pf_slot;
	unsigned char *Wf, *Wfs, *Wst;
	__device__ explicit GlobWS(unsigned char *p) {
		hl = reinterpret_cast<double *>(p); hu = hl + nval;
		pf_l = hu + HCAP_BIG; pf_u = pf_l + PFCAP_BIG;
		W = reinterpret_cast<int *>(pf_u + PFCAP_BIG);
		Wp = W + CMAX_BIG; We = Wp + CMAX_BIG; Ws = We + CMAX_BIG; Wps = Ws + CMAX_BIG; Wes = Wps + CMAX_BIG;
		Wlv = Wes + CMAX_BIG; Wb = Wlv + CMAX_BIG; wset = Wb + CMAX_BIG + 4;
		hkey = wset + 2 * CMAX_BIG; lst = hkey + HCAP_BIG; lsts = lst + HCAP_BIG; lkey = lsts + HCAP_BIG;
		pf_cf = reinterpret_cast<unsigned *>(lkey + HCAP_BIG);
		sc = reinterpret_cast<int *>(pf_cf + PFCAP_BIG);
		pf_slot = reinterpret_cast<short *>(sc + 4);
		Wf = reinterpret_cast<unsigned char *>(pf_slot + PFCAP_BIG); Wfs = Wf + CMAX_BIG; Wst = Wfs + CMAX_BIG;
		wbits = reinterpret_cast<unsigned *>(Wst + CMAX_BIG);
		slots = reinterpret_cast<int *>(wbits + mwin / 32);
	}
};

__device__ __forceinline__ unsigned hash_u(int k) { return (unsigned)k * 2654435761u; }

// Exclusive prefix sum of v over the warp; total gets the sum.
__device__ __forceinline__ int warp_excl_scan(int v, int lane, int &total) {
	int x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const int y = __shfl_up_sync(0xffffffffu, x, o);
		if (lane >= o) x += y;
	}
	total = __shfl_sync(0xffffffffu, x, 31);
	return x - v;
}

// Index of the last segment base <= k in b[0 .. n) (b ascending, b[0] <= k).
__device__ __forceinline__ int seg_owner(const int *b, int n, int k) {
	int lo = 0, hi = n - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (b[mid] <= k) lo = mid; else hi = mid - 1;
	}
	return lo;
}

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
				if (WS::big) s.slots[atomicAdd(&s.sc[3], 1)] = (int)h;
				if (WS::blk) {
#pragma unroll
					for (int k = 0; k < 9; k++) s.hl[9 * h + k] = 0.0;
					if (WS::ilu)
#pragma unroll
						for (int k = 0; k < 9; k++) s.hl[9 * (s.hcap + h) + k] = 0.0;
				} else {
					s.hl[h] = 0.0;
					if (WS::ilu) s.hu[h] = 0.0;
				}
				return (int)h;
			}
			if (old == c) return (int)h;
		}
		h = (h + 1) & (s.hcap - 1);
	}
	return -1;
}

// Insert row k into the member set of row i; 1 if new, 0 if present, -1
// if full.  Near rows: one bit each.  Far rows: a hash; most candidates are
// already members, so probe with plain reads and CAS only into an empty slot.
template <class WS>
__device__ int wset_insert(WS &s, int i, int k) {
	const int d = i - 1 - k;
	if (d < WS::mwin) {
		const unsigned bit = 1u << (d & 31);
		if (s.wbits[d >> 5] & bit) return 0;
		return (atomicOr(&s.wbits[d >> 5], bit) & bit) ? 0 : 1;
	}
	unsigned h = hash_u(k) & (s.wcap - 1);
	for (int probe = 0; probe < s.wcap; probe++) {
		int cur = s.wset[h];
		if (cur == k) return 0;
		if (cur == -1) {
			int old = atomicCAS(&s.wset[h], -1, k);
			if (old == -1) return 1;
			if (old == k) return 0;
		}
		h = (h + 1) & (s.wcap - 1);
	}
	return -1;
}

// Ranks of keys t0 + 32 q + lane (q < NQ) among the nl distinct keys, by one
// broadcast key per step; entry t goes to position rank(t) of out.
template <int NQ>
__device__ __forceinline__ void rank_sort(const int *key_of, const int *val, int *out, int nl, int t0, int lane) {
	int key[NQ], rnk[NQ];
#pragma unroll
	for (int q = 0; q < NQ; q++) {
		const int t = t0 + q * 32 + lane;
		key[q] = t < nl ? key_of[t] : 0x7fffffff;
		rnk[q] = 0;
	}
#pragma unroll 4
	for (int u = 0; u < nl; u++) {
		const int x = key_of[u];
#pragma unroll
		for (int q = 0; q < NQ; q++) rnk[q] += x < key[q];
	}
#pragma unroll
	for (int q = 0; q < NQ; q++) {
		const int t = t0 + q * 32 + lane;
		if (t < nl) out[rnk[q]] = val[t];
	}
}

// Add a nonnegative compensation to row j's 64-bit fixed-point accumulator
// (value * 2^scale_bits, truncated): integer addition makes the sum exact and
// independent of the order of the adds, and a reduction without return value
// costs no round trip.  The sum cannot wrap: a compensation is theta * |v|
// with |v| < tau2, so below 2^51 after scaling (bsg_comp_scale), and only the
// members of C(j) push to row j, at most CMAX_BIG = 2^13 of them (a row with
// more fails with BSG_ERR_WORKSPACE), so the sum stays below 2^64.  A term
// outside that bound (it cannot occur) is reported as BSG_ERR_WORKSPACE
// rather than added.
__device__ void acc_push(unsigned long long *acc, int j, double comp, double scale, bsg_devstat *st) {
	const double t = comp * scale;
	if (!(t < 0x1p51)) {
		devstat_fail(st, BSG_ERR_WORKSPACE, j, 7);
		return;
	}
	atomicAdd(acc + j, (unsigned long long)t);
}

// The queue is a ring of qcap slots (a power of two, at least twice the
// rows): a row is in the queue at most once at a time (queued on admission,
// or re-queued once per park), so a slot is free again long before its
// ticket comes round; -1 marks a free slot.
__device__ void q_push(const FactArgs &A, int row) {
	const unsigned long long t = atomicAdd(A.qtail, 1ull);
	int *slot = A.queue + (t & (unsigned long long)(A.qcap - 1));
	const unsigned long long t0 = globaltimer_ns();
	for (unsigned it = 0; atomicCAS(slot, -1, row) != -1; it++) {
		__nanosleep(64);
		if ((it & 31) == 31 && globaltimer_ns() - t0 > BSG_SPIN_LIMIT_NS) {
			devstat_fail(A.st, BSG_ERR_WORKSPACE, row, 1);
			return;
		}
	}
}

// Pop the next queued row; -1 when the factorisation is finished or failed.
__device__ int q_pop(const FactArgs &A) {
	const unsigned long long h = atomicAdd(A.qhead, 1ull);
	int *slot = A.queue + (h & (unsigned long long)(A.qcap - 1));
	int v = atomicExch(slot, -1);
	if (v >= 0) return v;
	// the limit runs from the last finished row: an empty queue while other
	// warps still finish rows (a long chain of dependent rows) is progress
	unsigned long long t0 = globaltimer_ns();
	int seen = *(volatile int *)A.done_count;
	for (unsigned it = 1;; it++) {
		__nanosleep(64);
		if (*(volatile int *)slot >= 0) {
			v = atomicExch(slot, -1);
			if (v >= 0) return v;
		}
		if ((it & 31) == 0) {
			const int done = *(volatile int *)A.done_count;
			if (done >= A.n) return -1;
			if (*(volatile int *)&A.st->code != 0) return -1;
			if (done != seen) {
				seen = done;
				t0 = globaltimer_ns();
			} else if (globaltimer_ns() - t0 > BSG_SPIN_LIMIT_NS) {
				devstat_fail(A.st, BSG_ERR_TIMEOUT, (int)(h & 0x7fffffff));
				return -1;
			}
		}
	}
}

// Admission.  nstat[j] packs the static contributors of row j (the rows k
// < j with A(k,j) != 0) that are unfinished (bits 0..14) and unclaimed (bits
// 15..29); bit 30 marks j queued once, bit 31 claimed once.  Row j enters the
// queue when all of them are claimed and at most one is unfinished: it then
// starts while its last predecessor is being computed and waits for it.  A
// row that another row waits for is queued earlier (promoted) if nobody has
// queued it yet.  Bit 30 makes the first of the two the only one: a row is
// queued once this way, and again only when a row it parked on finishes.
#define ADM_ONE_FIN 1u
#define ADM_ONE_CLAIM (1u << 15)
#define ADM_QUEUED (1u << 30)
#define ADM_CLAIMED (1u << 31)
#ifndef BSG_ADMIT_UNFINISHED
#define BSG_ADMIT_UNFINISHED 1
#endif
__device__ __forceinline__ bool admissible(unsigned v) {
	return ((v >> 15) & 0x7fffu) == 0 && (v & 0x7fffu) <= BSG_ADMIT_UNFINISHED;
}
__device__ void enqueue_once(const FactArgs &A, int j) {
	if (!(atomicOr(reinterpret_cast<unsigned *>(A.nstat) + j, ADM_QUEUED) & ADM_QUEUED)) q_push(A, j);
}
__device__ void admit_step(const FactArgs &A, int j, unsigned delta) {
	const unsigned old = atomicSub(reinterpret_cast<unsigned *>(A.nstat) + j, delta);
	if (!admissible(old) && admissible(old - delta)) enqueue_once(A, j);
}

// Wait (lane 0) for row m while a warp is computing it: 1 once m is
// finished, 0 when nobody is computing m (the caller parks), -1 on the
// spin limit or another warp's failure.
__device__ int wait_row(const FactArgs &A, int m) {
	const unsigned long long t0 = globaltimer_ns();
	for (unsigned it = 0;; it++) {
		if (ld_acquire_u64(A.rec + m) & REC_DONE) return 1;
		if (*(volatile int *)(A.inprog + m) == 0) return (ld_acquire_u64(A.rec + m) & REC_DONE) ? 1 : 0;
		if (*(volatile int *)&A.st->code != 0) return -1;
		__nanosleep(32);
		if ((it & 63) == 63 && globaltimer_ns() - t0 > BSG_SPIN_LIMIT_NS) return -1;
	}
}

// Row m, which row i needs, is unfinished and nobody computes it (lane 0):
// queue it if it never was, then give an idle warp up to PROMOTE_WAIT_NS to
// take it.  1: m finished meanwhile; 2: a warp computes m now; 0: neither
// (the caller parks).
#define PROMOTE_WAIT_NS 20000ull
__device__ int promote(const FactArgs &A, int m) {
	enqueue_once(A, m);
	const unsigned long long t0 = globaltimer_ns();
	for (;;) {
		if (ld_acquire_u64(A.rec + m) & REC_DONE) return 1;
		if (*(volatile int *)(A.inprog + m) != 0) return 2;
		if (*(volatile int *)&A.st->code != 0 || globaltimer_ns() - t0 > PROMOTE_WAIT_NS) return 0;
		__nanosleep(64);
	}
}

// Rows queued and not yet taken by a warp (negative: warps wait for rows).
__device__ __forceinline__ long long q_backlog(const FactArgs &A) {
	return (long long)(*(volatile unsigned long long *)A.qtail - *(volatile unsigned long long *)A.qhead);
}

// Hold row i (lane 0) for member m that no warp computes right now (m is
// queued, or parked on a member of its own): spin until m is finished, for
// at most HOLD_NS, instead of parking, which would recompute row i from the
// start once m finishes.  At most hold_max warps hold at once, so the other
// half keep serving the queue and m is computed without this warp.  A warp
// holds only while no more than HOLD_BACKLOG queued rows wait for a warp:
// with rows waiting, m is taken late and this warp does better on one of
// them (many independent problems keep the queue long; a chain-limited front
// keeps it empty).  1: m finished; 0: the caller parks; -1: another warp
// failed.
#define HOLD_NS 1000000ull
#ifndef HOLD_BACKLOG
#define HOLD_BACKLOG 0
#endif
__device__ int hold_for(const FactArgs &A, int m) {
	if (q_backlog(A) > HOLD_BACKLOG) return 0;
	if (atomicAdd(A.nhold, 1) >= A.hold_max) {
		atomicSub(A.nhold, 1);
		return 0;
	}
	const unsigned long long t0 = globaltimer_ns();
	int res = 0;
	for (unsigned it = 0;; it++) {
		if (ld_acquire_u64(A.rec + m) & REC_DONE) { res = 1; break; }
		if ((it & 15) == 15) {
			if (*(volatile int *)&A.st->code != 0) { res = -1; break; }
			if (globaltimer_ns() - t0 > HOLD_NS || q_backlog(A) > HOLD_BACKLOG) break;
		}
		__nanosleep(128);
	}
	atomicSub(A.nhold, 1);
	return res;
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

// One closure pass, warp-cooperative: every unclosed member that is finished
// gets closed.  The rows of those members are flattened into 16-byte chunks
// spread over the lanes and loaded once: column i is found in each row (its
// pool index and flag, or none: the member dropped i), entry 0 carries the
// member's forward-solve depth, and the stored columns between the member
// and i (R x R skipped) are inserted into the member set, new members taking
// slots by a prefix sum.  Returns the number closed; the smallest member
// still unfinished goes to pmin, the number of members the pass discovered
// to added.
template <class WS>
__device__ int close_pass(const FactArgs &A, WS &s, int i, int lane, int &levmax, int &pmin, int &err, int &added) {
	const int nW = min(s.sc[0], s.cmax);
	added = 0;
	const unsigned lt = (1u << lane) - 1;
	int pm = 0x7fffffff;
	int nd = 0;
	// finished unclosed members: W index, pool offset, length (scratch in Ws/Wps/Wes)
	for (int base = 0; base < nW; base += 32) {
		const int t = base + lane;
		int m = -1;
		unsigned long long rec = 0;
		if (t < nW && s.Wst[t] == 0) {
			m = s.W[t];
			rec = ld_acquire_u64(A.rec + m);
		}
		const bool done = m >= 0 && (rec & REC_DONE);
		if (m >= 0 && !done) pm = min(pm, m);
		const unsigned b = __ballot_sync(0xffffffffu, done);
		if (done) {
			const int q = nd + __popc(b & lt);
			s.Ws[q] = t;
			s.Wps[q] = (int)REC_OFF(rec);
			s.Wes[q] = REC_LEN(rec);
			s.Wf[t] = (unsigned char)F_D; // until column i is found
		}
		nd += __popc(b);
	}
	pmin = __reduce_min_sync(0xffffffffu, pm);
	if (nd == 0) return 0;
	__syncwarp();
	// chunk bases of the flattened rows
	int T = 0;
	for (int d0 = 0; d0 < nd; d0 += 32) {
		const int d = d0 + lane;
		int tot;
		const int ex = warp_excl_scan(d < nd ? (s.Wes[d] + 3) >> 2 : 0, lane, tot);
		if (d < nd) s.Wb[d] = T + ex;
		T += tot;
	}
	if (lane == 0) s.Wb[nd] = T;
	__syncwarp();
	// load every chunk once (the first NREG rounds stay in registers): column
	// i and the depth
	constexpr int NREG = 4;
	uint4 reg[NREG];
	int rown[NREG];
#pragma unroll
	for (int r = 0; r < NREG; r++) {
		reg[r] = make_uint4(0u, 0u, 0u, 0u);
		rown[r] = 0;
	}
	for (int k0 = 0, r = 0; k0 < T; k0 += 32, r++) {
		const int k = k0 + lane;
		if (k >= T) continue;
		const int lo = seg_owner(s.Wb, nd, k);
		const int ch = k - s.Wb[lo], len = s.Wes[lo];
		const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(A.pool_cf + s.Wps[lo]) + ch);
		const unsigned e4[4] = {v.x, v.y, v.z, v.w};
		const int t = s.Ws[lo];
		if (ch == 0) s.Wlv[t] = CF_COL(e4[0]);
#pragma unroll
		for (int c = 0; c < 4; c++) {
			const int e = 4 * ch + c;
			if (e >= 1 && e < len && CF_COL(e4[c]) == i) {
				s.Wp[t] = s.Wps[lo] + e;
				s.Wf[t] = (unsigned char)CF_FLAG(e4[c]);
			}
		}
#pragma unroll
		for (int q = 0; q < NREG; q++)
			if (q == r) {
				reg[q] = v;
				rown[q] = lo;
			}
	}
	__syncwarp();
	// the stored columns between the member and i become members
	for (int k0 = 0, r = 0; k0 < T && !err; k0 += 32, r++) {
		const int k = k0 + lane;
		unsigned e4[4] = {0u, 0u, 0u, 0u};
		int pos = 0, ch = 0;
		unsigned fi = F_D;
		if (k < T) {
			int lo = 0;
			uint4 v = make_uint4(0u, 0u, 0u, 0u);
			if (r < NREG) {
#pragma unroll
				for (int q = 0; q < NREG; q++)
					if (q == r) {
						v = reg[q];
						lo = rown[q];
					}
			} else {
				lo = seg_owner(s.Wb, nd, k);
			}
			ch = k - s.Wb[lo];
			const int t = s.Ws[lo];
			fi = s.Wf[t];
			if (fi != F_D) {
				pos = s.Wp[t] - s.Wps[lo];
				if (4 * ch < pos) {
					if (r >= NREG) v = __ldcg(reinterpret_cast<const uint4 *>(A.pool_cf + s.Wps[lo]) + ch);
					e4[0] = v.x; e4[1] = v.y; e4[2] = v.z; e4[3] = v.w;
				}
			}
		}
		unsigned fresh = 0; // bit c: entry c is a new member
#pragma unroll
		for (int c = 0; c < 4; c++) {
			const int e = 4 * ch + c;
			if (e >= 1 && e < pos && !(fi == F_R && CF_FLAG(e4[c]) == F_R)) {
				const int isnew = wset_insert(s, i, CF_COL(e4[c]));
				if (isnew < 0) err = BSG_ERR_WORKSPACE;
				else if (isnew) fresh |= 1u << c;
			}
		}
		int tot;
		const int ex = warp_excl_scan(__popc(fresh), lane, tot);
		const int q0 = s.sc[0];
#pragma unroll
		for (int c = 0; c < 4; c++)
			if (fresh & (1u << c)) {
				const int slot = q0 + ex + __popc(fresh & ((1u << c) - 1));
				if (slot < s.cmax) { s.W[slot] = CF_COL(e4[c]); s.Wst[slot] = 0; } else err = BSG_ERR_WORKSPACE;
			}
		__syncwarp();
		if (lane == 0) s.sc[0] = q0 + tot;
		added += tot;
		__syncwarp();
		err = __reduce_min_sync(0xffffffffu, err);
	}
	// closed: pool end, state, forward-solve depth through U members
	for (int d = lane; d < nd; d += 32) {
		const int t = s.Ws[d];
		s.We[t] = s.Wps[d] + s.Wes[d];
		s.Wst[t] = 1;
		if (s.Wf[t] == F_U) levmax = max(levmax, s.Wlv[t] + 1);
	}
	__syncwarp();
	return nd;
}

// Apply the updates of the closed members below `bound` (all members below
// it are known by then) in ascending order, in groups of consecutive members
// whose segments fit the prefetch buffer; marks them applied.  Returns 0, or
// a BSG_ERR_* code (uniform over the warp).
template <class WS>
__device__ int apply_members(const FactArgs &A, WS &s, int bound, int lane, PhaseClock &pc) {
	constexpr bool ilu = WS::ilu;
	const int nW = min(s.sc[0], s.cmax);
	// compact the selected members (closed, below the bound) in index order
	if (lane == 0) s.sc[2] = 0;
	__syncwarp();
	for (int base = 0; base < nW; base += 32) {
		const int t = base + lane;
		const bool sel = t < nW && s.Wst[t] == 1 && s.W[t] < bound;
		const unsigned b = __ballot_sync(0xffffffffu, sel);
		const int pos0 = s.sc[2];
		if (sel) s.lsts[pos0 + __popc(b & ((1u << lane) - 1))] = t;
		__syncwarp();
		if (lane == 0) s.sc[2] = pos0 + __popc(b);
		__syncwarp();
	}
	const int nb = s.sc[2];
	if (nb == 0) return 0;
	pc.v[FS_BATCHES]++;
	pc.v[FS_CLOSED] += nb;
	// rank sort by row index (rows are distinct); mark applied.  Up to 32
	// members: the keys stay in registers and are broadcast by shuffles
	if (nb <= 32) {
		const int t = lane < nb ? s.lsts[lane] : 0;
		const int k = lane < nb ? s.W[t] : 0x7fffffff;
		int r = 0;
		for (int u = 0; u < nb; u++) r += __shfl_sync(0xffffffffu, k, u) < k;
		if (lane < nb) {
			s.Ws[r] = k; s.Wps[r] = s.Wp[t]; s.Wes[r] = s.We[t]; s.Wfs[r] = s.Wf[t];
			s.Wst[t] = 2;
		}
	} else {
		for (int q = lane; q < nb; q += 32) {
			const int t = s.lsts[q], k = s.W[t];
			int r = 0;
			for (int u = 0; u < nb; u++) r += s.W[s.lsts[u]] < k;
			s.Ws[r] = k; s.Wps[r] = s.Wp[t]; s.Wes[r] = s.We[t]; s.Wfs[r] = s.Wf[t];
			s.Wst[t] = 2;
		}
	}
	__syncwarp();
	// segment bases: stored member t contributes its entries [pos, end)
	{
		int run = 0;
		for (int t0 = 0; t0 < nb; t0 += 32) {
			const int t = t0 + lane;
			int tot;
			const int ex = warp_excl_scan(t < nb && s.Wfs[t] != F_D ? s.Wes[t] - s.Wps[t] : 0, lane, tot);
			if (t < nb) s.Wb[t] = run + ex;
			run += tot;
		}
		if (lane == 0) s.Wb[nb] = run;
		__syncwarp();
	}
	int err = 0;
	for (int t0 = 0; t0 < nb && !err;) {
		int t1 = t0;
		while (t1 < nb && s.Wb[t1 + 1] - s.Wb[t0] <= s.pfcap) t1++;
		if (t1 == t0) return BSG_ERR_WORKSPACE; // one segment longer than the buffer
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
					const int lo = t0 + seg_owner(s.Wb + t0, t1 - t0, gb + f);
					const long long g = (long long)s.Wps[lo] + (gb + f - s.Wb[lo]);
					c4[r] = __ldcg(A.pool_cf + g);
					l4[r] = __ldcg(A.pool_l + g);
					if (ilu) u4[r] = __ldcg(A.pool_u + g);
				}
			}
#pragma unroll
			for (int r = 0; r < 4; r++) {
				const int f = f0 + r * 32 + lane;
				if (f < npf) {
					s.pf_cf[f] = c4[r];
					s.pf_l[f] = l4[r];
					if (ilu) s.pf_u[f] = u4[r];
				}
			}
		}
		__syncwarp();
		long long g1 = clock64();
		pc.v[FS_CYC_PF] += g1 - g0;
		// phase A: accumulator slot of every entry, in parallel (R x R gets none)
		for (int f = lane; f < npf; f += 32) {
			const int lo = t0 + seg_owner(s.Wb + t0, t1 - t0, gb + f);
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
					s.hl[sl] = fma(-lel, s.pf_l[b + e], s.hl[sl]);
				}
			}
			__syncwarp();
		}
		pc.v[FS_CYC_PB] += clock64() - g2;
		t0 = t1;
		__syncwarp();
	}
	return __reduce_min_sync(0xffffffffu, err);
}


// After row i is published: release the rows of A's row i, wake the rows
// parked on i, count.
__device__ void after_publish(const FactArgs &A, int i, int lane) {
	for (int k = A.iu[i] + 1 + lane; k < A.iu[i + 1]; k += 32) admit_step(A, A.ju[k], ADM_ONE_FIN);
	if (lane == 0) {
		__threadfence();
		int w = atomicExch(A.whead + i, W_CLOSED);
		while (w >= 0) {
			int nx = *(volatile int *)(A.wnext + w);
			q_push(A, w);
			w = nx;
		}
	}
	__syncwarp();
	if (lane == 0) atomicAdd(A.done_count, 1);
}

// ---- block rows (CSMatrixRS::Ich2 / Ilu2, 3 x 3 column-major blocks) -------
// A's blocks, the scalings and the scaled diagonal blocks are 9 doubles
// each (al / au / scll / sclu / diag0); a pool entry holds a block column
// (cf) and 9 doubles in pool_l (the L side; IC2: the only side) and, for
// ILU2, pool_u.  Entry 0 of a row is the pivot scaling (pool_l = dl^T,
// pool_u = du^T) with the row's depth in its column field.

template <class WS>
__device__ __forceinline__ double *bv_u(WS &s, int h) { return s.hl + 9 * h; }
template <class WS>
__device__ __forceinline__ double *bv_l(WS &s, int h) { return s.hl + 9 * (s.hcap + h); }

// The scaled block row of A (Ilu2 / Ich2 init: scll_i A_ij scll_j^T, the
// diagonal block with its scaling done).
template <class WS>
__device__ int init_blk(const FactArgs &A, WS &s, int i, int lane) {
	int err = 0;
	if (lane == 0) {
		const int h = hfind_insert(s, i);
		double *u = bv_u(s, h);
#pragma unroll
		for (int k = 0; k < 9; k++) u[k] = __ldg(A.diag0 + 9 * (size_t)i + k);
		if (WS::ilu) {
			double *l = bv_l(s, h);
#pragma unroll
			for (int k = 0; k < 9; k++) l[k] = u[k];
		}
	}
	__syncwarp();
	const double *sli = A.scll + 9 * (size_t)i, *sui = A.sclu + 9 * (size_t)i;
	for (int k = A.iu[i] + 1 + lane; k < A.iu[i + 1]; k += 32) {
		const int j = A.ju[k];
		const int h = hfind_insert(s, j);
		if (h < 0) {
			err = BSG_ERR_WORKSPACE;
			continue;
		}
		double t[9];
		mm3(sli, 1, 3, A.au + 9 * (size_t)k, 1, 3, t);
		mm3(t, 1, 3, A.sclu + 9 * (size_t)j, 3, 1, bv_u(s, h));
		if (WS::ilu) {
			mm3(sui, 1, 3, A.al + 9 * (size_t)k, 1, 3, t);
			mm3(t, 1, 3, A.scll + 9 * (size_t)j, 3, 1, bv_l(s, h));
		}
	}
	err = __reduce_min_sync(0xffffffffu, err);
	__syncwarp();
	return err;
}

// The updates of the closed members below `bound`, ascending: member k with
// its block at column i (L: gl, U: gu) updates every block e of its row from
// column i on: f_u(c) -= gl^T gu_e, f_l(c) -= gu^T gl_e (R x R skipped).
// The lanes take the blocks of one member (distinct columns), the members
// go in order, so the sums do not depend on the schedule.
template <class WS>
__device__ int apply_blk(const FactArgs &A, WS &s, int bound, int lane, PhaseClock &pc) {
	constexpr bool ilu = WS::ilu;
	const int nW = min(s.sc[0], s.cmax);
	if (lane == 0) s.sc[2] = 0;
	__syncwarp();
	for (int base = 0; base < nW; base += 32) {
		const int t = base + lane;
		const bool sel = t < nW && s.Wst[t] == 1 && s.W[t] < bound;
		const unsigned b = __ballot_sync(0xffffffffu, sel);
		const int pos0 = s.sc[2];
		if (sel) s.lsts[pos0 + __popc(b & ((1u << lane) - 1))] = t;
		__syncwarp();
		if (lane == 0) s.sc[2] = pos0 + __popc(b);
		__syncwarp();
	}
	const int nb = s.sc[2];
	if (nb == 0) return 0;
	pc.v[FS_BATCHES]++;
	pc.v[FS_CLOSED] += nb;
	for (int q = lane; q < nb; q += 32) {
		const int t = s.lsts[q], k = s.W[t];
		int r = 0;
		for (int u = 0; u < nb; u++) r += s.W[s.lsts[u]] < k;
		s.Ws[r] = k; s.Wps[r] = s.Wp[t]; s.Wes[r] = s.We[t]; s.Wfs[r] = s.Wf[t];
		s.Wst[t] = 2;
	}
	__syncwarp();
	const double *pg_l = A.pool_l, *pg_u = ilu ? A.pool_u : A.pool_l;
	int err = 0;
	for (int t = 0; t < nb && !err; t++) {
		if (s.Wfs[t] == F_D) continue;
		const long long q = s.Wps[t], end = s.Wes[t];
		const bool rr = s.Wfs[t] == F_R;
		double lel[9], uel[9];
#pragma unroll
		for (int k = 0; k < 9; k++) {
			lel[k] = __ldcg(pg_l + 9 * q + k);
			uel[k] = ilu ? __ldcg(pg_u + 9 * q + k) : 0.0;
		}
		for (long long e = q + lane; e < end; e += 32) {
			const unsigned cf = __ldcg(A.pool_cf + e);
			if (rr && CF_FLAG(cf) == F_R) continue;
			double gu[9], gl[9];
#pragma unroll
			for (int k = 0; k < 9; k++) {
				gu[k] = __ldcg(pg_u + 9 * e + k);
				gl[k] = ilu ? __ldcg(pg_l + 9 * e + k) : 0.0;
			}
			const int h = hfind_insert(s, CF_COL(cf));
			if (h < 0) {
				err = BSG_ERR_WORKSPACE;
				continue;
			}
			double tu[9];
			mm3(lel, 3, 1, gu, 1, 3, tu); // gl_q^T gu_e
			double *u = bv_u(s, h);
#pragma unroll
			for (int k = 0; k < 9; k++) u[k] -= tu[k];
			if (ilu) {
				double tl[9];
				mm3(uel, 3, 1, gl, 1, 3, tl); // gu_q^T gl_e
				double *l = bv_l(s, h);
#pragma unroll
				for (int k = 0; k < 9; k++) l[k] -= tl[k];
			}
		}
		__syncwarp();
		err = __reduce_min_sync(0xffffffffu, err);
	}
	return err;
}

// Finish of a block row (Ilu2FiltrRow / Ilu2PivScaleRow, Bslib/ilu2rs.cpp:
// 616-852; Ich2 forms, Bslib/ich2rs.cpp:532-647): blocks of max-norm below
// tau2 are dropped, theta times their entries going to this row's pivot
// block (row sums) and to the dropped column's diagonal block (column sums,
// through its fixed-point accumulators); the pivot block with the
// compensations received from other rows takes its SVD (IC2: eigenpairs,
// a negative eigenvalue is a pivot error); the kept blocks are scaled and
// stored as U (max-norm >= tau1) or R in ascending column order.
template <class WS>
__device__ int finish_blk(const FactArgs &A, WS &s, int i, int lane, int levmax, unsigned long long accraw,
                          PhaseClock &pc, long long tail0) {
	constexpr bool ilu = WS::ilu;
	// the three received compensations (lanes 0..2)
	const double comp = __dmul_rn((double)accraw, A.acc_inv_scale);
	// ---- filter, in slot order: blocks of max-norm below tau2 are dropped,
	//      theta times their entries going to this row's pivot block (row
	//      sums, added exactly in fixed point, so their order does not
	//      matter) and to the dropped column's pivot block; the kept ones
	//      are listed in lsts / lkey
	unsigned long long rq0 = 0, rq1 = 0, rq2 = 0;
	int nl = 0;
	if (lane == 0) s.sc[2] = 0;
	__syncwarp();
	const int hscan = WS::big ? s.sc[3] : s.hcap; // slots to look at
	for (int q0 = 0; q0 < hscan; q0 += 32) { // whole warp in every round (ballots)
		const int q = q0 + lane;
		const int h = q < hscan ? (WS::big ? s.slots[q] : q) : -1;
		const int c = h >= 0 ? s.hkey[h] : -1;
		const bool take = c >= 0 && c != i;
		bool keep = false;
		if (take) {
			const double *u = bv_u(s, h), *l = ilu ? bv_l(s, h) : u;
			double a[9], mx = 0.0;
#pragma unroll
			for (int k = 0; k < 9; k++) {
				a[k] = fmax(fabs(l[k]), fabs(u[k]));
				mx = fmax(mx, a[k]);
			}
			keep = mx >= A.tau2;
			if (!keep) {
				double cs0 = 0.0, cs1 = 0.0, cs2 = 0.0;
#pragma unroll
				for (int r = 0; r < 3; r++) {
					const double v0 = A.theta * a[r], v1 = A.theta * a[r + 3], v2 = A.theta * a[r + 6];
					const unsigned long long rsum = (unsigned long long)((v0 + v1 + v2) * A.acc_scale);
					if (r == 0) rq0 += rsum; else if (r == 1) rq1 += rsum; else rq2 += rsum;
					cs0 += v0;
					cs1 += v1;
					cs2 += v2;
				}
				acc_push(A.acc, 3 * c, cs0, A.acc_scale, A.st);
				acc_push(A.acc, 3 * c + 1, cs1, A.acc_scale, A.st);
				acc_push(A.acc, 3 * c + 2, cs2, A.acc_scale, A.st);
			}
		}
		nl += __popc(__ballot_sync(0xffffffffu, take));
		const unsigned b = __ballot_sync(0xffffffffu, keep);
		const int base = s.sc[2];
		if (keep) {
			const int at = base + __popc(b & ((1u << lane) - 1));
			s.lsts[at] = h;
			s.lkey[at] = c;
		}
		__syncwarp();
		if (lane == 0) s.sc[2] = base + __popc(b);
		__syncwarp();
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		rq0 += __shfl_xor_sync(0xffffffffu, rq0, o);
		rq1 += __shfl_xor_sync(0xffffffffu, rq1, o);
		rq2 += __shfl_xor_sync(0xffffffffu, rq2, o);
	}
	const double rs0 = __dmul_rn((double)rq0, A.acc_inv_scale), rs1 = __dmul_rn((double)rq1, A.acc_inv_scale),
	             rs2 = __dmul_rn((double)rq2, A.acc_inv_scale);
	const int nk = s.sc[2];
	// ---- the kept columns ascending (rank sort): lst
	if (nk <= 32) rank_sort<1>(s.lkey, s.lsts, s.lst, nk, 0, lane);
	else if (nk <= 64) rank_sort<2>(s.lkey, s.lsts, s.lst, nk, 0, lane);
	else if (nk <= 128) rank_sort<4>(s.lkey, s.lsts, s.lst, nk, 0, lane);
	else
		for (int t0 = 0; t0 < nk; t0 += 256) rank_sort<8>(s.lkey, s.lsts, s.lst, nk, t0, lane);
	__syncwarp();
	const int di = hfind_insert(s, i);
	const double c0 = __shfl_sync(0xffffffffu, comp, 0), c1 = __shfl_sync(0xffffffffu, comp, 1),
	             c2 = __shfl_sync(0xffffffffu, comp, 2);
	const int len = nk + 1;
	const int alloc = (len + 3) & ~3;
	long long off = 0;
	if (lane == 0) off = (long long)atomicAdd(A.pool_len, (unsigned long long)alloc);
	// ---- pivot (lane 0): dl = diag(s^-1/2) U^T, du = diag(s^-1/2) V^T into
	//      the diagonal slot (its values are not needed after this)
	int bad = 0;
	if (lane == 0) {
		double fd[9];
		double *u = bv_u(s, di);
#pragma unroll
		for (int k = 0; k < 9; k++) fd[k] = u[k];
		fd[0] = (fd[0] + rs0) + c0;
		fd[4] = (fd[4] + rs1) + c1;
		fd[8] = (fd[8] + rs2) + c2;
		double uu[9], vv[9], sv[3];
		svd3(fd, uu, sv, vv);
		if (!ilu) {
			for (int k = 0; k < 3; k++) {
				if (uu[3 * k] * vv[3 * k] + uu[1 + 3 * k] * vv[1 + 3 * k] + uu[2 + 3 * k] * vv[2 + 3 * k] < 0.0 &&
				    sv[k] > 0.0)
					bad = 1;
				for (int r = 0; r < 3; r++) uu[r + 3 * k] = vv[r + 3 * k];
				sv[k] = 1.0 / sqrt(sv[k]);
			}
		} else {
			for (int k = 0; k < 3; k++) sv[k] = 1.0 / sqrt(sv[k] < A.pivmin ? A.pivmin : sv[k]);
		}
		double *dl = bv_u(s, di), *du = ilu ? bv_l(s, di) : dl;
		for (int r = 0; r < 3; r++)
			for (int c = 0; c < 3; c++) {
				dl[r + 3 * c] = uu[c + 3 * r] * sv[r];
				if (ilu) du[r + 3 * c] = vv[c + 3 * r] * sv[r];
			}
	}
	bad = __shfl_sync(0xffffffffu, bad, 0);
	if (bad) {
		if (lane == 0) devstat_fail(A.st, BSG_ERR_PIVOT, i);
		return -2;
	}
	off = __shfl_sync(0xffffffffu, off, 0);
	if (off + alloc > A.pool_cap || len > 0xffff) {
		if (lane == 0) devstat_fail(A.st, BSG_ERR_WORKSPACE, i, 6);
		return -2;
	}
	__syncwarp();
	const double *dl = bv_u(s, di), *du = ilu ? bv_l(s, di) : dl;
	// ---- store: the pivot scaling, then the kept blocks scaled
	if (lane < 9) {
		const int r = lane % 3, c = lane / 3;
		if (lane == 0) A.pool_cf[off] = (unsigned)levmax | (F_U << 30);
		A.pool_l[9 * off + lane] = dl[c + 3 * r];
		if (ilu) A.pool_u[9 * off + lane] = du[c + 3 * r];
	}
	for (int t = lane; t < nk; t += 32) {
		const int h = s.lst[t];
		const double *u = bv_u(s, h), *l = ilu ? bv_l(s, h) : u;
		double tu[9], tl[9];
		mm3(dl, 1, 3, u, 1, 3, tu);
		if (ilu) mm3(du, 1, 3, l, 1, 3, tl);
		double mx = 0.0;
#pragma unroll
		for (int k = 0; k < 9; k++) {
			if (!ilu) tl[k] = tu[k];
			mx = fmax(mx, fmax(fabs(tl[k]), fabs(tu[k])));
		}
		const unsigned flag = mx >= A.tau1 ? F_U : F_R;
		const long long e = off + 1 + t;
		A.pool_cf[e] = (unsigned)s.hkey[h] | (flag << 30);
#pragma unroll
		for (int k = 0; k < 9; k++) {
			A.pool_l[9 * e + k] = tl[k];
			if (ilu) A.pool_u[9 * e + k] = tu[k];
		}
	}
	if (lane == 0) A.lev[i] = levmax;
	__threadfence();
	__syncwarp();
	if (lane == 0) st_release_u64(A.rec + i, REC_DONE | ((unsigned long long)off << 32) | (unsigned long long)len);
	__syncwarp();
	const long long cpub = clock64();
	pc.v[FS_CYC_TOPUB] += cpub - tail0;
	after_publish(A, i, lane);
	pc.v[FS_CYC_TAIL] += clock64() - tail0;
	pc.v[FS_MASK] += nl;
	return -1;
}

// Factor row i.  Returns -1 when done, the unfinished row it waits for
// (>= 0), -2 on error (reported through the status word), or -3 when the
// row does not fit a shared-memory workspace (nothing was published yet, so
// the caller retries it in the global one).
//
// Pipelined: the row closes the members that are finished, applies the
// updates of every closed member below the smallest unfinished one (the
// members below it are all known: a member is only discovered from a
// smaller member), then waits for that member while a warp computes it.
// When the last predecessor finishes, only its own segment and the finish
// are left.
template <class WS>
__device__ int try_row(const FactArgs &A, WS &s, int i, int lane, PhaseClock &pc) {
	constexpr bool ilu = WS::ilu;
	const long long c0 = clock64();
	for (int t = lane; t < s.wcap; t += 32) s.wset[t] = -1;
	if (lane == 0) s.sc[3] = 0;
	for (int t = lane; t < WS::mwin / 32; t += 32) s.wbits[t] = 0u; // (no bitmap: mwin 0)
	for (int t = lane; t < s.hcap; t += 32) s.hkey[t] = -1;
	if (lane == 0) s.sc[0] = 0;
	__syncwarp();

	// ---- seed with A's column i
	const int tb = A.it[i], te = A.it[i + 1];
	if (te - tb > s.cmax) {
		if (!WS::big) return -3;
		if (lane == 0) devstat_fail(A.st, BSG_ERR_WORKSPACE, i, 2);
		return -2;
	}
	for (int t = tb + lane; t < te; t += 32) {
		int k = A.jt[t];
		s.W[t - tb] = k;
		s.Wst[t - tb] = 0;
		wset_insert(s, i, k);
	}
	if (lane == 0) s.sc[0] = te - tb;
	__syncwarp();

	// ---- init the scaled row (Ich2InitRow / Ilu2InitRow); the compensations
	//      received from rows that dropped column i join the diagonal last
	int err = 0;
	const int ab = A.iu[i], ae = A.iu[i + 1];
	if constexpr (WS::blk) {
		err = init_blk(A, s, i, lane);
		if (err) {
			if (!WS::big) return -3;
			if (lane == 0) devstat_fail(A.st, err, i, 4);
			return -2;
		}
	} else {
	if (lane == 0) {
		int slot = hfind_insert(s, i);
		s.hl[slot] = A.diag0[i];
		if (ilu) s.hu[slot] = A.diag0[i];
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
				s.hl[sl] = __dmul_rn(__dmul_rn(A.al[k], si_l), A.scll[j]);
			}
		}
		err = __reduce_min_sync(0xffffffffu, err);
		__syncwarp();
	}
	if (err) {
		if (!WS::big) return -3;
		if (lane == 0) devstat_fail(A.st, err, i, 4);
		return -2;
	}
	}

	int levmax = 0;
	unsigned long long accraw = 0;
	bool waited = false;
	long long tail0 = clock64(); // end of the last wait: the row's own latency starts here
	for (;;) {
		// ---- close the finished members, pass after pass, until a pass
		//      closes none; the smallest member left is the bound
		// (a pass that closed members but discovered none leaves nothing
		// for another pass: every member is known, and the ones it found
		// unfinished are waited for below)
		int bound = i;
		const long long k0 = clock64();
		for (;;) {
			pc.v[FS_ROUNDS]++;
			int pmin = 0x7fffffff, added = 0;
			const long long q0 = clock64();
			const int closed = close_pass(A, s, i, lane, levmax, pmin, err, added);
			pc.v[FS_CYC_PCLOSE] += clock64() - q0;
			if (err) break;
			if (!closed || !added) {
				bound = pmin == 0x7fffffff ? i : pmin;
				break;
			}
		}
		if (err) {
			if (!WS::big) return -3;
			if (lane == 0) devstat_fail(A.st, err, i, 3);
			return -2;
		}
		const long long k1 = clock64();
		pc.v[FS_CYC_CLOSE] += k1 - k0;
		if (waited) pc.v[FS_CYC_TCLOSE] += k1 - k0;
		// the compensations received so far (every member seen finished has
		// pushed its own before publishing): loaded now, used after the last
		// pass, so the load overlaps the updates
		if (lane < (WS::blk ? 3 : 1)) accraw = __ldcg(A.acc + (WS::blk ? 3 * (size_t)i + lane : (size_t)i));
		// ---- updates of the closed members below the bound
		if constexpr (WS::blk) err = apply_blk(A, s, bound, lane, pc);
		else err = apply_members(A, s, bound, lane, pc);
		const long long k2 = clock64();
		pc.v[FS_CYC_UPD] += k2 - k1;
		if (err) {
			if (!WS::big) return -3;
			if (lane == 0) devstat_fail(A.st, err, i, 5);
			return -2;
		}
		if (bound == i) break;
		// ---- wait for the smallest unfinished member while a warp computes
		//      it; park when nobody does
		int res = 0;
		if (lane == 0) {
			res = wait_row(A, bound);
			if (res == 0 && promote(A, bound)) res = wait_row(A, bound);
			if (res == 0) res = hold_for(A, bound);
		}
		res = __shfl_sync(0xffffffffu, res, 0);
		tail0 = clock64();
		waited = true;
		pc.v[FS_CYC_BLOCKED] += tail0 - k2;
		if (res == 0) return bound;
		if (res < 0) {
			if (lane == 0) devstat_fail(A.st, BSG_ERR_TIMEOUT, i, 7);
			return -2;
		}
	}
	levmax = __reduce_max_sync(0xffffffffu, levmax);
	pc.v[FS_CONTRIB] += min(s.sc[0], s.cmax);
	if constexpr (WS::blk) return finish_blk(A, s, i, lane, levmax, accraw, pc, tail0);
	{
		const double comp = __dmul_rn((double)__shfl_sync(0xffffffffu, accraw, 0), A.acc_inv_scale);
		if (lane == 0) {
			const int di0 = hfind_insert(s, i);
			s.hl[di0] = __dadd_rn(s.hl[di0], comp);
			if (ilu) s.hu[di0] = __dadd_rn(s.hu[di0], comp);
		}
		__syncwarp();
	}
	const long long c3 = clock64();
	(void)c0;

	// ---- extract the off-diagonal mask columns and sort them ascending
	if (lane == 0) s.sc[1] = 0;
	__syncwarp();
	const int hscan = WS::big ? s.sc[3] : s.hcap; // slots to look at
	for (int q0 = 0; q0 < hscan; q0 += 32) { // whole warp in every round (ballots)
		const int q = q0 + lane;
		const int h = q < hscan ? (WS::big ? s.slots[q] : q) : -1;
		int c = h >= 0 ? s.hkey[h] : -1;
		bool take = c >= 0 && c != i;
		unsigned b = __ballot_sync(0xffffffffu, take);
		int base = s.sc[1];
		if (take) {
			const int at = base + __popc(b & ((1u << lane) - 1));
			s.lst[at] = h;
			s.lkey[at] = c;
		}
		__syncwarp();
		if (lane == 0) s.sc[1] = base + __popc(b);
		__syncwarp();
	}
	const int nl = s.sc[1];
	// rank sort (columns are distinct): each lane ranks its keys (as few per
	// lane as the row needs) against one broadcast key per step
	if (nl <= 32) rank_sort<1>(s.lkey, s.lst, s.lsts, nl, 0, lane);
	else if (nl <= 64) rank_sort<2>(s.lkey, s.lst, s.lsts, nl, 0, lane);
	else if (nl <= 128) rank_sort<4>(s.lkey, s.lst, s.lsts, nl, 0, lane);
	else
		for (int t0 = 0; t0 < nl; t0 += 256) rank_sort<8>(s.lkey, s.lst, s.lsts, nl, t0, lane);
	__syncwarp();
	const int di = hfind_insert(s, i); // existing slot of the diagonal

	// ---- filter by tau2 with theta compensation (ascending columns): the
	//      compensations of the dropped columns are formed in parallel (in
	//      pf_l), the kept columns compacted into lst[] in ascending order,
	//      and lane 0 adds the compensations to the diagonal in column order
	if (lane == 0) s.sc[2] = 0;
	__syncwarp();
	for (int t0 = 0; t0 < nl; t0 += 32) {
		const int t = t0 + lane;
		bool keep = false;
		if (t < nl) {
			const int h = s.lsts[t];
			double v = fabs(s.hl[h]);
			if (ilu) v = fmax(v, fabs(s.hu[h]));
			keep = v >= A.tau2;
			s.pf_l[t] = keep ? 0.0 : __dmul_rn(v, A.theta);
		}
		const unsigned b = __ballot_sync(0xffffffffu, keep);
		const int base = s.sc[2];
		if (keep) s.lst[base + __popc(b & ((1u << lane) - 1))] = s.lsts[t];
		__syncwarp();
		if (lane == 0) s.sc[2] = base + __popc(b);
		__syncwarp();
	}
	// the stored length is known: reserve the pool space now, so the
	// atomic's round trip overlaps the compensation sum and the pivot
	const int len = s.sc[2] + 1;
	const int alloc = (len + 3) & ~3;
	long long off = 0;
	if (lane == 0) off = (long long)atomicAdd(A.pool_len, (unsigned long long)alloc);
	// ---- hand the dropped entries' compensations to their rows now: the
	//      reductions are done by the time this row publishes (rows read a
	//      row's pushes only after acquiring its record)
	for (int t = lane; t < nl; t += 32) {
		const double v = s.pf_l[t];
		if (v != 0.0) acc_push(A.acc, s.hkey[s.lsts[t]], v, A.acc_scale, A.st);
	}
	// ---- the row's own compensations into its diagonal, in ascending column
	//      order; a kept column contributes +0.0, which leaves the (positive)
	//      sum unchanged, so the adds need no branch and the loads run ahead
	if (lane == 0) {
		double dl = s.hl[di], du = ilu ? s.hu[di] : 0.0;
		int t = 0;
		for (; t + 8 <= nl; t += 8) {
			double v[8];
#pragma unroll
			for (int q = 0; q < 8; q++) v[q] = s.pf_l[t + q];
#pragma unroll
			for (int q = 0; q < 8; q++) {
				dl = __dadd_rn(dl, v[q]);
				if (ilu) du = __dadd_rn(du, v[q]);
			}
		}
		for (; t < nl; t++) {
			const double v = s.pf_l[t];
			dl = __dadd_rn(dl, v);
			if (ilu) du = __dadd_rn(du, v);
		}
		s.hl[di] = dl;
		if (ilu) s.hu[di] = du;
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
	off = __shfl_sync(0xffffffffu, off, 0);
	if (off + alloc > A.pool_cap || len > 0xffff) {
		if (lane == 0) devstat_fail(A.st, BSG_ERR_WORKSPACE, i, 6);
		return -2;
	}
	if (lane == 0) {
		// entry 0 is the diagonal; its column field carries the row's depth
		A.pool_cf[off] = (unsigned)levmax | (F_U << 30);
		A.pool_l[off] = deleml;
		if (ilu) A.pool_u[off] = delemu;
	}
	for (int t = lane; t < nk; t += 32) {
		const int h = s.lst[t];
		double l = s.hl[h], u = ilu ? s.hu[h] : l;
		if (ilu) { l = __dmul_rn(l, delemu); u = __dmul_rn(u, deleml); } else { l = __dmul_rn(l, deleml); u = l; }
		double w = fabs(l);
		if (ilu) w = fmax(w, fabs(u));
		const unsigned flag = (w >= A.tau1) ? F_U : F_R;
		A.pool_cf[off + 1 + t] = (unsigned)s.hkey[h] | (flag << 30);
		A.pool_l[off + 1 + t] = l;
		if (ilu) A.pool_u[off + 1 + t] = u;
	}
	if (lane == 0) A.lev[i] = levmax;
	__threadfence();
	__syncwarp();
	if (lane == 0) st_release_u64(A.rec + i, REC_DONE | ((unsigned long long)off << 32) | (unsigned long long)len);
	__syncwarp();
	const long long cpub = clock64();
	pc.v[FS_CYC_TOPUB] += cpub - tail0;
	pc.v[FS_CYC_FPRE] += cpub - c3;

	after_publish(A, i, lane);
	const long long c4 = clock64();
	pc.v[FS_CYC_POSTPUB] += c4 - cpub;
	pc.v[FS_CYC_FIN] += c4 - c3;
	pc.v[FS_CYC_TAIL] += c4 - tail0;
	pc.v[FS_MASK] += nl;
	return -1;
}

template <bool ILU, bool BLK>
__global__ void __launch_bounds__((BLK ? FACT_WARPS_BLK : FACT_WARPS) * 32, FACT_MINB) k_fact_rows(FactArgs A) {
	constexpr int fw = BLK ? FACT_WARPS_BLK : FACT_WARPS;
	extern __shared__ unsigned char smem_raw[];
	const int warp = threadIdx.x >> 5;
	SmemWS<ILU, BLK> &s = reinterpret_cast<SmemWS<ILU, BLK> *>(smem_raw)[warp];
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
		if (lane == 0) {
			*(volatile int *)(A.inprog + i) = 1;
			__threadfence();
		}
		// first claim: the rows of A's row i have one static contributor
		// fewer that is unclaimed
		int first = 0;
		if (lane == 0) first = !(atomicOr(reinterpret_cast<unsigned *>(A.nstat) + i, ADM_CLAIMED) & ADM_CLAIMED);
		first = __shfl_sync(0xffffffffu, first, 0);
		if (first)
			for (int k = A.iu[i] + 1 + lane; k < A.iu[i + 1]; k += 32) admit_step(A, A.ju[k], ADM_ONE_CLAIM);
		__syncwarp();
		int r = try_row(A, s, i, lane, pc);
		if (r == -3) {
			// a shared workspace is too small: take a free global one, or
			// give the row back to the queue (a warp never waits for a
			// workspace, so workspace holders cannot deadlock)
			pc.v[FS_BIG]++;
			int slot = -1;
			if (lane == 0) {
				const int start = (int)((blockIdx.x * fw + warp) % BIG_SLOTS);
				for (int k = 0; k < BIG_SLOTS && slot < 0; k++) {
					const int q = (start + k) % BIG_SLOTS;
					if (atomicCAS(A.big_owner + q, 0, 1) == 0) slot = q;
				}
			}
			slot = __shfl_sync(0xffffffffu, slot, 0);
			if (slot < 0) {
				if (lane == 0) {
					*(volatile int *)(A.inprog + i) = 0;
					__threadfence();
					q_push(A, i);
				}
				__syncwarp();
				continue;
			}
			__threadfence();
			GlobWS<ILU, BLK> g(A.big_ws + (size_t)slot * GlobWS<ILU, BLK>::bytes);
			r = try_row(A, g, i, lane, pc);
			__syncwarp();
			if (lane == 0) {
				__threadfence();
				atomicExch(A.big_owner + slot, 0);
			}
		}
		if (r == -2) break;
		if (r >= 0) {
			pc.v[FS_PARK]++;
			if (lane == 0) {
				*(volatile int *)(A.inprog + i) = 0;
				__threadfence();
				park(A, i, r);
			}
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
                            unsigned long long *acc, int *lev, int *inprog, bsg_devstat *st) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	int cnt = it[i + 1] - it[i];
	if (cnt > 0x7fff) { // the admission counters hold 15 bits
		devstat_fail(st, BSG_ERR_WORKSPACE, i, 8);
		cnt = 0;
	}
	nstat[i] = (cnt << 15) | cnt | (cnt == 0 ? ADM_QUEUED : 0u); // k_fact_seed queues those
	inprog[i] = 0;
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
		int j = e == off ? i : CF_COL(x); // entry 0: the diagonal (its column field holds the depth)
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

// block rows: stored blocks per row, then the rows in order (pivot scaling
// first: column i; U blocks +column, R blocks -column), counts of U / R
__global__ void k_blk_len(int nb, const unsigned long long *rec, int *cnt) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < nb) cnt[i] = REC_LEN(rec[i]);
}
__global__ void k_blk_emit(int nb, int ilu, const unsigned long long *rec, const unsigned *cf, const double *pl,
                           const double *pu, const int *ig, int *jg, double *gl, double *gu, unsigned long long *nst) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nb) return;
	const long long off = REC_OFF(rec[i]);
	const int len = REC_LEN(rec[i]);
	const long long o = ig[i];
	unsigned long long nu = 0, nr = 0;
	for (int e = 0; e < len; e++) {
		const unsigned x = cf[off + e];
		const bool u = e == 0 || CF_FLAG(x) == F_U;
		const int col = e == 0 ? i : CF_COL(x);
		jg[o + e] = u ? col : -col;
		nu += u;
		nr += !u;
		for (int k = 0; k < 9; k++) {
			gl[9 * (o + e) + k] = pl[9 * (off + e) + k];
			gu[9 * (o + e) + k] = ilu ? pu[9 * (off + e) + k] : pl[9 * (off + e) + k];
		}
	}
	atomicAdd(nst, nu);
	atomicAdd(nst + 1, nr);
}

inline int nb(long long n, int t) { return n > 0 ? (int)((n + t - 1) / t) : 1; }
inline int nb_blocks(long long n) { return nb(n, 256); }

} // namespace

int bsg_fct_finish(bsg_ctx *c, bsg_fct *f);

// Scale of the fixed-point compensation sums: a compensation is at most
// tau2 * theta < 2^e, so 2^(51 - e) keeps each term below 2^51 and the sum of
// the at most 2^13 terms a row receives below 2^64; the rule is exact (frexp)
// so the oracle derives the same scale.
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
// [1] parks, [2..7] SM cycles summed over warps in queue wait, closure
// passes, waits for members, a row's own latency after its last wait,
// updates, finish; [8] members of C(i),
// [9] mask columns, [10] closure rounds, [11..13] SM cycles in prefetch,
// slot resolution and fma phases, [14] rows retried in the global-memory
// workspace, [15] warps launched, [16..19] SM cycles loading / closing in
// the passes, from the last wait to publishing, after publishing, [20]
// update batches, [21] members applied, [22] SM cycles of the closure passes
// after a wait, [23] of the finish before publishing.
extern "C" int bsg_fact_stats(unsigned long long *out, int nout) {
	if (!out && nout > 0) return bsg_set_error(BSG_ERR_ARG, "bsg_fact_stats: null output");
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
	long long qcap = 1;
	while (qcap < 2LL * n + 65536) qcap <<= 1; // ring of slots, see q_push
	double *scll, *sclu, *diag0, *pl, *pu = nullptr;
	unsigned *cf;
	unsigned long long *rec, *acc;
	int *lev, *nstat, *whead, *wnext, *queue, *done_count, *inprog;
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
	BSG_CUDA(cudaMallocAsync(&inprog, sizeof(int) * n, st));
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
	k_fact_init<<<nb(n, 256), 256, 0, st>>>(n, m->d_it, nstat, whead, rec, acc, lev, inprog, c->d_stat);
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
	A.nstat = nstat; A.whead = whead; A.wnext = wnext; A.inprog = inprog; A.queue = queue; A.qcap = qcap;
	A.qhead = qhead; A.qtail = qtail; A.done_count = done_count; A.st = c->d_stat;
	BSG_CUDA(cudaMallocAsync(&A.stats, sizeof(unsigned long long) * FACT_NSTAT, st));
	BSG_CUDA(cudaMemsetAsync(A.stats, 0, sizeof(unsigned long long) * FACT_NSTAT, st));
	k_fact_seed<<<nb(n, 256), 256, 0, st>>>(A);
	void (*kern)(FactArgs) = kind == 1 ? k_fact_rows<true, false> : k_fact_rows<false, false>;
	const size_t smem = (kind == 1 ? sizeof(SmemWS<true>) : sizeof(SmemWS<false>)) * FACT_WARPS;
	BSG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	int per_sm = 0;
	BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, FACT_WARPS * 32, smem));
	if (per_sm < 1) per_sm = 1;
	int grid = per_sm * BSG_SMS;
	int need = (n + FACT_WARPS - 1) / FACT_WARPS;
	if (grid > need) grid = need;
	if (grid < 1) grid = 1;
	if (cudaMallocAsync(&A.big_ws, GlobWS<true>::bytes * (size_t)BIG_SLOTS, st) != cudaSuccess)
		return bsg_set_error(BSG_ERR_NOMEM, "factor row workspace");
	BSG_CUDA(cudaMallocAsync(&A.big_owner, sizeof(int) * (BIG_SLOTS + 1), st));
	BSG_CUDA(cudaMemsetAsync(A.big_owner, 0, sizeof(int) * (BIG_SLOTS + 1), st));
	A.nhold = A.big_owner + BIG_SLOTS;
	A.hold_max = grid * FACT_WARPS / 2;
	kern<<<grid, FACT_WARPS * 32, smem, st>>>(A);
	BSG_CUDA(cudaGetLastError());
	int rc = bsg_check_devstat(c);
	cudaMemcpyAsync(g_fact_stats, A.stats, sizeof(g_fact_stats), cudaMemcpyDeviceToHost, st);
	cudaStreamSynchronize(st);
	g_fact_stats[FS_WARPS] = (unsigned long long)grid * FACT_WARPS; // warps launched
	cudaFreeAsync(A.stats, st);
	cudaFreeAsync(A.big_ws, st);
	cudaFreeAsync(A.big_owner, st);
	int ndone = 0;
	if (!rc) {
		BSG_CUDA(cudaMemcpy(&ndone, done_count, sizeof(int), cudaMemcpyDeviceToHost));
		if (ndone != n) rc = bsg_set_error(BSG_ERR_TIMEOUT, "factorisation scheduler stopped early");
	}
	auto release = [&]() {
		for (void *q : {(void *)scll, (void *)sclu, (void *)diag0, (void *)cf, (void *)pl, (void *)pu, (void *)rec,
		                (void *)acc, (void *)lev, (void *)nstat, (void *)whead, (void *)wnext, (void *)inprog, (void *)queue,
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

// this unit's copy of the spin-wait bound (bsg_set_spin_limit_ns)
int bsg_spin_limit_set_fact(unsigned long long ns) {
	return bsg_spin_limit_set_here(ns) == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}

// Block IC2 (sym) / ILU2 of 3 x 3 block rows with the dynamic schedule of
// the point factorisation: a warp per block row, the closure over finished
// rows, admission, waiting, parking and promotion unchanged; the row's
// arithmetic on blocks (init_blk / apply_blk / finish_blk).  Input: the
// CombineLU block pattern (diagonal first) with its scaled values and
// scalings (9 doubles each, column-major).  Output: the stored rows in row
// order (ig[nb + 1]; jg: +column U, -column R, the pivot scaling first;
// gl / gu: 9 doubles a block), allocated here, and the U / R counts.
int bsg_bfact_dyn(bsg_ctx *c, int nb, int sym, const bsg_param *p, const int *bia, const int *bja, int nnzb,
                  const double *bal, const double *bau, const double *scll, const double *sclu, const double *diagg,
                  int **ig_o, int **jg_o, double **gl_o, double **gu_o, unsigned long long *nstored) {
	const int kind = sym ? 0 : 1;
	cudaStream_t st = c->stream;
	int *it = nullptr, *jt = nullptr, nt = 0;
	int rc = bsg_strict_transpose(c, nb, bia, bja, nnzb, &it, &jt, nullptr, &nt);
	if (rc) return rc;
	double mem = p->memory < 0 ? -p->memory : p->memory;
	if (mem < 8.0) mem = 8.0;
	long long qcap = 1;
	while (qcap < 2LL * nb + 65536) qcap <<= 1;
	double *pl = nullptr, *pu = nullptr;
	unsigned *cf = nullptr;
	unsigned long long *rec, *acc, *pool_len, *qhead, *qtail;
	int *lev, *nstat, *whead, *wnext, *queue, *done_count, *inprog;
	BSG_CUDA(cudaMallocAsync(&rec, sizeof(unsigned long long) * nb, st));
	BSG_CUDA(cudaMallocAsync(&acc, sizeof(unsigned long long) * 3 * (size_t)nb, st));
	BSG_CUDA(cudaMallocAsync(&lev, sizeof(int) * nb, st));
	BSG_CUDA(cudaMallocAsync(&nstat, sizeof(int) * nb, st));
	BSG_CUDA(cudaMallocAsync(&whead, sizeof(int) * nb, st));
	BSG_CUDA(cudaMallocAsync(&wnext, sizeof(int) * nb, st));
	BSG_CUDA(cudaMallocAsync(&inprog, sizeof(int) * nb, st));
	BSG_CUDA(cudaMallocAsync(&queue, sizeof(int) * qcap, st));
	BSG_CUDA(cudaMallocAsync(&done_count, sizeof(int), st));
	BSG_CUDA(cudaMallocAsync(&pool_len, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMallocAsync(&qhead, sizeof(unsigned long long), st));
	BSG_CUDA(cudaMallocAsync(&qtail, sizeof(unsigned long long), st));
	void (*kern)(FactArgs) = kind == 1 ? k_fact_rows<true, true> : k_fact_rows<false, true>;
	const size_t smem = (kind == 1 ? sizeof(SmemWS<true, true>) : sizeof(SmemWS<false, true>)) * FACT_WARPS_BLK;
	const size_t big = kind == 1 ? GlobWS<true, true>::bytes : GlobWS<false, true>::bytes;
	BSG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	int per_sm = 0;
	BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, FACT_WARPS_BLK * 32, smem));
	if (per_sm < 1) per_sm = 1;
	int grid = per_sm * BSG_SMS;
	const int need = (nb + FACT_WARPS_BLK - 1) / FACT_WARPS_BLK;
	if (grid > need) grid = need;
	if (grid < 1) grid = 1;
	FactArgs A;
	A.n = nb; A.kind = kind;
	A.iu = bia; A.ju = bja; A.al = bal; A.au = bau;
	A.it = it; A.jt = jt;
	A.scll = scll; A.sclu = sclu; A.diag0 = diagg;
	A.tau1 = p->tau1; A.tau2 = p->tau2; A.theta = p->theta; A.pivmin = p->pivmin;
	A.pool_len = pool_len;
	A.rec = rec; A.acc = acc; A.lev = lev;
	// a compensation column sum has three terms below tau2 * theta each
	bsg_comp_scale(3.0 * p->tau2, p->theta, &A.acc_scale, &A.acc_inv_scale);
	A.nstat = nstat; A.whead = whead; A.wnext = wnext; A.inprog = inprog; A.queue = queue; A.qcap = qcap;
	A.qhead = qhead; A.qtail = qtail; A.done_count = done_count; A.st = c->d_stat;
	if (cudaMallocAsync(&A.big_ws, big * (size_t)BIG_SLOTS, st) != cudaSuccess)
		return bsg_set_error(BSG_ERR_NOMEM, "block factor row workspace");
	BSG_CUDA(cudaMallocAsync(&A.big_owner, sizeof(int) * (BIG_SLOTS + 1), st));
	A.nhold = A.big_owner + BIG_SLOTS;
	A.hold_max = grid * FACT_WARPS_BLK / 2;
	BSG_CUDA(cudaMallocAsync(&A.stats, sizeof(unsigned long long) * FACT_NSTAT, st));
	// The pool first holds 8 blocks per block of A (block IC2 / ILU2 keep
	// about 4); a factor that needs more is computed again with the pool
	// the memory parameter allows.
	for (double memu = mem < 8.0 ? mem : 8.0;; memu = mem) {
		long long cap = (long long)(memu * (double)nnzb) + 8LL * nb + 1024;
		if (cap > 0x7ffffff0LL) cap = 0x7ffffff0LL;
		if (cudaMallocAsync(&cf, sizeof(unsigned) * cap, st) != cudaSuccess ||
		    cudaMallocAsync(&pl, sizeof(double) * 9 * cap, st) != cudaSuccess ||
		    (kind == 1 && cudaMallocAsync(&pu, sizeof(double) * 9 * cap, st) != cudaSuccess))
			return bsg_set_error(BSG_ERR_NOMEM, "block factor pool");
		A.pool_cf = cf; A.pool_l = pl; A.pool_u = pu; A.pool_cap = cap;
		BSG_CUDA(cudaMemsetAsync(c->d_stat, 0, sizeof(bsg_devstat), st));
		BSG_CUDA(cudaMemsetAsync(pool_len, 0, sizeof(unsigned long long), st));
		BSG_CUDA(cudaMemsetAsync(qhead, 0, sizeof(unsigned long long), st));
		BSG_CUDA(cudaMemsetAsync(qtail, 0, sizeof(unsigned long long), st));
		BSG_CUDA(cudaMemsetAsync(done_count, 0, sizeof(int), st));
		BSG_CUDA(cudaMemsetAsync(A.big_owner, 0, sizeof(int) * (BIG_SLOTS + 1), st));
		BSG_CUDA(cudaMemsetAsync(A.stats, 0, sizeof(unsigned long long) * FACT_NSTAT, st));
		BSG_COUNT(4);
		k_fact_init<<<nb_blocks(nb), 256, 0, st>>>(nb, it, nstat, whead, rec, acc, lev, inprog, c->d_stat);
		BSG_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * 3 * (size_t)nb, st));
		k_fill_int<<<BSG_SMS * 4, 256, 0, st>>>(qcap, queue, -1);
		k_fact_seed<<<nb_blocks(nb), 256, 0, st>>>(A);
		kern<<<grid, FACT_WARPS_BLK * 32, smem, st>>>(A);
		BSG_CUDA(cudaGetLastError());
		bsg_devstat h;
		BSG_CUDA(cudaMemcpyAsync(&h, c->d_stat, sizeof(h), cudaMemcpyDeviceToHost, st));
		BSG_CUDA(cudaStreamSynchronize(st));
		if (h.code == BSG_ERR_WORKSPACE && h.pad[0] == 6 && memu < mem) { // the pool was too small
			cudaFreeAsync(cf, st);
			cudaFreeAsync(pl, st);
			if (pu) cudaFreeAsync(pu, st);
			cf = nullptr; pl = pu = nullptr;
			continue;
		}
		break;
	}
	rc = bsg_check_devstat(c);
	cudaMemcpyAsync(g_fact_stats, A.stats, sizeof(g_fact_stats), cudaMemcpyDeviceToHost, st);
	cudaStreamSynchronize(st);
	g_fact_stats[FS_WARPS] = (unsigned long long)grid * FACT_WARPS_BLK;
	cudaFreeAsync(A.stats, st);
	cudaFreeAsync(A.big_ws, st);
	cudaFreeAsync(A.big_owner, st);
	if (!rc) {
		int ndone = 0;
		BSG_CUDA(cudaMemcpy(&ndone, done_count, sizeof(int), cudaMemcpyDeviceToHost));
		if (ndone != nb) rc = bsg_set_error(BSG_ERR_TIMEOUT, "block factorisation scheduler stopped early");
	}
	int *cnt = nullptr, *ig = nullptr;
	if (!rc && (cudaMallocAsync(&cnt, sizeof(int) * (nb + 1), st) != cudaSuccess ||
	            cudaMallocAsync(&ig, sizeof(int) * (nb + 1), st) != cudaSuccess))
		rc = bsg_set_error(BSG_ERR_NOMEM, "block factor rows");
	long long total = 0;
	if (!rc) {
		BSG_COUNT(1);
		cudaMemsetAsync(cnt + nb, 0, sizeof(int), st);
		k_blk_len<<<nb_blocks(nb), 256, 0, st>>>(nb, rec, cnt);
		size_t tmp = 0;
		cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, ig, nb + 1, st);
		void *d_tmp = nullptr;
		if (cudaMallocAsync(&d_tmp, tmp + 1, st) != cudaSuccess) rc = bsg_set_error(BSG_ERR_NOMEM, "scan");
		else {
			cub::DeviceScan::ExclusiveSum(d_tmp, tmp, cnt, ig, nb + 1, st);
			int t = 0;
			cudaMemcpyAsync(&t, ig + nb, sizeof(int), cudaMemcpyDeviceToHost, st);
			cudaStreamSynchronize(st);
			total = t;
			cudaFreeAsync(d_tmp, st);
		}
	}
	int *jg = nullptr;
	double *gl = nullptr, *gu = nullptr;
	if (!rc && (cudaMallocAsync(&jg, sizeof(int) * (total > 0 ? total : 1), st) != cudaSuccess ||
	            cudaMallocAsync(&gl, sizeof(double) * 9 * (total > 0 ? total : 1), st) != cudaSuccess ||
	            cudaMallocAsync(&gu, sizeof(double) * 9 * (total > 0 ? total : 1), st) != cudaSuccess))
		rc = bsg_set_error(BSG_ERR_NOMEM, "block factor rows");
	if (!rc) {
		BSG_COUNT(1);
		cudaMemsetAsync(nstored, 0, sizeof(unsigned long long) * 2, st);
		k_blk_emit<<<nb_blocks(nb), 256, 0, st>>>(nb, kind, rec, cf, pl, pu, ig, jg, gl, gu, nstored);
		if (cudaGetLastError() != cudaSuccess) rc = bsg_set_error(BSG_ERR_CUDA, "block factor rows");
	}
	for (void *q : {(void *)it, (void *)jt, (void *)cf, (void *)pl, (void *)pu, (void *)rec, (void *)acc, (void *)lev,
	                (void *)nstat, (void *)whead, (void *)wnext, (void *)inprog, (void *)queue, (void *)done_count,
	                (void *)pool_len, (void *)qhead, (void *)qtail, (void *)cnt})
		if (q) cudaFreeAsync(q, st);
	if (rc) {
		for (void *q : {(void *)ig, (void *)jg, (void *)gl, (void *)gu})
			if (q) cudaFreeAsync(q, st);
		return rc;
	}
	*ig_o = ig;
	*jg_o = jg;
	*gl_o = gl;
	*gu_o = gu;
	return BSG_OK;
}
