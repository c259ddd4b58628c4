// SELL-8 storage and kernels for the bandwidth-bound products of the path:
// the SpMV of a point matrix and the Jacobi sweeps of the triangular solves.
//
// Layout.  Rows are cut into slices of C = 8 consecutive rows; slice s has
// width w_s = the longest row in it, and its entries are stored column-major
// in [off_s, off_s + 8 w_s): entry k of row 8 s + l at off_s + 8 k + l.
// Short rows are padded with (column = the row itself, value 0).
//
// Why: a warp serves 4 consecutive slices, an 8-lane group one slice, lane l
// its row.  Every column / value load of a group is one 32 B sector (FP32,
// int32) or two (FP64), and the 8 gathers of the input vector for entry k hit
// the columns of 8 neighbouring rows -- for stencil-like matrices and their
// incomplete factors, consecutive addresses.  Slices of 8 rather than 32 rows
// keep the padding small when row lengths vary (threshold factors), while the
// DRAM sector stays fully used.  Each lane keeps 8 entries in flight
// (unrolled), enough bytes per SM to run at the HBM roofline: per entry 4 B
// column + 4 B (FP32) or 8 B (FP64) value.
//
// Long rows.  A slice is as slow as its longest row walked by one lane, so
// rows of more than SELL_LONG entries (the wrap-around fill of periodic
// problems reaches thousands) leave the slices and are summed as CSR rows by
// a warp, or by a block beyond SELL_VLONG entries, in the same kernel, ahead
// of the slices.  Their sums run in another order than the sequential one.
#include "bsg_internal.cuh"
#include <cub/device/device_scan.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_select.cuh>

#define SELL_C 8
#define SELL_LONG 256   // entries: longer rows leave the slices
#define SELL_VLONG 4096 // entries: longer rows take a whole block

namespace {

// Slice widths; rows longer than longlen (> 0) count as empty, and bit l of
// lmask[slice] marks slot l as such a row.
__global__ void k_sell_width(int n, const int *rp, int skip, const int *perm, int even, int longlen,
                             long long *width, unsigned char *lmask) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int slice = t / SELL_C;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int r = t < n ? (perm ? perm[t] : t) : n; // one thread per row slot
	int len = r < n ? rp[r + 1] - rp[r] - skip : 0;
	if (len < 0) len = 0;
	const bool lng = longlen > 0 && len > longlen;
	if (lng) len = 0;
	const unsigned bits = __ballot_sync(0xffffffffu, lng);
#pragma unroll
	for (int o = SELL_C / 2; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, o, SELL_C));
	if (even) len = (len + 1) & ~1;
	if ((t % SELL_C) == 0 && slice < nsl) {
		width[slice] = (long long)SELL_C * len;
		if (lmask) lmask[slice] = (unsigned char)(bits >> (threadIdx.x & 31 & ~(SELL_C - 1)));
	}
}

// class of every row: 2 more than SELL_VLONG entries, 1 more than SELL_LONG
__global__ void k_long_flags(int n, const int *rp, int skip, unsigned char *fv, unsigned char *fl, int *iota) {
	for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
		const int len = rp[r + 1] - rp[r] - skip;
		fv[r] = len > SELL_VLONG;
		fl[r] = len > SELL_LONG && len <= SELL_VLONG;
		iota[r] = r;
	}
}

__global__ void k_long_len(int nl, const int *lrow, const int *rp, int skip, long long *len) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= nl; i += gridDim.x * blockDim.x)
		len[i] = i < nl ? rp[lrow[i] + 1] - rp[lrow[i]] - skip : 0;
}

// one warp per long row: its entries in CSR order
template <typename VT>
__global__ void k_long_fill(int nl, const int *lrow, const long long *loff, const int *rp, const int *ci,
                            const double *v, int skip, int *lcol, VT *lval) {
	const int lane = threadIdx.x & 31;
	for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nl; i += (gridDim.x * blockDim.x) >> 5) {
		const int b = rp[lrow[i]] + skip;
		const long long o = loff[i], len = loff[i + 1] - o;
		for (long long k = lane; k < len; k += 32) {
			lcol[o + k] = ci[b + k];
			lval[o + k] = (VT)v[b + k];
		}
	}
}

template <typename VT>
struct sell_long {
	int nlong, nvlong;
	const int *row;
	const long long *off;
	const int *col;
	const VT *val;
	const unsigned char *mask;
};

template <typename VT>
sell_long<VT> long_of(const bsg_sell *m) {
	return {m->nlong, m->nvlong, m->lrow, m->loff, m->lcol, (const VT *)m->lval, m->lmask};
}

// Sum of the products of entries [b, e) of a long row by one warp (BLOCK
// false, tid = lane) or by a block of 256 threads (red: 8 doubles of shared
// memory): thread t takes entries t, t + T, t + 2 T, ... in order, U loads in
// flight, then a fixed tree.  Every thread of the warp / block gets the sum.
template <typename VT, typename XT, int IN, bool BLOCK, int U>
__device__ __forceinline__ double long_row_sum(long long b, long long e, int tid, const int *__restrict__ lcol,
                                               const VT *__restrict__ lval, const XT *__restrict__ x,
                                               const double *__restrict__ dinv_in, double *red) {
	constexpr int T = BLOCK ? 256 : 32;
	double sum = 0.0;
	for (long long j = b + tid; j < e; j += (long long)U * T) {
		int c[U];
		double a[U], xv[U];
#pragma unroll
		for (int u = 0; u < U; u++) {
			const long long q = j + (long long)u * T;
			c[u] = q < e ? __ldcs(lcol + q) : -1;
			a[u] = q < e ? (double)__ldcs(lval + q) : 0.0;
		}
#pragma unroll
		for (int u = 0; u < U; u++) {
			xv[u] = c[u] >= 0 ? (double)__ldg(x + c[u]) : 0.0;
			if (IN == 1 && c[u] >= 0) xv[u] *= __ldg(dinv_in + c[u]);
		}
#pragma unroll
		for (int u = 0; u < U; u++)
			if (c[u] >= 0) sum = fma(a[u], xv[u], sum);
	}
	sum = warp_sum(sum);
	if (BLOCK) {
		if ((tid & 31) == 0) red[tid >> 5] = sum;
		__syncthreads();
		double t = 0.0;
#pragma unroll
		for (int w = 0; w < 8; w++) t += red[w];
		__syncthreads(); // red is free for the next row
		sum = t;
	}
	return sum;
}

// The long rows of a product or pass (blockDim 256): out(r, sum) by thread 0
// of the block or lane 0 of the warp that summed row r.
template <typename VT, typename XT, int IN, typename F>
__device__ __forceinline__ void long_rows(const sell_long<VT> &lg, const XT *__restrict__ x,
                                          const double *__restrict__ dinv_in, F out) {
	if (!lg.nlong) return;
	__shared__ double red[8];
	for (int i = blockIdx.x; i < lg.nvlong; i += gridDim.x) {
		const double s = long_row_sum<VT, XT, IN, true, 4>(__ldg(lg.off + i), __ldg(lg.off + i + 1), threadIdx.x,
		                                                   lg.col, lg.val, x, dinv_in, red);
		if (threadIdx.x == 0) out(__ldg(lg.row + i), s);
	}
	const int lane = threadIdx.x & 31;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int i = lg.nvlong + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < lg.nlong; i += nwarps) {
		const double s = long_row_sum<VT, XT, IN, false, 8>(__ldg(lg.off + i), __ldg(lg.off + i + 1), lane, lg.col,
		                                                    lg.val, x, dinv_in, nullptr);
		if (lane == 0) out(__ldg(lg.row + i), s);
	}
}

// ---- tiled form ----------------------------------------------------------
// A tile is SELL_TILE consecutive row slots (32 slices).  Its entries read x
// only inside a few 32-float blocks (for stencil factors: a band around the
// row and one around each neighbouring plane / line), so the tiled sweep
// copies those blocks to shared memory with coalesced loads and gathers from
// there, and each column shrinks to a 16-bit index into the staged blocks.
#define SELL_TILE 256
#define TB_MAX 512    // blocks per tile: 64 KB of staging, indices < 2^14
#define TB_HASH 2048  // open-addressing table of a tile's distinct blocks

__device__ __forceinline__ unsigned tb_hash(int key) { return ((unsigned)key * 2654435761u) >> 21; }

// slot of key, inserted if new (count incremented); -1 if the table is full
__device__ int tb_insert(int *hk, int key, int *count) {
	unsigned h = tb_hash(key);
	for (int i = 0; i < TB_HASH; i++) {
		const int prev = atomicCAS(hk + h, -1, key);
		if (prev == -1) {
			atomicAdd(count, 1);
			return (int)h;
		}
		if (prev == key) return (int)h;
		h = (h + 1) & (TB_HASH - 1);
	}
	return -1;
}

__device__ int tb_find(const int *hk, int key) {
	unsigned h = tb_hash(key);
	for (int i = 0; i < TB_HASH; i++) {
		const int k = hk[h];
		if (k == key) return (int)h;
		if (k == -1) return -1;
		h = (h + 1) & (TB_HASH - 1);
	}
	return -1;
}

// FILL 0: cnt[t] = distinct x blocks of tile t (bad = 1 if a tile exceeds
// TB_MAX).  FILL 1: tb[tb_off[t] ..] = those blocks ascending, and the packed
// 16-bit local columns of every entry (padding: index 0, value 0 in sval).
template <int FILL>
__global__ void __launch_bounds__(SELL_TILE) k_tile_blocks(int n, const int *rp, const int *ci, int skip,
                                                           const int *perm, const long long *off, int ntile, int *cnt,
                                                           int *bad, const int *tb_off, int *tb, unsigned *cpair) {
	__shared__ int hk[TB_HASH];
	__shared__ int hr[TB_HASH];
	__shared__ int lst[TB_MAX];
	__shared__ int count, pos, fail;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int tid = threadIdx.x;
	for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
		for (int i = tid; i < TB_HASH; i += SELL_TILE) hk[i] = -1;
		if (tid == 0) {
			count = 0;
			pos = 0;
			fail = 0;
		}
		__syncthreads();
		const int t = tile * SELL_TILE + tid;
		const int r = t < n ? (perm ? perm[t] : t) : -1;
		int b = 0, e = 0;
		if (r >= 0) {
			b = rp[r] + skip;
			e = rp[r + 1];
			if (e < b) e = b;
		}
		for (int j = b; j < e; j++)
			if (tb_insert(hk, ci[j] >> 5, &count) < 0) fail = 1;
		__syncthreads();
		if (!FILL) {
			if (tid == 0) {
				cnt[tile] = count;
				if (fail || count > TB_MAX) atomicExch(bad, 1);
			}
			__syncthreads();
			continue;
		}
		// the host checked count <= TB_MAX for every tile
		for (int i = tid; i < TB_HASH; i += SELL_TILE)
			if (hk[i] != -1) lst[atomicAdd(&pos, 1)] = hk[i];
		int P = 1;
		while (P < count) P <<= 1;
		__syncthreads();
		for (int i = count + tid; i < P; i += SELL_TILE) lst[i] = 0x7fffffff;
		__syncthreads();
		for (int k = 2; k <= P; k <<= 1) // bitonic sort, ascending
			for (int jj = k >> 1; jj > 0; jj >>= 1) {
				for (int i = tid; i < P; i += SELL_TILE) {
					const int ixj = i ^ jj;
					if (ixj > i) {
						const int a = lst[i], c = lst[ixj];
						if ((a > c) == ((i & k) == 0)) {
							lst[i] = c;
							lst[ixj] = a;
						}
					}
				}
				__syncthreads();
			}
		const int tb0 = tb_off[tile];
		for (int i = tid; i < count; i += SELL_TILE) {
			tb[tb0 + i] = lst[i];
			hr[tb_find(hk, lst[i])] = i;
		}
		__syncthreads();
		const int slice = t / SELL_C, l = t % SELL_C;
		if (slice < nsl) {
			const long long base = off[slice];
			const int w = (int)((off[slice + 1] - base) / SELL_C);
			unsigned *cp = cpair + base / 2 + l;
			const int len = e - b;
			for (int k = 0; k < w; k += 2) {
				unsigned lo = 0, hi = 0;
				if (k < len) {
					const int c = ci[b + k];
					lo = (unsigned)(hr[tb_find(hk, c >> 5)] * 32 + (c & 31));
				}
				if (k + 1 < len) {
					const int c = ci[b + k + 1];
					hi = (unsigned)(hr[tb_find(hk, c >> 5)] * 32 + (c & 31));
				}
				cp[SELL_C * (k / 2)] = lo | (hi << 16);
			}
		}
		__syncthreads();
	}
}

// The FP32-iterate Jacobi pass of k_sell_sweep32 on the tiled form: per
// tile, stage its x blocks in shared memory, then every thread forms one
// row slot's sum from 4-byte values and 2-byte local columns.  The products
// are summed in the same order as k_sell_sweep32, so the results agree bit
// for bit.  The staging is double-buffered: the next tile's x blocks are
// copied with asynchronous 16-byte copies (cp.async, columns past n
// zero-filled) while the current tile computes, so each tile costs one
// barrier and the copies' latency hides behind the value stream.
template <int OUT64>
__global__ void __launch_bounds__(SELL_TILE) k_tsell_sweep32(int n, int ntile, const int *__restrict__ perm,
                                                             const long long *__restrict__ off,
                                                             const unsigned *__restrict__ cpair,
                                                             const float *__restrict__ sval,
                                                             const int *__restrict__ tb_off,
                                                             const int *__restrict__ tb, const float *__restrict__ x32,
                                                             const double *__restrict__ rhs,
                                                             const double *__restrict__ dinv, double *__restrict__ y,
                                                             float *__restrict__ y32, int tstride) {
	extern __shared__ __align__(16) float sx[]; // two buffers of tmax x 32 floats
	const int nsl = (n + SELL_C - 1) / SELL_C;
	// the x blocks of a tile into one buffer, 16 bytes a copy; an iterate
	// that does not start on a 16-byte boundary (the second half of an
	// odd-length ping-pong pair) is staged with plain loads instead
	const bool async16 = (reinterpret_cast<unsigned long long>(x32) & 15ull) == 0;
	auto stage = [&](int tile, float *buf) {
		const int b0 = __ldg(tb_off + tile), npc = (__ldg(tb_off + tile + 1) - b0) * 8;
		for (int q = threadIdx.x; q < npc; q += SELL_TILE) {
			const int c = __ldg(tb + b0 + (q >> 3)) * 32 + (q & 7) * 4; // first column of the piece
			const int left = n - c;
			if (async16) {
				const unsigned bytes = left >= 4 ? 16u : (left > 0 ? 4u * (unsigned)left : 0u);
				const float *src = bytes ? x32 + c : x32; // nothing is read when bytes is 0
				const unsigned dst = (unsigned)__cvta_generic_to_shared(buf + 4 * q);
				asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
			} else {
#pragma unroll
				for (int e = 0; e < 4; e++) buf[4 * q + e] = e < left ? __ldg(x32 + c + e) : 0.f;
			}
		}
		asm volatile("cp.async.commit_group;" ::: "memory");
	};
	int tile = blockIdx.x;
	if (tile < ntile) stage(tile, sx);
	for (int it = 0; tile < ntile; it++, tile += gridDim.x) {
		float *cur = sx + (it & 1) * tstride;
		asm volatile("cp.async.wait_group 0;" ::: "memory");
		// this tile's copies are visible to all; every thread is done with the
		// tile before, whose buffer the next copies overwrite
		__syncthreads();
		if (tile + (int)gridDim.x < ntile) stage(tile + gridDim.x, sx + ((it + 1) & 1) * tstride);
		const int t = tile * SELL_TILE + threadIdx.x;
		const int slice = t / SELL_C, l = t % SELL_C;
		if (slice < nsl) {
			const long long base = __ldg(off + slice);
			const int w = (int)((__ldg(off + slice + 1) - base) / SELL_C);
			const float *vp = sval + base + l;
			const unsigned *cp = cpair + base / 2 + l;
			double sum = 0.0;
			int k = 0;
			for (; k + 8 <= w; k += 8) {
				unsigned cc[4];
				float a[8];
#pragma unroll
				for (int u = 0; u < 4; u++) cc[u] = __ldcs(cp + SELL_C * (k / 2 + u));
#pragma unroll
				for (int u = 0; u < 8; u++) a[u] = __ldcs(vp + SELL_C * (k + u));
#pragma unroll
				for (int u = 0; u < 4; u++) {
					sum = fma((double)a[2 * u], (double)cur[cc[u] & 0xffffu], sum);
					sum = fma((double)a[2 * u + 1], (double)cur[cc[u] >> 16], sum);
				}
			}
			for (; k < w; k += 2) {
				const unsigned cc = __ldcs(cp + SELL_C * (k / 2));
				sum = fma((double)__ldcs(vp + SELL_C * k), (double)cur[cc & 0xffffu], sum);
				sum = fma((double)__ldcs(vp + SELL_C * (k + 1)), (double)cur[cc >> 16], sum);
			}
			if (t < n) {
				const int r = perm ? __ldg(perm + t) : t;
				const double v = (rhs[r] - sum) * dinv[r];
				if (OUT64) y[r] = v;
				else y32[r] = (float)v;
			}
		}
	}
}

template <typename VT>
__global__ void k_sell_fill(int n, const int *rp, const int *ci, const double *v, int skip, const int *perm,
                            int longlen, const long long *off, int *scol, VT *sval) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int slice = t / SELL_C, l = t % SELL_C;
	if (slice >= nsl) return;
	const int r = t < n ? (perm ? perm[t] : t) : n;
	const long long base = off[slice];
	const int w = (int)((off[slice + 1] - base) / SELL_C);
	const int b = r < n ? rp[r] + skip : 0;
	int len = r < n ? rp[r + 1] - b : 0;
	if (longlen > 0 && len > longlen) len = 0; // a long row: padding only
	for (int k = 0; k < w; k++) {
		const long long p = base + (long long)SELL_C * k + l;
		if (k < len) {
			scol[p] = ci[b + k];
			sval[p] = (VT)v[b + k];
		} else {
			scol[p] = r < n ? r : 0;
			sval[p] = (VT)0;
		}
	}
}

// y = A x (OUT 0) or y = (x - N yin) * dinv (OUT 1); IN 1 forms
// yin[c] = x[c] * dinv[c] on the fly (the first two Jacobi iterates in one
// pass).  LG: the matrix has long rows (without, the kernel keeps the
// registers, and so the occupancy, of the plain slice loop).
template <typename VT, int IN, int OUT, bool LG>
__global__ void __launch_bounds__(256) k_sell_apply(int n, const int *__restrict__ perm,
                                                    const long long *__restrict__ off,
                                                    const int *__restrict__ scol, const VT *__restrict__ sval,
                                                    const double *__restrict__ xin, const double *__restrict__ dinv_in,
                                                    const double *__restrict__ xrhs,
                                                    const double *__restrict__ dinv_out, double *__restrict__ y,
                                                    sell_long<VT> lg) {
	constexpr int SPW = 32 / SELL_C; // slices per warp
	if (LG)
		long_rows<VT, double, IN>(lg, xin, dinv_in, [&](int r, double sum) {
			if (OUT == 0) y[r] = sum;
			else y[r] = (xrhs[r] - sum) * dinv_out[r];
		});
	const int lane = threadIdx.x & 31;
	const int grp = lane / SELL_C, l = lane % SELL_C;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int s0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * SPW; s0 < nsl; s0 += nwarps * SPW) {
		const int slice = s0 + grp;
		if (slice >= nsl) continue;
		const long long base = __ldg(off + slice);
		const int w = (int)((__ldg(off + slice + 1) - base) / SELL_C);
		const unsigned lm = LG && lg.mask ? __ldg(lg.mask + slice) : 0u;
		const int *cp = scol + base + l;
		const VT *vp = sval + base + l;
		double sum = 0.0;
		int k = 0;
		for (; k + 8 <= w; k += 8) {
			int c[8];
			double a[8], xv[8];
#pragma unroll
			for (int u = 0; u < 8; u++) {
				c[u] = __ldcs(cp + SELL_C * (k + u));
				a[u] = (double)__ldcs(vp + SELL_C * (k + u));
			}
#pragma unroll
			for (int u = 0; u < 8; u++) {
				xv[u] = __ldg(xin + c[u]);
				if (IN == 1) xv[u] *= __ldg(dinv_in + c[u]);
			}
#pragma unroll
			for (int u = 0; u < 8; u++) sum = fma(a[u], xv[u], sum);
		}
		for (; k < w; k++) {
			const int c = __ldcs(cp + SELL_C * k);
			const double a = (double)__ldcs(vp + SELL_C * k);
			double xv = __ldg(xin + c);
			if (IN == 1) xv *= __ldg(dinv_in + c);
			sum = fma(a, xv, sum);
		}
		const int t = slice * SELL_C + l;
		if (t < n && !((lm >> l) & 1u)) {
			const int r = perm ? __ldg(perm + t) : t;
			if (OUT == 0) y[r] = sum;
			else y[r] = (xrhs[r] - sum) * dinv_out[r];
		}
	}
}

// One Jacobi pass of an FP32 factor with FP32 iterates: out = (rhs - N x32)
// * dinv, written as FP64 (the last pass, OUT64 1) or as the FP32 iterate the
// next pass gathers (OUT64 0).  Gathering 4-byte iterates halves the
// sector traffic of the gathers; the products and sums stay FP64.
template <int OUT64, bool LG>
__global__ void __launch_bounds__(256) k_sell_sweep32(int n, const int *__restrict__ perm,
                                                      const long long *__restrict__ off,
                                                      const int *__restrict__ scol, const float *__restrict__ sval,
                                                      const float *__restrict__ x32, const double *__restrict__ rhs,
                                                      const double *__restrict__ dinv, double *__restrict__ y,
                                                      float *__restrict__ y32, sell_long<float> lg) {
	constexpr int SPW = 32 / SELL_C;
	if (LG)
		long_rows<float, float, 0>(lg, x32, nullptr, [&](int r, double sum) {
			const double v = (rhs[r] - sum) * dinv[r];
			if (OUT64) y[r] = v;
			else y32[r] = (float)v;
		});
	const int lane = threadIdx.x & 31;
	const int grp = lane / SELL_C, l = lane % SELL_C;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int s0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * SPW; s0 < nsl; s0 += nwarps * SPW) {
		const int slice = s0 + grp;
		if (slice >= nsl) continue;
		const long long base = __ldg(off + slice);
		const int w = (int)((__ldg(off + slice + 1) - base) / SELL_C);
		const unsigned lm = LG && lg.mask ? __ldg(lg.mask + slice) : 0u;
		const int *cp = scol + base + l;
		const float *vp = sval + base + l;
		double sum = 0.0;
		int k = 0;
		for (; k + 8 <= w; k += 8) {
			int c[8];
			float a[8], xv[8];
#pragma unroll
			for (int u = 0; u < 8; u++) {
				c[u] = __ldcs(cp + SELL_C * (k + u));
				a[u] = __ldcs(vp + SELL_C * (k + u));
			}
#pragma unroll
			for (int u = 0; u < 8; u++) xv[u] = __ldg(x32 + c[u]);
#pragma unroll
			for (int u = 0; u < 8; u++) sum = fma((double)a[u], (double)xv[u], sum);
		}
		for (; k < w; k++) {
			const int c = __ldcs(cp + SELL_C * k);
			sum = fma((double)__ldcs(vp + SELL_C * k), (double)__ldg(x32 + c), sum);
		}
		const int t = slice * SELL_C + l;
		if (t < n && !((lm >> l) & 1u)) {
			const int r = perm ? __ldg(perm + t) : t;
			const double v = (rhs[r] - sum) * dinv[r];
			if (OUT64) y[r] = v;
			else y32[r] = (float)v;
		}
	}
}

// ---- several vectors ------------------------------------------------------
// The products of k_sell_apply / k_sell_sweep32 for nr <= NRM vectors at
// stride ld (vector q at x + q ld), the matrix read once: every lane keeps
// NRM sums.  Per vector the products are summed in the single-vector
// kernels' order (entry by entry per lane, then the same trees for long
// rows), so each vector's result is bit-identical to a single-vector call.

template <typename VT, typename XT, int IN, bool BLOCK, int NRM>
__device__ __forceinline__ void long_row_sum_m(long long b, long long e, int tid, int nr, long long ld,
                                               const int *__restrict__ lcol, const VT *__restrict__ lval,
                                               const XT *__restrict__ x, const double *__restrict__ dinv_in,
                                               double (*red)[8], double *sum) {
	constexpr int T = BLOCK ? 256 : 32;
#pragma unroll
	for (int q = 0; q < NRM; q++) sum[q] = 0.0;
#pragma unroll 2
	for (long long j = b + tid; j < e; j += T) {
		const int c = __ldcs(lcol + j);
		const double a = (double)__ldcs(lval + j);
		const double di = IN == 1 ? __ldg(dinv_in + c) : 1.0;
#pragma unroll
		for (int q = 0; q < NRM; q++)
			if (q < nr) {
				double xv = (double)__ldg(x + q * ld + c);
				if (IN == 1) xv *= di;
				sum[q] = fma(a, xv, sum[q]);
			}
	}
#pragma unroll
	for (int q = 0; q < NRM; q++) sum[q] = warp_sum(sum[q]);
	if (BLOCK) {
		if ((tid & 31) == 0)
#pragma unroll
			for (int q = 0; q < NRM; q++) red[q][tid >> 5] = sum[q];
		__syncthreads();
#pragma unroll
		for (int q = 0; q < NRM; q++) {
			double t = 0.0;
#pragma unroll
			for (int w = 0; w < 8; w++) t += red[q][w];
			sum[q] = t;
		}
		__syncthreads();
	}
}

template <typename VT, typename XT, int IN, int NRM, typename F>
__device__ __forceinline__ void long_rows_m(const sell_long<VT> &lg, int nr, long long ld, const XT *__restrict__ x,
                                            const double *__restrict__ dinv_in, F out) {
	if (!lg.nlong) return;
	__shared__ double red[NRM][8];
	double sum[NRM];
	for (int i = blockIdx.x; i < lg.nvlong; i += gridDim.x) {
		long_row_sum_m<VT, XT, IN, true, NRM>(__ldg(lg.off + i), __ldg(lg.off + i + 1), threadIdx.x, nr, ld, lg.col,
		                                      lg.val, x, dinv_in, red, sum);
		if (threadIdx.x == 0) {
			const int r = __ldg(lg.row + i);
#pragma unroll
			for (int q = 0; q < NRM; q++)
				if (q < nr) out(r, q, sum[q]);
		}
	}
	const int lane = threadIdx.x & 31;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int i = lg.nvlong + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < lg.nlong; i += nwarps) {
		long_row_sum_m<VT, XT, IN, false, NRM>(__ldg(lg.off + i), __ldg(lg.off + i + 1), lane, nr, ld, lg.col, lg.val,
		                                       x, dinv_in, nullptr, sum);
		if (lane == 0) {
			const int r = __ldg(lg.row + i);
#pragma unroll
			for (int q = 0; q < NRM; q++)
				if (q < nr) out(r, q, sum[q]);
		}
	}
}

// Slice part of the several-vector kernels: the NRM sums of slot l of a slice.
template <typename VT, typename XT, int IN, int NRM>
__device__ __forceinline__ void slice_sums_m(int w, const int *__restrict__ cp, const VT *__restrict__ vp, int nr,
                                             long long ld, const XT *__restrict__ x,
                                             const double *__restrict__ dinv_in, double *sum) {
#pragma unroll
	for (int q = 0; q < NRM; q++) sum[q] = 0.0;
	int k = 0;
	for (; k + 4 <= w; k += 4) {
		int c[4];
		double a[4];
#pragma unroll
		for (int u = 0; u < 4; u++) {
			c[u] = __ldcs(cp + SELL_C * (k + u));
			a[u] = (double)__ldcs(vp + SELL_C * (k + u));
		}
#pragma unroll
		for (int u = 0; u < 4; u++) {
			const double di = IN == 1 ? __ldg(dinv_in + c[u]) : 1.0;
#pragma unroll
			for (int q = 0; q < NRM; q++)
				if (q < nr) {
					double xv = (double)__ldg(x + q * ld + c[u]);
					if (IN == 1) xv *= di;
					sum[q] = fma(a[u], xv, sum[q]);
				}
		}
	}
	for (; k < w; k++) {
		const int c = __ldcs(cp + SELL_C * k);
		const double a = (double)__ldcs(vp + SELL_C * k);
		const double di = IN == 1 ? __ldg(dinv_in + c) : 1.0;
#pragma unroll
		for (int q = 0; q < NRM; q++)
			if (q < nr) {
				double xv = (double)__ldg(x + q * ld + c);
				if (IN == 1) xv *= di;
				sum[q] = fma(a, xv, sum[q]);
			}
	}
}

// k_sell_apply for nr vectors (the pivots dinv_in / dinv_out are shared)
template <typename VT, int IN, int OUT, int NRM>
__global__ void __launch_bounds__(256) k_sell_apply_m(int n, int nr, long long ld, const int *__restrict__ perm,
                                                      const long long *__restrict__ off,
                                                      const int *__restrict__ scol, const VT *__restrict__ sval,
                                                      const double *__restrict__ xin,
                                                      const double *__restrict__ dinv_in,
                                                      const double *__restrict__ xrhs,
                                                      const double *__restrict__ dinv_out, double *__restrict__ y,
                                                      sell_long<VT> lg) {
	constexpr int SPW = 32 / SELL_C;
	auto out = [&](int r, int q, double sum) {
		if (OUT == 0) y[q * ld + r] = sum;
		else y[q * ld + r] = (xrhs[q * ld + r] - sum) * dinv_out[r];
	};
	long_rows_m<VT, double, IN, NRM>(lg, nr, ld, xin, dinv_in, out);
	const int lane = threadIdx.x & 31;
	const int grp = lane / SELL_C, l = lane % SELL_C;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int s0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * SPW; s0 < nsl; s0 += nwarps * SPW) {
		const int slice = s0 + grp;
		if (slice >= nsl) continue;
		const long long base = __ldg(off + slice);
		const int w = (int)((__ldg(off + slice + 1) - base) / SELL_C);
		const unsigned lm = lg.mask ? __ldg(lg.mask + slice) : 0u;
		double sum[NRM];
		slice_sums_m<VT, double, IN, NRM>(w, scol + base + l, sval + base + l, nr, ld, xin, dinv_in, sum);
		const int t = slice * SELL_C + l;
		if (t < n && !((lm >> l) & 1u)) {
			const int r = perm ? __ldg(perm + t) : t;
#pragma unroll
			for (int q = 0; q < NRM; q++)
				if (q < nr) out(r, q, sum[q]);
		}
	}
}

// k_sell_sweep32 for nr vectors: FP32 iterates x32 + q ld in, out to
// y + q ld (OUT64) or y32 + q ld
template <int OUT64, int NRM>
__global__ void __launch_bounds__(256) k_sell_sweep32_m(int n, int nr, long long ld, const int *__restrict__ perm,
                                                        const long long *__restrict__ off,
                                                        const int *__restrict__ scol, const float *__restrict__ sval,
                                                        const float *__restrict__ x32, const double *__restrict__ rhs,
                                                        const double *__restrict__ dinv, double *__restrict__ y,
                                                        float *__restrict__ y32, sell_long<float> lg) {
	constexpr int SPW = 32 / SELL_C;
	auto out = [&](int r, int q, double sum) {
		const double v = (rhs[q * ld + r] - sum) * dinv[r];
		if (OUT64) y[q * ld + r] = v;
		else y32[q * ld + r] = (float)v;
	};
	long_rows_m<float, float, 0, NRM>(lg, nr, ld, x32, nullptr, out);
	const int lane = threadIdx.x & 31;
	const int grp = lane / SELL_C, l = lane % SELL_C;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	for (int s0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * SPW; s0 < nsl; s0 += nwarps * SPW) {
		const int slice = s0 + grp;
		if (slice >= nsl) continue;
		const long long base = __ldg(off + slice);
		const int w = (int)((__ldg(off + slice + 1) - base) / SELL_C);
		const unsigned lm = lg.mask ? __ldg(lg.mask + slice) : 0u;
		double sum[NRM];
		slice_sums_m<float, float, 0, NRM>(w, scol + base + l, sval + base + l, nr, ld, x32, nullptr, sum);
		const int t = slice * SELL_C + l;
		if (t < n && !((lm >> l) & 1u)) {
			const int r = perm ? __ldg(perm + t) : t;
#pragma unroll
			for (int q = 0; q < NRM; q++)
				if (q < nr) out(r, q, sum[q]);
		}
	}
}

// x32 + q n = (x + q n) * dinv rounded to FP32, q < nr
__global__ void k_scale32_m(int n, int nr, const double *x, const double *dinv, float *x32) {
	const long long N = (long long)n * nr;
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
		x32[i] = (float)(x[i] * dinv[i % n]);
}

// x32 = x * dinv rounded to FP32 (the first Jacobi iterate)
__global__ void k_scale32(int n, const double *x, const double *dinv, float *x32) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		x32[i] = (float)(x[i] * dinv[i]);
}

inline int nb(long long n, int t) { return n > 0 ? (int)((n + t - 1) / t) : 1; }

} // namespace

// Build SELL-8 of a CSR matrix (device arrays); skip = 1 drops the first
// entry of every row (the diagonal of a factor row).  Values are stored as VT.
__global__ void k_len_keys(int n, const int *rp, int skip, int sigma, unsigned long long *keys, int *vals) {
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= n) return;
	int len = rp[r + 1] - rp[r] - skip;
	if (len < 0) len = 0;
	if (len > 0xfffff) len = 0xfffff;
	// window ascending, then longer rows first, then row index (stable)
	keys[r] = ((unsigned long long)(r / sigma) << 20) | (unsigned long long)(0xfffff - len);
	vals[r] = r;
}

static void bsg_sell_untile(bsg_sell *m, cudaStream_t s) {
	if (m->tb_off) cudaFreeAsync(m->tb_off, s);
	if (m->tb) cudaFreeAsync(m->tb, s);
	if (m->cpair) cudaFreeAsync(m->cpair, s);
	m->tb_off = nullptr;
	m->tb = nullptr;
	m->cpair = nullptr;
	m->ntile = 0;
	m->tmax = 0;
	m->tgrid = 0;
}

// The tiled form of a built SELL matrix (widths even).  A tile whose entries
// touch more than TB_MAX blocks of x leaves the matrix untiled (the sweeps
// then gather from global memory): that is not an error.
static int bsg_sell_tile(bsg_ctx *c, int n, const int *rp, const int *ci, int skip, bsg_sell *m) {
	cudaStream_t s = c->stream;
	const int ntile = (n + SELL_TILE - 1) / SELL_TILE;
	const int grid = ntile < BSG_SMS * 8 ? ntile : BSG_SMS * 8;
	int *cnt = nullptr, *bad = nullptr;
	BSG_CUDA(cudaMallocAsync(&cnt, sizeof(int) * (ntile + 1), s));
	BSG_CUDA(cudaMallocAsync(&bad, sizeof(int), s));
	BSG_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
	BSG_CUDA(cudaMemsetAsync(cnt + ntile, 0, sizeof(int), s));
	BSG_COUNT(1);
	k_tile_blocks<0><<<grid, SELL_TILE, 0, s>>>(n, rp, ci, skip, m->perm, m->off, ntile, cnt, bad, nullptr, nullptr,
	                                            nullptr);
	BSG_CUDA(cudaGetLastError());
	int hbad = 0;
	BSG_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	cudaFreeAsync(bad, s);
	if (hbad) {
		cudaFreeAsync(cnt, s);
		return BSG_OK;
	}
	// most blocks of a tile, then the offsets (exclusive scan)
	int *dmax = nullptr;
	void *tmp = nullptr;
	size_t t1 = 0, t2 = 0;
	BSG_CUDA(cudaMallocAsync(&dmax, sizeof(int), s));
	BSG_CUDA(cudaMallocAsync(&m->tb_off, sizeof(int) * (ntile + 1), s));
	BSG_CUDA(cub::DeviceReduce::Max(nullptr, t1, cnt, dmax, ntile, s));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t2, cnt, m->tb_off, ntile + 1, s));
	BSG_CUDA(cudaMallocAsync(&tmp, (t1 > t2 ? t1 : t2) + 1, s));
	BSG_CUDA(cub::DeviceReduce::Max(tmp, t1, cnt, dmax, ntile, s));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t2, cnt, m->tb_off, ntile + 1, s));
	int h[2] = {0, 0};
	BSG_CUDA(cudaMemcpyAsync(h, dmax, sizeof(int), cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaMemcpyAsync(h + 1, m->tb_off + ntile, sizeof(int), cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	cudaFreeAsync(tmp, s);
	cudaFreeAsync(dmax, s);
	cudaFreeAsync(cnt, s);
	m->ntile = ntile;
	m->tmax = h[0];
	BSG_CUDA(cudaMallocAsync(&m->tb, sizeof(int) * (h[1] > 0 ? h[1] : 1), s));
	BSG_CUDA(cudaMallocAsync(&m->cpair, sizeof(unsigned) * (m->entries / 2 > 0 ? m->entries / 2 : 1), s));
	BSG_COUNT(1);
	k_tile_blocks<1><<<grid, SELL_TILE, 0, s>>>(n, rp, ci, skip, m->perm, m->off, ntile, nullptr, nullptr, m->tb_off,
	                                            m->tb, m->cpair);
	BSG_CUDA(cudaGetLastError());
	// persistent grid: as many tiles at once as the staging lets reside
	// the limit covers every tiled form: the L and U copies of one factor
	// (and other factors) stage different amounts, and the attribute is per
	// kernel, not per launch
	const size_t smem = 2 * (size_t)m->tmax * 32 * sizeof(float); // two staging buffers
	const int smem_cap = 2 * TB_MAX * 32 * (int)sizeof(float);
	BSG_CUDA(cudaFuncSetAttribute(k_tsell_sweep32<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap));
	BSG_CUDA(cudaFuncSetAttribute(k_tsell_sweep32<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap));
	int per_sm = 0;
	BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tsell_sweep32<0>, SELL_TILE, smem));
	if (per_sm < 1) {
		bsg_sell_untile(m, s);
		return BSG_OK;
	}
	m->tgrid = ntile < BSG_SMS * per_sm ? ntile : BSG_SMS * per_sm;
	return BSG_OK;
}

// The long rows of a CSR matrix into m->lrow / loff / lcol / lval: first the
// rows of more than SELL_VLONG entries, then those of more than SELL_LONG,
// each group in row order.
template <typename VT>
static int bsg_sell_long(bsg_ctx *c, int n, const int *rp, const int *ci, const double *v, int skip, bsg_sell *m) {
	cudaStream_t s = c->stream;
	unsigned char *fv, *fl;
	int *iota, *sel, *num;
	BSG_CUDA(cudaMallocAsync(&fv, n, s));
	BSG_CUDA(cudaMallocAsync(&fl, n, s));
	BSG_CUDA(cudaMallocAsync(&iota, sizeof(int) * n, s));
	BSG_CUDA(cudaMallocAsync(&sel, sizeof(int) * 2 * (size_t)n, s));
	BSG_CUDA(cudaMallocAsync(&num, sizeof(int) * 2, s));
	const int g = nb(n, 256) < BSG_SMS * 8 ? nb(n, 256) : BSG_SMS * 8;
	BSG_COUNT(1);
	k_long_flags<<<g, 256, 0, s>>>(n, rp, skip, fv, fl, iota);
	size_t tb = 0;
	BSG_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, iota, fv, sel, num, n, s));
	void *tmp;
	BSG_CUDA(cudaMallocAsync(&tmp, tb > 0 ? tb : 1, s));
	BSG_CUDA(cub::DeviceSelect::Flagged(tmp, tb, iota, fv, sel, num, n, s));
	BSG_CUDA(cub::DeviceSelect::Flagged(tmp, tb, iota, fl, sel + n, num + 1, n, s));
	int h[2] = {0, 0};
	BSG_CUDA(cudaMemcpyAsync(h, num, sizeof(int) * 2, cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	cudaFreeAsync(tmp, s);
	cudaFreeAsync(fv, s);
	cudaFreeAsync(fl, s);
	cudaFreeAsync(iota, s);
	cudaFreeAsync(num, s);
	const int nl = h[0] + h[1];
	if (nl == 0) {
		cudaFreeAsync(sel, s);
		return BSG_OK;
	}
	m->nlong = nl;
	m->nvlong = h[0];
	BSG_CUDA(cudaMallocAsync(&m->lrow, sizeof(int) * nl, s));
	if (h[0]) BSG_CUDA(cudaMemcpyAsync(m->lrow, sel, sizeof(int) * h[0], cudaMemcpyDeviceToDevice, s));
	if (h[1]) BSG_CUDA(cudaMemcpyAsync(m->lrow + h[0], sel + n, sizeof(int) * h[1], cudaMemcpyDeviceToDevice, s));
	cudaFreeAsync(sel, s);
	long long *len;
	BSG_CUDA(cudaMallocAsync(&len, sizeof(long long) * (nl + 1), s));
	BSG_CUDA(cudaMallocAsync(&m->loff, sizeof(long long) * (nl + 1), s));
	BSG_COUNT(1);
	k_long_len<<<nb(nl + 1, 256), 256, 0, s>>>(nl, m->lrow, rp, skip, len);
	size_t ts = 0;
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, ts, len, m->loff, nl + 1, s));
	BSG_CUDA(cudaMallocAsync(&tmp, ts > 0 ? ts : 1, s));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, ts, len, m->loff, nl + 1, s));
	long long total = 0;
	BSG_CUDA(cudaMemcpyAsync(&total, m->loff + nl, sizeof(long long), cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	cudaFreeAsync(tmp, s);
	cudaFreeAsync(len, s);
	BSG_CUDA(cudaMallocAsync(&m->lcol, sizeof(int) * total, s));
	BSG_CUDA(cudaMallocAsync(&m->lval, sizeof(VT) * total, s));
	BSG_COUNT(1);
	k_long_fill<VT><<<nb((long long)nl * 32, 256) < BSG_SMS * 8 ? nb((long long)nl * 32, 256) : BSG_SMS * 8, 256, 0,
	                  s>>>(nl, m->lrow, m->loff, rp, ci, v, skip, m->lcol, (VT *)m->lval);
	BSG_CUDA(cudaGetLastError());
	m->entries += total;
	return BSG_OK;
}

template <typename VT>
int bsg_sell_build_t(bsg_ctx *c, int n, const int *rp, const int *ci, const double *v, int skip, bsg_sell *out,
                     int sigma, int tiled) {
	cudaStream_t s = c->stream;
	const int nsl = (n + SELL_C - 1) / SELL_C;
	out->perm = nullptr;
	out->entries = 0;
	if (n > 0) {
		int rc = bsg_sell_long<VT>(c, n, rp, ci, v, skip, out);
		if (rc) return rc;
	}
	// the tiled form has no long rows
	if (out->nlong) tiled = 0;
	if (sigma > 0 && n > 0) {
		// SELL-C-sigma: rows sorted by length inside windows of sigma rows
		unsigned long long *keys, *k2;
		int *vals;
		BSG_CUDA(cudaMallocAsync(&keys, sizeof(unsigned long long) * n, s));
		BSG_CUDA(cudaMallocAsync(&k2, sizeof(unsigned long long) * n, s));
		BSG_CUDA(cudaMallocAsync(&vals, sizeof(int) * n, s));
		BSG_CUDA(cudaMallocAsync(&out->perm, sizeof(int) * n, s));
		BSG_COUNT(1);
		k_len_keys<<<nb(n, 256), 256, 0, s>>>(n, rp, skip, sigma, keys, vals);
		size_t t2 = 0;
		int end_bit = 20;
		while ((1ull << (end_bit - 20)) <= (unsigned long long)(n / sigma + 1)) end_bit++;
		BSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t2, keys, k2, vals, out->perm, n, 0, end_bit, s));
		void *d_t2;
		BSG_CUDA(cudaMallocAsync(&d_t2, t2 > 0 ? t2 : 1, s));
		BSG_CUDA(cub::DeviceRadixSort::SortPairs(d_t2, t2, keys, k2, vals, out->perm, n, 0, end_bit, s));
		cudaFreeAsync(keys, s); cudaFreeAsync(k2, s); cudaFreeAsync(vals, s); cudaFreeAsync(d_t2, s);
	}
	const int longlen = out->nlong ? SELL_LONG : 0;
	if (out->nlong) BSG_CUDA(cudaMallocAsync(&out->lmask, nsl > 0 ? nsl : 1, s));
	long long *width;
	BSG_CUDA(cudaMallocAsync(&width, sizeof(long long) * (nsl + 1), s));
	BSG_CUDA(cudaMallocAsync(&out->off, sizeof(long long) * (nsl + 1), s));
	BSG_CUDA(cudaMemsetAsync(width + nsl, 0, sizeof(long long), s));
	BSG_COUNT(2);
	k_sell_width<<<nb((long long)nsl * SELL_C, 256), 256, 0, s>>>(n, rp, skip, out->perm, tiled, longlen, width,
	                                                               out->lmask);
	// off = exclusive scan of the slice sizes
	size_t tmp = 0;
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, width, out->off, nsl + 1, s));
	void *d_tmp;
	BSG_CUDA(cudaMallocAsync(&d_tmp, tmp > 0 ? tmp : 1, s));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, width, out->off, nsl + 1, s));
	long long total = 0;
	BSG_CUDA(cudaMemcpyAsync(&total, out->off + nsl, sizeof(long long), cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	out->n = n;
	out->entries += total;
	BSG_CUDA(cudaMallocAsync(&out->col, sizeof(int) * (total > 0 ? total : 1), s));
	BSG_CUDA(cudaMallocAsync(&out->val, sizeof(VT) * (total > 0 ? total : 1), s));
	out->fp32 = sizeof(VT) == 4;
	k_sell_fill<VT><<<nb((long long)nsl * SELL_C, 256), 256, 0, s>>>(n, rp, ci, v, skip, out->perm, longlen, out->off,
	                                                                out->col, (VT *)out->val);
	BSG_CUDA(cudaGetLastError());
	BSG_CUDA(cudaFreeAsync(width, s));
	BSG_CUDA(cudaFreeAsync(d_tmp, s));
	return tiled ? bsg_sell_tile(c, n, rp, ci, skip, out) : BSG_OK;
}

int bsg_sell_build(bsg_ctx *c, int n, const int *rp, const int *ci, const double *v, int skip, int fp32,
                   bsg_sell *out, int sigma, int tiled) {
	// the tiles must hold whole sorting windows
	tiled = tiled && fp32 && n > 0 && (sigma <= 0 || (SELL_TILE % sigma) == 0);
	return fp32 ? bsg_sell_build_t<float>(c, n, rp, ci, v, skip, out, sigma, tiled)
	            : bsg_sell_build_t<double>(c, n, rp, ci, v, skip, out, sigma, 0);
}

void bsg_sell_free(bsg_sell *m, cudaStream_t s) {
	bsg_sell_untile(m, s);
	if (m->lrow) cudaFreeAsync(m->lrow, s);
	if (m->loff) cudaFreeAsync(m->loff, s);
	if (m->lcol) cudaFreeAsync(m->lcol, s);
	if (m->lval) cudaFreeAsync(m->lval, s);
	if (m->lmask) cudaFreeAsync(m->lmask, s);
	m->lrow = nullptr;
	m->loff = nullptr;
	m->lcol = nullptr;
	m->lval = nullptr;
	m->lmask = nullptr;
	m->nlong = m->nvlong = 0;
	if (m->perm) cudaFreeAsync(m->perm, s);
	m->perm = nullptr;
	if (m->off) cudaFreeAsync(m->off, s);
	if (m->col) cudaFreeAsync(m->col, s);
	if (m->val) cudaFreeAsync(m->val, s);
	m->off = nullptr;
	m->col = nullptr;
	m->val = nullptr;
}

// CTAs of 256 threads of a kernel that are resident at once: the sliced
// loops stride over the grid, so more would only add a partial second wave
template <typename K>
static int wave_cap(K kern, int g) {
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
	const int cap = (per_sm > 0 ? per_sm : 1) * BSG_SMS;
	return g < cap ? g : cap;
}

static int sell_grid(int n) {
	int warps = (n + 31) / 32;
	int blocks = (warps + 7) / 8;
	int cap = BSG_SMS * 8;
	return blocks < 1 ? 1 : (blocks < cap ? blocks : cap);
}

// y = A x
int bsg_sell_spmv(cudaStream_t s, const bsg_sell *m, const double *x, double *y) {
	BSG_COUNT(1);
	const int g = sell_grid(m->n);
#define BSG_SPMV(VT, LG)                                                                                               \
	k_sell_apply<VT, 0, 0, LG><<<g, 256, 0, s>>>(m->n, m->perm, m->off, m->col, (const VT *)m->val, x, nullptr, nullptr, \
	                                             nullptr, y, long_of<VT>(m))
	if (m->fp32) {
		if (m->nlong) BSG_SPMV(float, true); else BSG_SPMV(float, false);
	} else {
		if (m->nlong) BSG_SPMV(double, true); else BSG_SPMV(double, false);
	}
#undef BSG_SPMV
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// One Jacobi pass yout = (x - N yin) * dinv; scaled_in: yin = x * dinv.
int bsg_sell_sweep(cudaStream_t s, const bsg_sell *m, const double *x, const double *dinv, const double *yin,
                   int scaled_in, double *yout) {
	BSG_COUNT(1);
	const int g = sell_grid(m->n);
#define BSG_SW(VT, IN, LG)                                                                                             \
	k_sell_apply<VT, IN, 1, LG><<<g, 256, 0, s>>>(m->n, m->perm, m->off, m->col, (const VT *)m->val,                     \
	                                              IN ? x : yin, IN ? dinv : nullptr, x, dinv, yout, long_of<VT>(m))
	const bool lg = m->nlong > 0;
	if (m->fp32) {
		if (scaled_in) { if (lg) BSG_SW(float, 1, true); else BSG_SW(float, 1, false); }
		else { if (lg) BSG_SW(float, 0, true); else BSG_SW(float, 0, false); }
	} else {
		if (scaled_in) { if (lg) BSG_SW(double, 1, true); else BSG_SW(double, 1, false); }
		else { if (lg) BSG_SW(double, 0, true); else BSG_SW(double, 0, false); }
	}
#undef BSG_SW
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// Jacobi sweeps of an FP32 factor with FP32 iterates: nsweeps >= 2 iterates
// in total (the first, D^-1 x, formed by k_scale32), the last written to
// yout in FP64.  work32 holds 2 n floats (the ping-pong iterates).
int bsg_sell_sweeps32(cudaStream_t s, const bsg_sell *m, const double *x, const double *dinv, int nsweeps,
                      float *work32, double *yout) {
	if (!m->fp32 || nsweeps < 2) return BSG_ERR_ARG;
	const int n = m->n, g = sell_grid(n);
	const float *v = (const float *)m->val;
	float *a = work32, *b = work32 + n;
	BSG_COUNT(nsweeps);
	k_scale32<<<nb(n, 256) < BSG_SMS * 16 ? nb(n, 256) : BSG_SMS * 16, 256, 0, s>>>(n, x, dinv, b);
	const size_t smem = 2 * (size_t)m->tmax * 32 * sizeof(float);
	const int tstride = m->tmax * 32;
	for (int pass = 0; pass < nsweeps - 1; pass++) {
		const bool last = pass == nsweeps - 2;
		if (m->ntile) {
			if (last)
				k_tsell_sweep32<1><<<m->tgrid, SELL_TILE, smem, s>>>(n, m->ntile, m->perm, m->off, m->cpair, v, m->tb_off,
				                                                     m->tb, b, x, dinv, yout, nullptr, tstride);
			else
				k_tsell_sweep32<0><<<m->tgrid, SELL_TILE, smem, s>>>(n, m->ntile, m->perm, m->off, m->cpair, v, m->tb_off,
				                                                     m->tb, b, x, dinv, nullptr, a, tstride);
		} else if (last) {
			if (m->nlong)
				k_sell_sweep32<1, true><<<g, 256, 0, s>>>(n, m->perm, m->off, m->col, v, b, x, dinv, yout, nullptr,
				                                          long_of<float>(m));
			else
				k_sell_sweep32<1, false><<<g, 256, 0, s>>>(n, m->perm, m->off, m->col, v, b, x, dinv, yout, nullptr,
				                                           long_of<float>(m));
		} else {
			if (m->nlong)
				k_sell_sweep32<0, true><<<g, 256, 0, s>>>(n, m->perm, m->off, m->col, v, b, x, dinv, nullptr, a,
				                                          long_of<float>(m));
			else
				k_sell_sweep32<0, false><<<g, 256, 0, s>>>(n, m->perm, m->off, m->col, v, b, x, dinv, nullptr, a,
				                                           long_of<float>(m));
		}
		float *t = a; a = b; b = t;
	}
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// One full FP32-iterate pass (timing of the sweep kernel alone).
int bsg_sell_sweep32_pass(cudaStream_t s, const bsg_sell *m, const double *x, const double *dinv, const float *x32,
                          double *yout) {
	BSG_COUNT(1);
	if (m->ntile)
		k_tsell_sweep32<1><<<m->tgrid, SELL_TILE, 2 * (size_t)m->tmax * 32 * sizeof(float), s>>>(
		    m->n, m->ntile, m->perm, m->off, m->cpair, (const float *)m->val, m->tb_off, m->tb, x32, x, dinv, yout, nullptr,
		    m->tmax * 32);
	else if (m->nlong)
		k_sell_sweep32<1, true><<<sell_grid(m->n), 256, 0, s>>>(m->n, m->perm, m->off, m->col, (const float *)m->val,
		                                                        x32, x, dinv, yout, nullptr, long_of<float>(m));
	else
		k_sell_sweep32<1, false><<<sell_grid(m->n), 256, 0, s>>>(m->n, m->perm, m->off, m->col, (const float *)m->val,
		                                                         x32, x, dinv, yout, nullptr, long_of<float>(m));
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// Stored entries (with padding) of a SELL matrix: the bytes a product reads.
long long bsg_sell_entries(const bsg_sell *m) { return m->entries; }

// ---- several vectors: launchers -------------------------------------------
// Vectors at stride n (vector q at x + q n), nr >= 1; the matrix is read once
// per group of up to 8 vectors.

// One Jacobi pass for nr vectors: yout = (x - N yin) * dinv; scaled_in: yin
// = x * dinv.
int bsg_sell_sweep_multi(cudaStream_t s, const bsg_sell *m, int nr, const double *x, const double *dinv,
                         const double *yin, int scaled_in, double *yout) {
	const int n = m->n, g = sell_grid(n);
	const long long ld = n;
	for (int q0 = 0; q0 < nr; q0 += 8) {
		const int k = nr - q0 < 8 ? nr - q0 : 8;
		const long long o = (long long)q0 * n;
		const double *xi = scaled_in ? x + o : yin + o;
		BSG_COUNT(1);
#define BSG_SW(VT, NRM)                                                                                                \
	do {                                                                                                               \
		const VT *v = (const VT *)m->val;                                                                              \
		if (scaled_in)                                                                                                 \
			k_sell_apply_m<VT, 1, 1, NRM><<<wave_cap(k_sell_apply_m<VT, 1, 1, NRM>, g), 256, 0, s>>>(                    \
			    n, k, ld, m->perm, m->off, m->col, v, xi, dinv, x + o, dinv, yout + o, long_of<VT>(m));                  \
		else                                                                                                           \
			k_sell_apply_m<VT, 0, 1, NRM><<<wave_cap(k_sell_apply_m<VT, 0, 1, NRM>, g), 256, 0, s>>>(                    \
			    n, k, ld, m->perm, m->off, m->col, v, xi, nullptr, x + o, dinv, yout + o, long_of<VT>(m));               \
	} while (0)
		if (m->fp32) {
			if (k <= 4) BSG_SW(float, 4);
			else BSG_SW(float, 8);
		} else {
			if (k <= 4) BSG_SW(double, 4);
			else BSG_SW(double, 8);
		}
#undef BSG_SW
	}
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// bsg_sell_sweeps32 for nr vectors; work32 holds 2 n nr floats.  The tiled
// form is not used (its staging is per vector).
int bsg_sell_sweeps32_multi(cudaStream_t s, const bsg_sell *m, int nr, const double *x, const double *dinv,
                            int nsweeps, float *work32, double *yout) {
	if (!m->fp32 || nsweeps < 2) return BSG_ERR_ARG;
	const int n = m->n, g = sell_grid(n);
	const long long ld = n;
	float *a = work32, *b = work32 + (size_t)n * nr;
	BSG_COUNT(1);
	{
		const long long N = (long long)n * nr;
		const int gs = nb(N, 256) < BSG_SMS * 16 ? nb(N, 256) : BSG_SMS * 16;
		k_scale32_m<<<gs, 256, 0, s>>>(n, nr, x, dinv, b);
	}
	const float *v = (const float *)m->val;
	const sell_long<float> lg = long_of<float>(m);
	for (int pass = 0; pass < nsweeps - 1; pass++) {
		const bool last = pass == nsweeps - 2;
		for (int q0 = 0; q0 < nr; q0 += 8) {
			const int k = nr - q0 < 8 ? nr - q0 : 8;
			const long long o = (long long)q0 * n;
			BSG_COUNT(1);
			if (last) {
				if (k <= 4)
					k_sell_sweep32_m<1, 4><<<wave_cap(k_sell_sweep32_m<1, 4>, g), 256, 0, s>>>(n, k, ld, m->perm, m->off, m->col, v, b + o, x + o, dinv,
					                                         yout + o, nullptr, lg);
				else
					k_sell_sweep32_m<1, 8><<<wave_cap(k_sell_sweep32_m<1, 8>, g), 256, 0, s>>>(n, k, ld, m->perm, m->off, m->col, v, b + o, x + o, dinv,
					                                         yout + o, nullptr, lg);
			} else {
				if (k <= 4)
					k_sell_sweep32_m<0, 4><<<wave_cap(k_sell_sweep32_m<0, 4>, g), 256, 0, s>>>(n, k, ld, m->perm, m->off, m->col, v, b + o, x + o, dinv,
					                                         nullptr, a + o, lg);
				else
					k_sell_sweep32_m<0, 8><<<wave_cap(k_sell_sweep32_m<0, 8>, g), 256, 0, s>>>(n, k, ld, m->perm, m->off, m->col, v, b + o, x + o, dinv,
					                                         nullptr, a + o, lg);
			}
		}
		float *t = a; a = b; b = t;
	}
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}
