// Block SELL of 3 x 3 blocks for the Jacobi sweeps of a block factor
// (CSMatrixRS::SolveL / SolveU in sweep mode, Bslib/mvm.cpp:3140 / 3410).
//
// Layout.  Block rows are cut into slices of 8; slice s has width w_s = the
// most blocks of its rows, block k of slot l stores its block column at
// off_s + 8 k + l and its 9 values (row-major) in planes, value p at
// 9 off_s + 72 k + 8 p + l.  A group of 8 lanes serves one slice, lane l one
// block row: every column load is one 32-byte sector, every value plane one
// sector (FP32) or two (FP64), and the 3 gathered x values of a block sit in
// one or two sectors.  Against the point expansion (a column index per
// entry) the factor shrinks from 9 x (4 + 4) = 72 to 4 + 36 = 40 bytes per
// FP32 block.
//
// One pass y <- D (x - N y) is one kernel: the lane holding block row i has
// its three sums and applies the 3 x 3 diagonal block D_i itself.
// Per point row the products are summed block by block in column order,
// entries of a block in column order: the order of the sequential loop.
//
// Block rows of more than BS_LONG blocks (the wrap-around fill of periodic
// problems) leave the slices and are summed by a warp, or by a whole block
// beyond BS_VLONG blocks, in the same kernel.  Their blocks are padded to a
// multiple of 32 and stored in chunks of 32 with the values in planes
// (value p of block j at 9 (j - j % 32) + 32 p + j % 32), so the 32 lanes of
// a warp read one chunk's planes as whole lines.
#include "bsg_internal.cuh"
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#define BS_C 8
#define BS_LONG 64
#define BS_VLONG 1024

namespace {

inline int nbk(long long n, int t) { return n > 0 ? (int)((n + t - 1) / t) : 1; }
inline int capped(long long n, int t) {
	const int g = nbk(n, t);
	return g < BSG_SMS * 8 ? g : BSG_SMS * 8;
}

__device__ __forceinline__ int blen(const int *rp, int i) { return (rp[3 * i + 1] - rp[3 * i]) / 3; }

__global__ void k_bs_flags(int nb, const int *rp, unsigned char *fv, unsigned char *fl, int *iota) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
		const int len = blen(rp, i);
		fv[i] = len > BS_VLONG;
		fl[i] = len > BS_LONG && len <= BS_VLONG;
		iota[i] = i;
	}
}

// blocks of the long rows, each padded to a multiple of 32
__global__ void k_bs_len(int nl, const int *lrow, const int *rp, long long *len) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= nl; i += gridDim.x * blockDim.x)
		len[i] = i < nl ? (blen(rp, lrow[i]) + 31) & ~31 : 0;
}

// one warp per long block row: chunk layout, padding blocks (column = the
// row itself, values 0) after the row's own
template <typename VT>
__global__ void k_bs_long_fill(int nl, const int *lrow, const long long *loff, const int *rp, const int *ci,
                               const double *v, int *lcol, VT *lval) {
	const int lane = threadIdx.x & 31;
	for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nl; i += (gridDim.x * blockDim.x) >> 5) {
		const int r = lrow[i];
		const int len = blen(rp, r);
		const long long o = loff[i], plen = loff[i + 1] - o;
		for (long long k = lane; k < plen; k += 32) {
			const long long j = o + k;
			VT *vp = lval + 9 * (j & ~31LL) + (j & 31);
			if (k < len) {
				lcol[j] = ci[rp[3 * r] + 3 * k] / 3;
#pragma unroll
				for (int p = 0; p < 9; p++) vp[32 * p] = (VT)v[rp[3 * r + p / 3] + 3 * k + p % 3];
			} else {
				lcol[j] = r;
#pragma unroll
				for (int p = 0; p < 9; p++) vp[32 * p] = (VT)0;
			}
		}
	}
}

// slice widths (blocks) without the long rows; bit l of lmask marks them
__global__ void k_bs_width(int nb, const int *rp, int longlen, long long *width, unsigned char *lmask) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int slice = t / BS_C;
	const int nsl = (nb + BS_C - 1) / BS_C;
	int len = t < nb ? blen(rp, t) : 0;
	const bool lng = longlen > 0 && len > longlen;
	if (lng) len = 0;
	const unsigned bits = __ballot_sync(0xffffffffu, lng);
#pragma unroll
	for (int o = BS_C / 2; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, o, BS_C));
	if ((t % BS_C) == 0 && slice < nsl) {
		width[slice] = (long long)BS_C * len;
		if (lmask) lmask[slice] = (unsigned char)(bits >> (threadIdx.x & 31 & ~(BS_C - 1)));
	}
}

template <typename VT>
__global__ void k_bs_fill(int nb, const int *rp, const int *ci, const double *v, int longlen, const long long *off,
                          int *col, VT *val) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	const int nsl = (nb + BS_C - 1) / BS_C;
	const int slice = t / BS_C, l = t % BS_C;
	if (slice >= nsl) return;
	const long long base = off[slice];
	const int w = (int)((off[slice + 1] - base) / BS_C);
	int len = t < nb ? blen(rp, t) : 0;
	if (longlen > 0 && len > longlen) len = 0;
	for (int k = 0; k < w; k++) {
		const long long p0 = base + (long long)BS_C * k + l;
		const long long v0 = 9 * base + 72LL * k + l;
		if (k < len) {
			col[p0] = ci[rp[3 * t] + 3 * k] / 3;
#pragma unroll
			for (int p = 0; p < 9; p++) val[v0 + BS_C * p] = (VT)v[rp[3 * t + p / 3] + 3 * k + p % 3];
		} else {
			col[p0] = t < nb ? t : 0;
#pragma unroll
			for (int p = 0; p < 9; p++) val[v0 + BS_C * p] = (VT)0;
		}
	}
}

template <typename VT>
struct bs_long {
	int nlong, nvlong;
	const int *row;
	const long long *off;
	const int *col;
	const VT *val;
	const unsigned char *mask;
};

// y_i = D_i (x_i - s) for one vector, x_i at ox and y_i at oy (D_i column-major)
__device__ __forceinline__ void bs_out(int i, long long ox, long long oy, const double *__restrict__ d,
                                       const double *__restrict__ x, const double *s, double *__restrict__ y) {
	const double *b = d + 9 * (size_t)i;
	const double t0 = x[ox] - s[0], t1 = x[ox + 1] - s[1], t2 = x[ox + 2] - s[2];
#pragma unroll
	for (int r = 0; r < 3; r++) y[oy + r] = fma(__ldg(b + r + 6), t2, fma(__ldg(b + r + 3), t1, __ldg(b + r) * t0));
}

// s[r] += row r of block a times (x0, x1, x2), entries in column order
template <typename VT>
__device__ __forceinline__ void bs_acc(const VT *a, double x0, double x1, double x2, double *s) {
#pragma unroll
	for (int r = 0; r < 3; r++) {
		s[r] = fma((double)a[3 * r], x0, s[r]);
		s[r] = fma((double)a[3 * r + 1], x1, s[r]);
		s[r] = fma((double)a[3 * r + 2], x2, s[r]);
	}
}

// s[q][r] += the products of block (J, a) with vector q.  Vectors either at
// stride ld (entry (J, q, r) at q ld + 3 J + r) or, with IL, interleaved by
// block row (entry at J ri + 3 q + r; ri even and the base 16-byte aligned),
// where a block's nr vectors are 3 nr contiguous doubles read as pairs.
template <int NRM, bool IL, typename VT>
__device__ __forceinline__ void bs_block(int J, const VT *a, int nr, long long ld, int ri,
                                         const double *__restrict__ y, double (*s)[3]) {
	if constexpr (IL) {
		static_assert(NRM % 2 == 0, "interleaved vectors in pairs");
		const double *yj = y + (long long)J * ri;
#pragma unroll
		for (int q = 0; q < NRM; q += 2) {
			if (q + 1 < nr) {
				const double2 p0 = __ldg(reinterpret_cast<const double2 *>(yj + 3 * q));
				const double2 p1 = __ldg(reinterpret_cast<const double2 *>(yj + 3 * q + 2));
				const double2 p2 = __ldg(reinterpret_cast<const double2 *>(yj + 3 * q + 4));
				bs_acc(a, p0.x, p0.y, p1.x, s[q]);
				bs_acc(a, p1.y, p2.x, p2.y, s[q + 1]);
			} else if (q < nr) { // the last of an odd count
				const double2 p0 = __ldg(reinterpret_cast<const double2 *>(yj + 3 * q));
				bs_acc(a, p0.x, p0.y, __ldg(yj + 3 * q + 2), s[q]);
			}
		}
	} else {
#pragma unroll
		for (int q = 0; q < NRM; q++)
			if (q < nr) {
				const double *yq = y + q * ld + 3 * (long long)J;
				bs_acc(a, __ldg(yq), __ldg(yq + 1), __ldg(yq + 2), s[q]);
			}
	}
}

// Sums of a long block row's blocks [b, e) (b, e multiples of 32) by a warp
// (tid = lane) or a block of 256 threads: thread t takes blocks t, t + T, ...
// in order, then a fixed tree; every thread gets the sums.
template <typename VT, bool BLOCK, int NRM, bool IL>
__device__ __forceinline__ void bs_long_sum(long long b, long long e, int tid, int nr, long long ld, int ri,
                                            const int *__restrict__ lcol, const VT *__restrict__ lval,
                                            const double *__restrict__ y, double (*red)[8], double (*s)[3]) {
	constexpr int T = BLOCK ? 256 : 32;
#pragma unroll
	for (int q = 0; q < NRM; q++) s[q][0] = s[q][1] = s[q][2] = 0.0;
#pragma unroll 2
	for (long long j = b + tid; j < e; j += T) {
		const int J = __ldcs(lcol + j);
		const VT *vp = lval + 9 * (j & ~31LL) + (j & 31);
		VT a[9];
#pragma unroll
		for (int p = 0; p < 9; p++) a[p] = __ldcs(vp + 32 * p);
		bs_block<NRM, IL>(J, a, nr, ld, ri, y, s);
	}
#pragma unroll
	for (int q = 0; q < NRM; q++)
#pragma unroll
		for (int r = 0; r < 3; r++) s[q][r] = warp_sum(s[q][r]);
	if (BLOCK) {
		if ((tid & 31) == 0)
#pragma unroll
			for (int q = 0; q < NRM; q++)
#pragma unroll
				for (int r = 0; r < 3; r++) red[3 * q + r][tid >> 5] = s[q][r];
		__syncthreads();
#pragma unroll
		for (int q = 0; q < NRM; q++)
#pragma unroll
			for (int r = 0; r < 3; r++) {
				double t = 0.0;
#pragma unroll
				for (int w = 0; w < 8; w++) t += red[3 * q + r][w];
				s[q][r] = t;
			}
		__syncthreads();
	}
}

// One pass yout = D (x - N yin) for nr <= NRM vectors; x at stride ld, yin
// and yout at stride ld or (LIN / LOUT) interleaved with row strides ri / ro.
template <typename VT, int NRM, bool LIN, bool LOUT>
// (256, 1): no register cap, so that the U blocks' values of the FP64
// single-vector pass are all in flight (122 registers; 40 under the default
// cap ran a third slower)
__global__ void __launch_bounds__(256, 1) k_bsell_sweep(int nb, int nr, long long ld, int ri, int ro,
                                                     const long long *__restrict__ off, const int *__restrict__ col,
                                                     const VT *__restrict__ val, const double *__restrict__ d,
                                                     const double *__restrict__ x, const double *__restrict__ yin,
                                                     double *__restrict__ yout, bs_long<VT> lg) {
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int nwarps = (gridDim.x * blockDim.x) >> 5;
	double s[NRM][3];
	auto out = [&](int r) {
#pragma unroll
		for (int q = 0; q < NRM; q++)
			if (q < nr)
				bs_out(r, q * ld + 3 * (long long)r, LOUT ? (long long)r * ro + 3 * q : q * ld + 3 * (long long)r, d, x,
				       s[q], yout);
	};
	if (lg.nlong) {
		__shared__ double red[3 * NRM][8];
		for (int i = blockIdx.x; i < lg.nvlong; i += gridDim.x) {
			bs_long_sum<VT, true, NRM, LIN>(__ldg(lg.off + i), __ldg(lg.off + i + 1), threadIdx.x, nr, ld, ri, lg.col,
			                                lg.val, yin, red, s);
			if (threadIdx.x == 0) out(__ldg(lg.row + i));
		}
		for (int i = lg.nvlong + gw; i < lg.nlong; i += nwarps) {
			bs_long_sum<VT, false, NRM, LIN>(__ldg(lg.off + i), __ldg(lg.off + i + 1), lane, nr, ld, ri, lg.col, lg.val,
			                                 yin, nullptr, s);
			if (lane == 0) out(__ldg(lg.row + i));
		}
	}
	constexpr int SPW = 32 / BS_C;
	const int grp = lane / BS_C, l = lane % BS_C;
	const int nsl = (nb + BS_C - 1) / BS_C;
	for (int s0 = gw * SPW; s0 < nsl; s0 += nwarps * SPW) {
		const int slice = s0 + grp;
		if (slice >= nsl) continue;
		const long long base = __ldg(off + slice);
		const int w = (int)((__ldg(off + slice + 1) - base) / BS_C);
		const unsigned lm = lg.mask ? __ldg(lg.mask + slice) : 0u;
		const int *cp = col + base + l;
		const VT *vp = val + 9 * base + l;
#pragma unroll
		for (int q = 0; q < NRM; q++) s[q][0] = s[q][1] = s[q][2] = 0.0;
		// U blocks' columns and values in flight at once, then their gathers
		constexpr int U = NRM == 1 ? 4 : 2;
		int k = 0;
		for (; k + U <= w; k += U) {
			int J[U];
			VT a[U][9];
#pragma unroll
			for (int u = 0; u < U; u++) {
				J[u] = __ldcs(cp + BS_C * (k + u));
#pragma unroll
				for (int p = 0; p < 9; p++) a[u][p] = __ldcs(vp + 72LL * (k + u) + BS_C * p);
			}
#pragma unroll
			for (int u = 0; u < U; u++) bs_block<NRM, LIN>(J[u], a[u], nr, ld, ri, yin, s);
		}
		for (; k < w; k++) {
			const int J = __ldcs(cp + BS_C * k);
			VT a[9];
#pragma unroll
			for (int p = 0; p < 9; p++) a[p] = __ldcs(vp + 72LL * k + BS_C * p);
			bs_block<NRM, LIN>(J, a, nr, ld, ri, yin, s);
		}
		const int i = slice * BS_C + l;
		if (i < nb && !((lm >> l) & 1u)) out(i);
	}
}

// y = D x for nr vectors, x at stride 3 nb, y at stride 3 nb or (ro > 0)
// interleaved with row stride ro (the first Jacobi iterate)
__global__ void k_bs_diag(int nb, int nr, int ro, const double *__restrict__ d, const double *__restrict__ x,
                          double *__restrict__ y) {
	const long long N = (long long)nb * nr;
	const double zero[3] = {0.0, 0.0, 0.0};
	for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(e % nb);
		const long long q = e / nb, ox = 3 * q * nb + 3 * i;
		bs_out(i, ox, ro > 0 ? (long long)i * ro + 3 * q : ox, d, x, zero, y);
	}
}

template <typename VT>
int bsell_long(bsg_ctx *c, int nb, const int *rp, const int *ci, const double *v, bsg_bsell *m) {
	cudaStream_t s = c->stream;
	unsigned char *fv, *fl;
	int *iota, *sel, *num;
	BSG_CUDA(cudaMallocAsync(&fv, nb, s));
	BSG_CUDA(cudaMallocAsync(&fl, nb, s));
	BSG_CUDA(cudaMallocAsync(&iota, sizeof(int) * nb, s));
	BSG_CUDA(cudaMallocAsync(&sel, sizeof(int) * 2 * (size_t)nb, s));
	BSG_CUDA(cudaMallocAsync(&num, sizeof(int) * 2, s));
	BSG_COUNT(1);
	k_bs_flags<<<capped(nb, 256), 256, 0, s>>>(nb, rp, fv, fl, iota);
	size_t tb = 0;
	BSG_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, iota, fv, sel, num, nb, s));
	void *tmp;
	BSG_CUDA(cudaMallocAsync(&tmp, tb > 0 ? tb : 1, s));
	BSG_CUDA(cub::DeviceSelect::Flagged(tmp, tb, iota, fv, sel, num, nb, s));
	BSG_CUDA(cub::DeviceSelect::Flagged(tmp, tb, iota, fl, sel + nb, num + 1, nb, s));
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
	if (h[1]) BSG_CUDA(cudaMemcpyAsync(m->lrow + h[0], sel + nb, sizeof(int) * h[1], cudaMemcpyDeviceToDevice, s));
	cudaFreeAsync(sel, s);
	long long *len;
	BSG_CUDA(cudaMallocAsync(&len, sizeof(long long) * (nl + 1), s));
	BSG_CUDA(cudaMallocAsync(&m->loff, sizeof(long long) * (nl + 1), s));
	BSG_COUNT(1);
	k_bs_len<<<nbk(nl + 1, 256), 256, 0, s>>>(nl, m->lrow, rp, len);
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
	BSG_CUDA(cudaMallocAsync(&m->lval, sizeof(VT) * 9 * total, s));
	BSG_COUNT(1);
	k_bs_long_fill<VT><<<capped((long long)nl * 32, 256), 256, 0, s>>>(nl, m->lrow, m->loff, rp, ci, v, m->lcol,
	                                                                   (VT *)m->lval);
	BSG_CUDA(cudaGetLastError());
	m->blocks += total;
	return BSG_OK;
}

template <typename VT>
int bsell_build(bsg_ctx *c, int nb, const int *rp, const int *ci, const double *v, bsg_bsell *out) {
	cudaStream_t s = c->stream;
	const int nsl = (nb + BS_C - 1) / BS_C;
	out->nb = nb;
	out->fp32 = sizeof(VT) == 4;
	out->blocks = 0;
	if (nb > 0) {
		int rc = bsell_long<VT>(c, nb, rp, ci, v, out);
		if (rc) return rc;
	}
	const int longlen = out->nlong ? BS_LONG : 0;
	if (out->nlong) BSG_CUDA(cudaMallocAsync(&out->lmask, nsl > 0 ? nsl : 1, s));
	long long *width;
	BSG_CUDA(cudaMallocAsync(&width, sizeof(long long) * (nsl + 1), s));
	BSG_CUDA(cudaMallocAsync(&out->off, sizeof(long long) * (nsl + 1), s));
	BSG_CUDA(cudaMemsetAsync(width + nsl, 0, sizeof(long long), s));
	BSG_COUNT(1);
	k_bs_width<<<nbk((long long)nsl * BS_C, 256), 256, 0, s>>>(nb, rp, longlen, width, out->lmask);
	size_t tmp = 0;
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, width, out->off, nsl + 1, s));
	void *d_tmp;
	BSG_CUDA(cudaMallocAsync(&d_tmp, tmp > 0 ? tmp : 1, s));
	BSG_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, width, out->off, nsl + 1, s));
	long long total = 0;
	BSG_CUDA(cudaMemcpyAsync(&total, out->off + nsl, sizeof(long long), cudaMemcpyDeviceToHost, s));
	BSG_CUDA(cudaStreamSynchronize(s));
	out->blocks += total;
	BSG_CUDA(cudaMallocAsync(&out->col, sizeof(int) * (total > 0 ? total : 1), s));
	BSG_CUDA(cudaMallocAsync(&out->val, sizeof(VT) * 9 * (total > 0 ? total : 1), s));
	BSG_COUNT(1);
	k_bs_fill<VT><<<nbk((long long)nsl * BS_C, 256), 256, 0, s>>>(nb, rp, ci, v, longlen, out->off, out->col,
	                                                              (VT *)out->val);
	BSG_CUDA(cudaGetLastError());
	cudaFreeAsync(width, s);
	cudaFreeAsync(d_tmp, s);
	return BSG_OK;
}

template <typename VT>
bs_long<VT> bs_long_of(const bsg_bsell *m) {
	return {m->nlong, m->nvlong, m->lrow, m->loff, m->lcol, (const VT *)m->lval, m->lmask};
}

// CTAs of a kernel that are resident at once (one wave): the sliced loops
// stride over the grid, so a grid beyond it only adds a partial second wave
template <typename VT, int NRM, bool LIN, bool LOUT>
void bs_launch(cudaStream_t s, const bsg_bsell *m, int g, int k, long long ld, int ri, int ro, const double *d,
               const double *x, const double *yin, double *yout) {
	static int cap = 0; // resident blocks of this instantiation on all SMs
	if (!cap) {
		int per_sm = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bsell_sweep<VT, NRM, LIN, LOUT>, 256, 0);
		cap = (per_sm > 0 ? per_sm : 1) * BSG_SMS;
	}
	k_bsell_sweep<VT, NRM, LIN, LOUT><<<min(g, cap), 256, 0, s>>>(m->nb, k, ld, ri, ro, m->off, m->col,
	                                                             (const VT *)m->val, d, x, yin, yout, bs_long_of<VT>(m));
}

// One pass over k vectors of a group; lin / lout pick the interleaved layouts
// (several vectors only).
template <typename VT>
void bs_pass(cudaStream_t s, const bsg_bsell *m, int g, int k, long long ld, int ri, int ro, bool lin, bool lout,
             const double *d, const double *x, const double *yin, double *yout) {
	if (k == 1) bs_launch<VT, 1, false, false>(s, m, g, k, ld, 0, 0, d, x, yin, yout);
	else if (lin && lout) {
		if (k <= 4) bs_launch<VT, 4, true, true>(s, m, g, k, ld, ri, ro, d, x, yin, yout);
		else bs_launch<VT, 8, true, true>(s, m, g, k, ld, ri, ro, d, x, yin, yout);
	} else if (lin) {
		if (k <= 4) bs_launch<VT, 4, true, false>(s, m, g, k, ld, ri, 0, d, x, yin, yout);
		else bs_launch<VT, 8, true, false>(s, m, g, k, ld, ri, 0, d, x, yin, yout);
	} else {
		if (k <= 4) bs_launch<VT, 4, false, false>(s, m, g, k, ld, 0, 0, d, x, yin, yout);
		else bs_launch<VT, 8, false, false>(s, m, g, k, ld, 0, 0, d, x, yin, yout);
	}
}

} // namespace

int bsg_bsell_build(bsg_ctx *c, int nb, const int *rp, const int *ci, const double *v, int fp32, bsg_bsell *out) {
	return fp32 ? bsell_build<float>(c, nb, rp, ci, v, out) : bsell_build<double>(c, nb, rp, ci, v, out);
}

void bsg_bsell_free(bsg_bsell *m, cudaStream_t s) {
	void *p[] = {m->off, m->col, m->val, m->lrow, m->loff, m->lcol, m->lval, m->lmask};
	for (void *q : p)
		if (q) cudaFreeAsync(q, s);
	*m = bsg_bsell();
}

size_t bsg_bsell_scratch(int nb, int nr) { return 2 * (size_t)nb * (size_t)(3 * nr + (nr & 1)); }

int bsg_bsell_sweeps(cudaStream_t s, const bsg_bsell *m, const double *d, int nsweeps, int nr, const double *x,
                     double *y, double *work, double *scr) {
	const int passes = nsweeps - 1;
	const int nb = m->nb;
	const long long ld = 3LL * nb;
	// Several vectors with scratch: the intermediate iterates alternate
	// between the two halves of scr, interleaved by block row (row stride
	// 3 nr rounded up to even), so that a block's gathers are 16-byte loads of
	// contiguous doubles; the last pass writes y at stride ld.  Otherwise the
	// iterates alternate between y and work at stride ld, the last one
	// landing in y.
	const bool il = passes > 0 && nr > 1 && scr && (reinterpret_cast<uintptr_t>(scr) & 15) == 0;
	if (passes > 0 && !il && !work) return bsg_set_error(BSG_ERR_ARG, "block sweeps: work vector missing");
	const int R = il ? 3 * nr + (nr & 1) : 0;
	double *bufs[2];
	if (il) bufs[0] = scr, bufs[1] = scr + (size_t)nb * R;
	else bufs[0] = y, bufs[1] = work;
	int a = il ? 0 : passes & 1;
	BSG_COUNT(1);
	k_bs_diag<<<capped((long long)nb * nr, 256), 256, 0, s>>>(nb, nr, R, d, x, bufs[a]);
	const int nsl = (nb + BS_C - 1) / BS_C;
	const int g = capped(nbk(nsl, 4), 8); // 4 slices a warp, 8 warps a block
	for (int p = 0; p < passes; p++) {
		const bool lout = il && p + 1 < passes;
		double *out = il && !lout ? y : bufs[a ^ 1];
		for (int q0 = 0; q0 < nr; q0 += 8) {
			const int k = nr - q0 < 8 ? nr - q0 : 8;
			const long long ox = (long long)q0 * ld, oi = il ? 3LL * q0 : ox, oo = lout ? 3LL * q0 : ox;
			BSG_COUNT(1);
			if (m->fp32) bs_pass<float>(s, m, g, k, ld, R, R, il, lout, d, x + ox, bufs[a] + oi, out + oo);
			else bs_pass<double>(s, m, g, k, ld, R, R, il, lout, d, x + ox, bufs[a] + oi, out + oo);
		}
		a ^= 1;
	}
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}
