// Device-side storage transforms for the solver path:
//   * symmetric expansion of an upper-stored matrix to both triangles (the
//     gather form of MvmASymm, Bslib/mvm.cpp:2637-2652);
//   * the CombineLU split (Bslib/smatrixr.cpp:1142-1258): the union upper
//     pattern with diagonal first plus the two value arrays al = A(j,i),
//     au = A(i,j);
//   * pattern transposes (static contributor lists for the factorisation,
//     row form of L for the forward solve).
// All transforms sort 64-bit (row << 32 | col) keys with CUB radix sort, then
// rebuild row pointers by binary search, so they are deterministic.
#include "bsg_internal.cuh"
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace {

__global__ void k_expand_keys(int n, const int *ia, const int *ja, unsigned long long *keys, int *vals, int *count) {
	// For each stored (i,j): emit (i,j); if j != i also emit (j,i).  Slots
	// are taken by an atomic counter; the sort restores a fixed order.
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	for (int k = ia[i]; k < ia[i + 1]; k++) {
		int j = ja[k];
		int s = atomicAdd(count, j != i ? 2 : 1);
		keys[s] = ((unsigned long long)(unsigned)i << 32) | (unsigned)j;
		vals[s] = k;
		if (j != i) {
			keys[s + 1] = ((unsigned long long)(unsigned)j << 32) | (unsigned)i;
			vals[s + 1] = k;
		}
	}
}

__global__ void k_split_keys(int n, const int *ia, const int *ja, unsigned long long *keys, int *vals) {
	// CombineLU: entry (i,j) goes to upper row min(i,j); vals carries the
	// source index and, in bit 31, whether it came from the lower triangle.
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	for (int k = ia[i]; k < ia[i + 1]; k++) {
		int j = ja[k];
		int r = j < i ? j : i, c = j < i ? i : j;
		keys[k] = ((unsigned long long)(unsigned)r << 32) | (unsigned)c;
		vals[k] = k | (j < i ? (int)0x80000000 : 0);
	}
}

__global__ void k_row_ptr(int n, int nk, const unsigned long long *keys, int *ia) {
	// ia[r] = first position with key row >= r (lower bound), r in [0, n].
	int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r > n) return;
	int lo = 0, hi = nk;
	while (lo < hi) {
		int mid = (lo + hi) >> 1;
		if ((int)(keys[mid] >> 32) < r) lo = mid + 1; else hi = mid;
	}
	ia[r] = lo;
}

__global__ void k_unique_flags(int nk, const unsigned long long *keys, int *flag) {
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nk) return;
	flag[k] = (k == 0 || keys[k] != keys[k - 1]) ? 1 : 0;
}

__global__ void k_split_scatter(int nk, const unsigned long long *keys, const int *vals, const int *pos,
                                const double *a, int *ja_out, double *al, double *au, unsigned long long *ukeys) {
	// pos[k] = inclusive scan of unique flags; slot = pos[k]-1.
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nk) return;
	int s = pos[k] - 1;
	unsigned long long key = keys[k];
	int r = (int)(key >> 32), c = (int)(key & 0xffffffffu);
	int v = vals[k];
	bool lower = v < 0;
	int src = v & 0x7fffffff;
	if (k == 0 || keys[k - 1] != key) {
		ja_out[s] = c;
		ukeys[s] = key;
	}
	// at most one lower and one upper (or one diagonal) source per key;
	// write without races by ownership: the diagonal writes both.
	if (r == c) {
		al[s] = a[src];
		au[s] = a[src];
	} else if (lower) {
		al[s] = a[src];
	} else {
		au[s] = a[src];
	}
}

__global__ void k_gather_vals(int nk, const int *vals, const double *a, double *out) {
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < nk) out[k] = a[vals[k]];
}

__global__ void k_cols_from_keys(int nk, const unsigned long long *keys, int *ja) {
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < nk) ja[k] = (int)(keys[k] & 0xffffffffu);
}

__global__ void k_strict_transpose_keys(int n, const int *ia, const int *ja, unsigned long long *keys, int *vals,
                                        int *count) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	for (int k = ia[i]; k < ia[i + 1]; k++) {
		int j = ja[k];
		if (j == i) continue;
		int s = atomicAdd(count, 1);
		keys[s] = ((unsigned long long)(unsigned)j << 32) | (unsigned)i;
		vals[s] = k;
	}
}

inline int nblk(long long n, int t) { return n > 0 ? (int)((n + t - 1) / t) : 1; }

} // namespace

// Sort (keys, vals) pairs on the context stream.  Keys < 2^63.
int bsg_sort_pairs(bsg_ctx *c, unsigned long long *keys, int *vals, int nk, int nbits_row) {
	if (nk <= 1) return BSG_OK;
	unsigned long long *k2;
	int *v2;
	BSG_CUDA(cudaMallocAsync(&k2, sizeof(unsigned long long) * nk, c->stream));
	BSG_CUDA(cudaMallocAsync(&v2, sizeof(int) * nk, c->stream));
	cub::DoubleBuffer<unsigned long long> dk(keys, k2);
	cub::DoubleBuffer<int> dv(vals, v2);
	size_t tmp = 0;
	int end_bit = 32 + nbits_row;
	BSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, nk, 0, end_bit, c->stream));
	void *d_tmp;
	BSG_CUDA(cudaMallocAsync(&d_tmp, tmp > 0 ? tmp : 1, c->stream));
	BSG_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tmp, dk, dv, nk, 0, end_bit, c->stream));
	if (dk.Current() != keys) {
		BSG_CUDA(cudaMemcpyAsync(keys, dk.Current(), sizeof(unsigned long long) * nk, cudaMemcpyDeviceToDevice, c->stream));
		BSG_CUDA(cudaMemcpyAsync(vals, dv.Current(), sizeof(int) * nk, cudaMemcpyDeviceToDevice, c->stream));
	}
	BSG_CUDA(cudaFreeAsync(d_tmp, c->stream));
	BSG_CUDA(cudaFreeAsync(k2, c->stream));
	BSG_CUDA(cudaFreeAsync(v2, c->stream));
	return BSG_OK;
}

static int bits_for(int n) {
	int b = 1;
	while ((1ll << b) <= (long long)n) b++;
	return b;
}

// Expand an upper-stored symmetric CSR (device arrays) to both triangles,
// columns ascending in every row.  Allocates *ia_o, *ja_o, *a_o.
int bsg_expand_symmetric(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, int nnz_up, int **ia_o,
                         int **ja_o, double **a_o, int *nnz_o) {
	int ndiag_max = nnz_up * 2;
	unsigned long long *keys;
	int *vals, *cnt;
	BSG_CUDA(cudaMallocAsync(&keys, sizeof(unsigned long long) * ndiag_max, c->stream));
	BSG_CUDA(cudaMallocAsync(&vals, sizeof(int) * ndiag_max, c->stream));
	BSG_CUDA(cudaMallocAsync(&cnt, sizeof(int), c->stream));
	BSG_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), c->stream));
	BSG_COUNT(4);
	k_expand_keys<<<nblk(n, 256), 256, 0, c->stream>>>(n, ia, ja, keys, vals, cnt);
	int nk = 0;
	BSG_CUDA(cudaMemcpyAsync(&nk, cnt, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
	BSG_CUDA(cudaStreamSynchronize(c->stream));
	int rc = bsg_sort_pairs(c, keys, vals, nk, bits_for(n));
	if (rc) return rc;
	BSG_CUDA(cudaMallocAsync(ia_o, sizeof(int) * (n + 1), c->stream));
	BSG_CUDA(cudaMallocAsync(ja_o, sizeof(int) * (nk > 0 ? nk : 1), c->stream));
	BSG_CUDA(cudaMallocAsync(a_o, sizeof(double) * (nk > 0 ? nk : 1), c->stream));
	k_row_ptr<<<nblk(n + 1, 256), 256, 0, c->stream>>>(n, nk, keys, *ia_o);
	k_cols_from_keys<<<nblk(nk, 256), 256, 0, c->stream>>>(nk, keys, *ja_o);
	k_gather_vals<<<nblk(nk, 256), 256, 0, c->stream>>>(nk, vals, a, *a_o);
	BSG_CUDA(cudaGetLastError());
	BSG_CUDA(cudaFreeAsync(keys, c->stream));
	BSG_CUDA(cudaFreeAsync(vals, c->stream));
	BSG_CUDA(cudaFreeAsync(cnt, c->stream));
	*nnz_o = nk;
	return BSG_OK;
}

// CombineLU on the device: union upper pattern (diagonal first because it is
// the smallest column >= row), al/au values.  Returns BSG_ERR_ARG when a
// diagonal entry is structurally missing.
int bsg_combine_lu(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, int nnz, int **iu_o,
                   int **ju_o, double **al_o, double **au_o, int *nnz_o) {
	unsigned long long *keys, *ukeys;
	int *vals, *flag, *pos;
	BSG_CUDA(cudaMallocAsync(&keys, sizeof(unsigned long long) * nnz, c->stream));
	BSG_CUDA(cudaMallocAsync(&vals, sizeof(int) * nnz, c->stream));
	BSG_COUNT(4);
	k_split_keys<<<nblk(n, 256), 256, 0, c->stream>>>(n, ia, ja, keys, vals);
	int rc = bsg_sort_pairs(c, keys, vals, nnz, bits_for(n));
	if (rc) return rc;
	BSG_CUDA(cudaMallocAsync(&flag, sizeof(int) * nnz, c->stream));
	BSG_CUDA(cudaMallocAsync(&pos, sizeof(int) * nnz, c->stream));
	k_unique_flags<<<nblk(nnz, 256), 256, 0, c->stream>>>(nnz, keys, flag);
	size_t tmp = 0;
	BSG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, flag, pos, nnz, c->stream));
	void *d_tmp;
	BSG_CUDA(cudaMallocAsync(&d_tmp, tmp > 0 ? tmp : 1, c->stream));
	BSG_CUDA(cub::DeviceScan::InclusiveSum(d_tmp, tmp, flag, pos, nnz, c->stream));
	int nu = 0;
	BSG_CUDA(cudaMemcpyAsync(&nu, pos + nnz - 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
	BSG_CUDA(cudaStreamSynchronize(c->stream));
	BSG_CUDA(cudaMallocAsync(iu_o, sizeof(int) * (n + 1), c->stream));
	BSG_CUDA(cudaMallocAsync(ju_o, sizeof(int) * nu, c->stream));
	BSG_CUDA(cudaMallocAsync(al_o, sizeof(double) * nu, c->stream));
	BSG_CUDA(cudaMallocAsync(au_o, sizeof(double) * nu, c->stream));
	BSG_CUDA(cudaMallocAsync(&ukeys, sizeof(unsigned long long) * nu, c->stream));
	BSG_CUDA(cudaMemsetAsync(*al_o, 0, sizeof(double) * nu, c->stream));
	BSG_CUDA(cudaMemsetAsync(*au_o, 0, sizeof(double) * nu, c->stream));
	k_split_scatter<<<nblk(nnz, 256), 256, 0, c->stream>>>(nnz, keys, vals, pos, a, *ju_o, *al_o, *au_o, ukeys);
	k_row_ptr<<<nblk(n + 1, 256), 256, 0, c->stream>>>(n, nu, ukeys, *iu_o);
	BSG_CUDA(cudaGetLastError());
	BSG_CUDA(cudaFreeAsync(keys, c->stream));
	BSG_CUDA(cudaFreeAsync(vals, c->stream));
	BSG_CUDA(cudaFreeAsync(flag, c->stream));
	BSG_CUDA(cudaFreeAsync(pos, c->stream));
	BSG_CUDA(cudaFreeAsync(d_tmp, c->stream));
	BSG_CUDA(cudaFreeAsync(ukeys, c->stream));
	*nnz_o = nu;
	return BSG_OK;
}

// Transpose of the strict part of a CSR pattern: row j lists the rows i < j
// with (i,j) stored, ascending.  perm[k] = source position of entry k.
int bsg_strict_transpose(bsg_ctx *c, int n, const int *ia, const int *ja, int nnz, int **it_o, int **jt_o,
                         int **perm_o, int *nnz_o) {
	unsigned long long *keys;
	int *vals, *cnt;
	BSG_CUDA(cudaMallocAsync(&keys, sizeof(unsigned long long) * (nnz > 0 ? nnz : 1), c->stream));
	BSG_CUDA(cudaMallocAsync(&vals, sizeof(int) * (nnz > 0 ? nnz : 1), c->stream));
	BSG_CUDA(cudaMallocAsync(&cnt, sizeof(int), c->stream));
	BSG_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), c->stream));
	BSG_COUNT(3);
	k_strict_transpose_keys<<<nblk(n, 256), 256, 0, c->stream>>>(n, ia, ja, keys, vals, cnt);
	int nk = 0;
	BSG_CUDA(cudaMemcpyAsync(&nk, cnt, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
	BSG_CUDA(cudaStreamSynchronize(c->stream));
	int rc = bsg_sort_pairs(c, keys, vals, nk, bits_for(n));
	if (rc) return rc;
	BSG_CUDA(cudaMallocAsync(it_o, sizeof(int) * (n + 1), c->stream));
	BSG_CUDA(cudaMallocAsync(jt_o, sizeof(int) * (nk > 0 ? nk : 1), c->stream));
	k_row_ptr<<<nblk(n + 1, 256), 256, 0, c->stream>>>(n, nk, keys, *it_o);
	k_cols_from_keys<<<nblk(nk, 256), 256, 0, c->stream>>>(nk, keys, *jt_o);
	BSG_CUDA(cudaGetLastError());
	BSG_CUDA(cudaFreeAsync(keys, c->stream));
	BSG_CUDA(cudaFreeAsync(cnt, c->stream));
	if (perm_o) *perm_o = vals; else BSG_CUDA(cudaFreeAsync(vals, c->stream));
	*nnz_o = nk;
	return BSG_OK;
}

namespace {
// Point row 3i+r of a block-CSR matrix with row-major bs x bs blocks: for
// every block k of block row i, columns bs*ja[k] + c with values
// a[bs*bs*k + bs*r + c].  Block columns ascending give point columns
// ascending.
__global__ void k_bsr_point_rows(int nsup, int bs, const int *ia, const int *ja, const double *a, int *pia, int *pja,
                                 double *pa) {
	const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (p >= (long long)nsup * bs) return;
	const int i = (int)(p / bs), r = (int)(p % bs);
	const int kb = ia[i], ke = ia[i + 1];
	int z = bs * bs * kb + r * bs * (ke - kb);
	pia[p] = z;
	if (p == (long long)nsup * bs - 1) pia[p + 1] = bs * bs * ke;
	for (int k = kb; k < ke; k++)
		for (int c = 0; c < bs; c++, z++) {
			pja[z] = bs * ja[k] + c;
			pa[z] = a[(size_t)bs * bs * k + bs * r + c];
		}
}
} // namespace

// Point CSR copy of a block-CSR matrix (row-major blocks): the operator the
// point factorisation of a block matrix works on.
int bsg_bsr_to_point(bsg_ctx *c, int nsup, int bs, const int *ia, const int *ja, const double *a, int nnzb, int **pia_o,
                     int **pja_o, double **pa_o) {
	const long long np = (long long)nsup * bs, nz = (long long)nnzb * bs * bs;
	if (nz > 0x7fffffffLL) return bsg_set_error(BSG_ERR_UNSUPPORTED, "point expansion exceeds 2^31 entries");
	BSG_CUDA(cudaMallocAsync(pia_o, sizeof(int) * (np + 1), c->stream));
	BSG_CUDA(cudaMallocAsync(pja_o, sizeof(int) * (nz > 0 ? nz : 1), c->stream));
	BSG_CUDA(cudaMallocAsync(pa_o, sizeof(double) * (nz > 0 ? nz : 1), c->stream));
	if (np == 0) BSG_CUDA(cudaMemsetAsync(*pia_o, 0, sizeof(int), c->stream));
	BSG_COUNT(1);
	k_bsr_point_rows<<<nblk(np, 256), 256, 0, c->stream>>>(nsup, bs, ia, ja, a, *pia_o, *pja_o, *pa_o);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

namespace {
__global__ void k_transpose_keys(int n, const int *ia, const int *ja, unsigned long long *keys, int *vals) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	for (int k = ia[i]; k < ia[i + 1]; k++) {
		keys[k] = ((unsigned long long)(unsigned)ja[k] << 32) | (unsigned)i;
		vals[k] = k;
	}
}
} // namespace

// Transpose of a full square CSR matrix (rows of A^T = columns of A, columns
// ascending), the operand of CSMatrixR::MvmAt in gather form.
int bsg_transpose_full(bsg_ctx *c, int n, const int *ia, const int *ja, const double *a, int nnz, int **ta_o,
                       int **tja_o, double **tv_o) {
	unsigned long long *keys;
	int *vals;
	BSG_CUDA(cudaMallocAsync(&keys, sizeof(unsigned long long) * (nnz > 0 ? nnz : 1), c->stream));
	BSG_CUDA(cudaMallocAsync(&vals, sizeof(int) * (nnz > 0 ? nnz : 1), c->stream));
	BSG_COUNT(1);
	k_transpose_keys<<<nblk(n, 256), 256, 0, c->stream>>>(n, ia, ja, keys, vals);
	int rc = bsg_sort_pairs(c, keys, vals, nnz, bits_for(n));
	if (rc) return rc;
	BSG_CUDA(cudaMallocAsync(ta_o, sizeof(int) * (n + 1), c->stream));
	BSG_CUDA(cudaMallocAsync(tja_o, sizeof(int) * (nnz > 0 ? nnz : 1), c->stream));
	BSG_CUDA(cudaMallocAsync(tv_o, sizeof(double) * (nnz > 0 ? nnz : 1), c->stream));
	BSG_COUNT(3);
	k_row_ptr<<<nblk(n + 1, 256), 256, 0, c->stream>>>(n, nnz, keys, *ta_o);
	k_cols_from_keys<<<nblk(nnz, 256), 256, 0, c->stream>>>(nnz, keys, *tja_o);
	k_gather_vals<<<nblk(nnz, 256), 256, 0, c->stream>>>(nnz, vals, a, *tv_o);
	BSG_CUDA(cudaGetLastError());
	BSG_CUDA(cudaFreeAsync(keys, c->stream));
	BSG_CUDA(cudaFreeAsync(vals, c->stream));
	return BSG_OK;
}

// ---- validation of a CSR pattern copied to the device ----------------------
// The checks of the host-buffer entry points, run where the arrays are:
// res[0] gets bit 0 for a decreasing row pointer, bit 1 for a column out of
// [0, n); res[1] / res[2] the first row that lacks its leading diagonal / has
// an entry below it (upper storage).
namespace {
__global__ void k_csr_rows_ok(int n, const int *__restrict__ ia, int *res) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		if (ia[i + 1] < ia[i]) atomicOr(res, 1);
}
__global__ void k_csr_cols_ok(int n, int nz, const int *__restrict__ ia, const int *__restrict__ ja, int upper,
                              int *res) {
	const int t0 = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
	for (int k = t0; k < nz; k += T) {
		const int c = ja[k];
		if (c < 0 || c >= n) atomicOr(res, 2);
	}
	if (upper)
		for (int i = t0; i < n; i += T) {
			const int a = ia[i], b = ia[i + 1];
			if (a == b || ja[a] != i) atomicMin(res + 1, i);
			for (int k = a; k < b; k++)
				if (ja[k] < i) {
					atomicMin(res + 2, i);
					break;
				}
		}
}
} // namespace

int bsg_check_csr_dev(bsg_ctx *c, int n, int nz, const int *d_ia, const int *d_ja, int stage, int upper) {
	cudaStream_t s = c->stream;
	int *d_res;
	const int init[3] = {0, 0x7fffffff, 0x7fffffff};
	BSG_CUDA(cudaMallocAsync(&d_res, sizeof(init), s));
	BSG_CUDA(cudaMemcpyAsync(d_res, init, sizeof(init), cudaMemcpyHostToDevice, s));
	BSG_COUNT(1);
	const long long work = stage == 0 ? n : (nz > n ? nz : n);
	const int g = (int)((work + 255) / 256 < BSG_SMS * 8 ? (work + 255) / 256 : BSG_SMS * 8);
	if (stage == 0) k_csr_rows_ok<<<g > 0 ? g : 1, 256, 0, s>>>(n, d_ia, d_res);
	else k_csr_cols_ok<<<g > 0 ? g : 1, 256, 0, s>>>(n, nz, d_ia, d_ja, upper, d_res);
	int res[3];
	const cudaError_t e = cudaMemcpyAsync(res, d_res, sizeof(res), cudaMemcpyDeviceToHost, s);
	cudaStreamSynchronize(s);
	cudaFreeAsync(d_res, s);
	BSG_CUDA(e);
	BSG_CUDA(cudaGetLastError());
	if (res[0] & 1) return bsg_set_error(BSG_ERR_ARG, "bad CSR: ia not monotone");
	if (res[0] & 2) return bsg_set_error(BSG_ERR_ARG, "bad CSR: column index out of range");
	if (res[1] != 0x7fffffff && res[1] <= res[2])
		return bsg_set_error(BSG_ERR_ARG, "symmetric input: every row must start with its diagonal");
	if (res[2] != 0x7fffffff) return bsg_set_error(BSG_ERR_ARG, "symmetric input: entry below the diagonal");
	return BSG_OK;
}

// ---- 3x3 block CSR from column-major input blocks ---------------------------
namespace {
__global__ void k_iota_d(int n, double *v) {
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) v[k] = (double)k;
}
// block k transposed in place: column-major (r, c) at 3 c + r to row-major
__global__ void k_bsr3_rowmajor(int nz, double *a) {
	for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nz; k += (long long)gridDim.x * blockDim.x) {
		double *b = a + 9 * k;
		const double t1 = b[1], t2 = b[2], t5 = b[5];
		b[1] = b[3];
		b[2] = b[6];
		b[5] = b[7];
		b[3] = t1;
		b[6] = t2;
		b[7] = t5;
	}
}
// full block row i from the upper input: A(i, j) = A_up(i, j) (j >= i), or
// A_up(j, i)^T (j < i); src[p] is the input block of entry p
__global__ void k_bsr3_fill_sym(int nb, const int *__restrict__ fia, const int *__restrict__ fja,
                                const double *__restrict__ src, const double *__restrict__ in, double *__restrict__ out) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
		for (int p = fia[i]; p < fia[i + 1]; p++) {
			const double *b = in + 9 * (long long)src[p];
			double *o = out + 9 * (long long)p;
			if (fja[p] >= i)
				for (int r = 0; r < 3; r++)
					for (int c = 0; c < 3; c++) o[3 * r + c] = b[3 * c + r];
			else
				for (int w = 0; w < 9; w++) o[w] = b[w];
		}
}
} // namespace

// Device 3x3 block CSR (blocks row-major) from device input with column-major
// blocks: as given (blocks transposed in place; ia, ja and a are taken over:
// *ia_o = ia, *ja_o = ja, *a_o = a), or (upper) expanded to both triangles
// with columns ascending in every row (*ia_o, *ja_o, *a_o allocated; ia, ja
// and a freed).  On failure the inputs stay the caller's.
int bsg_bsr3_from_input(bsg_ctx *c, int nb, int *ia, int *ja, double *a, int nz, int upper, int **ia_o, int **ja_o,
                        double **a_o, int *nnz_o) {
	cudaStream_t s = c->stream;
	const int cap = BSG_SMS * 8;
	if (!upper) {
		BSG_COUNT(1);
		k_bsr3_rowmajor<<<nblk(nz, 256) < cap ? nblk(nz, 256) : cap, 256, 0, s>>>(nz, a);
		BSG_CUDA(cudaGetLastError());
		*ia_o = ia;
		*ja_o = ja;
		*a_o = a;
		*nnz_o = nz;
		return BSG_OK;
	}
	double *idx, *src;
	BSG_CUDA(cudaMallocAsync(&idx, sizeof(double) * (nz > 0 ? nz : 1), s));
	BSG_COUNT(1);
	k_iota_d<<<nblk(nz, 256) < cap ? nblk(nz, 256) : cap, 256, 0, s>>>(nz, idx);
	int rc = bsg_expand_symmetric(c, nb, ia, ja, idx, nz, ia_o, ja_o, &src, nnz_o);
	cudaFreeAsync(idx, s);
	if (rc) return rc;
	BSG_CUDA(cudaMallocAsync(a_o, sizeof(double) * 9 * (size_t)(*nnz_o > 0 ? *nnz_o : 1), s));
	BSG_COUNT(1);
	k_bsr3_fill_sym<<<nblk(nb, 256), 256, 0, s>>>(nb, *ia_o, *ja_o, src, a, *a_o);
	cudaFreeAsync(src, s);
	cudaFreeAsync(ia, s);
	cudaFreeAsync(ja, s);
	cudaFreeAsync(a, s);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}
