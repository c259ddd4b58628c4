// Fused FP64 vector kernels of the Krylov loops (the reference's
// ScProdSVect / DaxpySVect / ScaleSVect, Bslib/svector.cpp:321-390, and the
// inline loops of Bslib/cg.cpp:247-285, Bslib/lanczos.cpp:684-697).
//
// Reductions are deterministic: a fixed grid of RED_BLOCKS blocks writes one
// partial per block and the last block to finish (ticket counter) sums the
// partials in block order, so results do not depend on scheduling.  Scalars
// stay on the device (d_s[]) so a loop needs no host round trip per kernel.
// Each reduction reads its vectors once: 16 B per element for a dot.
#include "bsg_internal.cuh"

#define RED_BLOCKS (2 * BSG_SMS)
#define RED_THREADS 256

namespace {

__device__ __forceinline__ double block_sum(double v, double *sh) {
	v = warp_sum(v);
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
	__syncthreads();
	if (l == 0) sh[w] = v;
	__syncthreads();
	double t = 0.0;
	if (threadIdx.x < 32) {
		t = (l < (int)(blockDim.x >> 5)) ? sh[l] : 0.0;
		t = warp_sum(t);
	}
	return t; // valid in thread 0
}

// Finish a Q-way reduction: partials[q*gridDim.x + b].  Returns true in the
// last block, which leaves the totals in out[q].
template <int Q>
__device__ bool finish_reduction(const double *vals, double *partials, unsigned int *counter, double *out,
                                 double *sh) {
	__shared__ bool last;
	for (int q = 0; q < Q; q++) {
		double t = block_sum(vals[q], sh);
		if (threadIdx.x == 0) partials[q * gridDim.x + blockIdx.x] = t;
	}
	__threadfence();
	__syncthreads();
	if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
	__syncthreads();
	if (!last) return false;
	__threadfence();
	for (int q = 0; q < Q; q++) {
		double v = 0.0;
		for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += __ldcg(partials + q * gridDim.x + b);
		double t = block_sum(v, sh);
		if (threadIdx.x == 0) out[q] = t;
	}
	if (threadIdx.x == 0) *counter = 0;
	return true;
}

// out[q] = x_q . y_q for Q pairs.
template <int Q>
__global__ void __launch_bounds__(RED_THREADS) k_dots(int n, const double *x0, const double *y0, const double *x1,
                                                      const double *y1, const double *x2, const double *y2,
                                                      double *partials, unsigned int *counter, double *out) {
	__shared__ double sh[32];
	double v[3] = {0.0, 0.0, 0.0};
	// four grid-stride steps a round, their loads issued before the products
	// (which keep the order of the plain loop)
	constexpr int U = 4;
	const int T = gridDim.x * blockDim.x;
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	for (; (long long)i + (U - 1) * T < n; i += U * T) {
		double a[3][U], b[3][U];
#pragma unroll
		for (int u = 0; u < U; u++) {
			a[0][u] = x0[i + u * T];
			b[0][u] = y0[i + u * T];
			if (Q > 1) a[1][u] = x1[i + u * T], b[1][u] = y1[i + u * T];
			if (Q > 2) a[2][u] = x2[i + u * T], b[2][u] = y2[i + u * T];
		}
#pragma unroll
		for (int u = 0; u < U; u++) {
			v[0] = fma(a[0][u], b[0][u], v[0]);
			if (Q > 1) v[1] = fma(a[1][u], b[1][u], v[1]);
			if (Q > 2) v[2] = fma(a[2][u], b[2][u], v[2]);
		}
	}
	for (; i < n; i += T) {
		v[0] = fma(x0[i], y0[i], v[0]);
		if (Q > 1) v[1] = fma(x1[i], y1[i], v[1]);
		if (Q > 2) v[2] = fma(x2[i], y2[i], v[2]);
	}
	finish_reduction<Q>(v, partials, counter, out, sh);
}

// out[j] = V_j . w, j < k (k <= 8), V column-major with leading dim ld.
template <int K>
__global__ void __launch_bounds__(RED_THREADS) k_mdot(int n, const double *V, long long ld, const double *w,
                                                      double *partials, unsigned int *counter, double *out) {
	__shared__ double sh[32];
	double v[K];
#pragma unroll
	for (int j = 0; j < K; j++) v[j] = 0.0;
	// U grid-stride steps a round (more for fewer vectors), all their loads
	// issued before the products, which keep the order of the plain loop
	constexpr int U = K <= 2 ? 4 : 2;
	const int T = gridDim.x * blockDim.x;
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	for (; (long long)i + (U - 1) * T < n; i += U * T) {
		double a[U][K], wu[U];
#pragma unroll
		for (int u = 0; u < U; u++) {
			wu[u] = w[i + u * T];
#pragma unroll
			for (int j = 0; j < K; j++) a[u][j] = V[j * ld + i + u * T];
		}
#pragma unroll
		for (int u = 0; u < U; u++)
#pragma unroll
			for (int j = 0; j < K; j++) v[j] = fma(a[u][j], wu[u], v[j]);
	}
	for (; i < n; i += T) {
		const double wi = w[i];
#pragma unroll
		for (int j = 0; j < K; j++) v[j] = fma(V[j * ld + i], wi, v[j]);
	}
	finish_reduction<K>(v, partials, counter, out, sh);
}

// s + sum_j c_j V_j[i] (c_j = -h_j when SUB), in the order j = 0, 1, ..;
// four vectors' loads are issued before their products
template <bool SUB>
__device__ __forceinline__ double comb(double s, const double *V, long long ld, int k, const double *h, int i) {
	int j = 0;
	for (; j + 4 <= k; j += 4) {
		double a[4];
#pragma unroll
		for (int q = 0; q < 4; q++) a[q] = V[(j + q) * ld + i];
#pragma unroll
		for (int q = 0; q < 4; q++) s = fma(SUB ? -h[j + q] : h[j + q], a[q], s);
	}
	for (; j < k; j++) s = fma(SUB ? -h[j] : h[j], V[j * ld + i], s);
	return s;
}

// w -= V h  (h on the device, k vectors)
__global__ void k_gemv_sub(int n, const double *V, long long ld, int k, const double *h, double *w) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		w[i] = comb<true>(w[i], V, ld, k, h, i);
}

// x += V y (y on device)
__global__ void k_gemv_add(int n, const double *V, long long ld, int k, const double *y, double *x) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		x[i] = comb<false>(x[i], V, ld, k, y, i);
}

// y = x * scale, scale = num / den with num/den on the device (den <= 0 -> 0)
__global__ void k_scale_by(int n, const double *x, double *y, const double *num, const double *den, int sqrt_den) {
	double d = *den;
	if (sqrt_den) d = sqrt(d);
	double f = (d > 0.0) ? ((num ? *num : 1.0) / d) : 0.0;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i] * f;
}

// r = b - r
__global__ void k_residual(int n, const double *b, double *r) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r[i] = b[i] - r[i];
}

// out = max_i |x_i| (CSVector::MaxProdSVect with unit weights,
// Bslib/svector.cpp:376): one partial per block, the last block takes the
// maximum of the partials.  Max is order-independent, so the result is exact.
__global__ void __launch_bounds__(RED_THREADS) k_maxabs(int n, const double *x, double *partials,
                                                        unsigned int *counter, double *out) {
	__shared__ double sh[32];
	__shared__ bool last;
	double v = 0.0;
	{
		const int T = gridDim.x * blockDim.x;
		int i = blockIdx.x * blockDim.x + threadIdx.x;
		for (; (long long)i + 3 * T < n; i += 4 * T) {
			const double a0 = x[i], a1 = x[i + T], a2 = x[i + 2 * T], a3 = x[i + 3 * T];
			v = fmax(fmax(fmax(fmax(v, fabs(a0)), fabs(a1)), fabs(a2)), fabs(a3));
		}
		for (; i < n; i += T) v = fmax(v, fabs(x[i]));
	}
	for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
	if (l == 0) sh[w] = v;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int k = 0; k < (int)(blockDim.x >> 5); k++) t = fmax(t, sh[k]);
		partials[blockIdx.x] = t;
		__threadfence();
		last = (atomicAdd(counter, 1u) == gridDim.x - 1);
	}
	__syncthreads();
	if (!last || threadIdx.x != 0) return;
	__threadfence();
	double t = 0.0;
	for (int b = 0; b < (int)gridDim.x; b++) t = fmax(t, __ldcg(partials + b));
	*out = t;
	*counter = 0;
}

__global__ void k_fill(int n, double *x, double v) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

} // namespace

static inline int ew_grid(long long n) {
	long long b = (n + 255) / 256;
	long long cap = (long long)BSG_SMS * 8;
	return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

int bsg_dots_launch(bsg_ctx *c, int q, int n, const double *x0, const double *y0, const double *x1,
                    const double *y1, const double *x2, const double *y2, double *d_out) {
	BSG_COUNT(1);
	if (q == 1)
		k_dots<1><<<RED_BLOCKS, RED_THREADS, 0, c->stream>>>(n, x0, y0, x1, y1, x2, y2, c->d_partials, c->d_counters, d_out);
	else if (q == 2)
		k_dots<2><<<RED_BLOCKS, RED_THREADS, 0, c->stream>>>(n, x0, y0, x1, y1, x2, y2, c->d_partials, c->d_counters, d_out);
	else
		k_dots<3><<<RED_BLOCKS, RED_THREADS, 0, c->stream>>>(n, x0, y0, x1, y1, x2, y2, c->d_partials, c->d_counters, d_out);
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}

int bsg_dot_launch(bsg_ctx *c, int n, const double *x, const double *y, double *d_out) {
	return bsg_dots_launch(c, 1, n, x, y, nullptr, nullptr, nullptr, nullptr, d_out);
}

// d_out[j] = V_j . w for j < k
int bsg_mdot_launch(bsg_ctx *c, int n, const double *V, long long ld, int k, const double *w, double *d_out) {
	for (int j0 = 0; j0 < k; j0 += 8) {
		BSG_COUNT(1);
		int kk = k - j0 < 8 ? k - j0 : 8;
		const double *Vj = V + j0 * ld;
		double *o = d_out + j0;
		switch (kk) {
#define BSG_MDOT(K) case K: k_mdot<K><<<RED_BLOCKS, RED_THREADS, 0, c->stream>>>(n, Vj, ld, w, c->d_partials, c->d_counters, o); break;
			BSG_MDOT(1) BSG_MDOT(2) BSG_MDOT(3) BSG_MDOT(4) BSG_MDOT(5) BSG_MDOT(6) BSG_MDOT(7) BSG_MDOT(8)
#undef BSG_MDOT
		}
	}
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}

int bsg_gemv_sub_launch(bsg_ctx *c, int n, const double *V, long long ld, int k, const double *h, double *w) {
	BSG_COUNT(1);
	k_gemv_sub<<<ew_grid(n), 256, 0, c->stream>>>(n, V, ld, k, h, w);
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}
int bsg_gemv_add_launch(bsg_ctx *c, int n, const double *V, long long ld, int k, const double *y, double *x) {
	BSG_COUNT(1);
	k_gemv_add<<<ew_grid(n), 256, 0, c->stream>>>(n, V, ld, k, y, x);
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}
int bsg_scale_by_launch(bsg_ctx *c, int n, const double *x, double *y, const double *num, const double *den,
                        int sqrt_den) {
	BSG_COUNT(1);
	k_scale_by<<<ew_grid(n), 256, 0, c->stream>>>(n, x, y, num, den, sqrt_den);
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}
int bsg_residual_launch(bsg_ctx *c, int n, const double *b, double *r) {
	BSG_COUNT(1);
	k_residual<<<ew_grid(n), 256, 0, c->stream>>>(n, b, r);
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}
int bsg_maxabs_launch(bsg_ctx *c, int n, const double *x, double *d_out) {
	BSG_COUNT(1);
	k_maxabs<<<RED_BLOCKS, RED_THREADS, 0, c->stream>>>(n, x, c->d_partials, c->d_counters, d_out);
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}

int bsg_fill_launch(cudaStream_t s, long long n, double *x, double v) {
	BSG_COUNT(1);
	k_fill<<<ew_grid(n), 256, 0, s>>>((int)n, x, v);
	return cudaGetLastError() == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}
