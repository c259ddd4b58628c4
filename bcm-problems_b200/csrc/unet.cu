// Learned preconditioner stage: a 4-level 3D convolutional U-Net applied
// after the ILU2 sweep inside FGMRES, with its own training kernels.  No
// counterpart in the reference (Bslib has no learned or reduced-precision
// part); the network is defined by oracle/unet_ref.py, which the tests hold
// these kernels to.
//
//   x0 = [r/|r|, normalised log diag(A), 0..]                 R0, 16 ch
//   e0 = relu(conv(x0; W0 16->16))          e1 = relu(conv(pool e0; W1 16->32))
//   e2 = relu(conv(pool e1; W2 32->64))     e3 = relu(conv(pool e2; W3 64->64))
//   d2 = relu(conv([up e3, e2]; W4 128->32))
//   d1 = relu(conv([up d2, e1]; W5 64->16))
//   d0 = relu(conv([up d1, e0]; W6 32->16)) y = w7 . d0
//   correction alpha y, alpha = (r . y) / (y . A y) (A-norm optimal step)
//
// Layout: activations channels-last [z][y][x][c] in bfloat16 (32 bytes per
// voxel at 16 channels), weights bfloat16 [tap][cout][cin], accumulation in
// FP32.  The 3x3x3 convolution is an implicit GEMM on the tensor cores
// (mma.sync m16n8k16 bf16 -> f32): M = voxels, N = output channels (16 per
// CTA), K = 27 taps x input channels, with the weight slice of the CTA
// staged in shared memory (rows padded by 8 so the B-fragment reads are
// bank-conflict free) and the A fragments read straight from the
// channels-last tensors (L1 serves the 27-fold tap reuse).  The decoder
// reads its upsampled input at coordinate / 2 instead of materialising it,
// and the concatenation is two input pointers.  The backward pass reuses
// the same kernel for the data gradient (flipped, channel-transposed
// weights, FP32 output); weight gradients are FP32 sums on the CUDA cores.
#include "bsg_internal.cuh"
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <cmath>
#include <cstring>
#include <vector>

typedef __nv_bfloat16 bf16;

int bsg_spmm_launch(const bsg_mat *m, int nrhs, const double *X, double *Y, long long ld, cudaStream_t s);

namespace {

enum { NW = 7 };
const int CIN[NW] = {16, 16, 32, 64, 128, 64, 32};
const int COUT[NW] = {16, 32, 64, 64, 32, 16, 16};

struct ConvArgs {
	int nz, ny, nx;       // output dims (B has these dims; A has them >> upA)
	const bf16 *A;
	int Ca, upA;
	const bf16 *B;
	int Cb;
	const bf16 *W;        // [27][Cout][Cin]
	int Cout;
	void *out;            // bf16 [v][Cout] (relu) or float [v][Cout]
};

__device__ __forceinline__ void mma_bf16(float *c, const unsigned *a, unsigned b0, unsigned b1) {
	asm volatile(
	    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
	    "{%0,%1,%2,%3};"
	    : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
	    : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned ld_u32(const bf16 *p) { return __ldg(reinterpret_cast<const unsigned *>(p)); }

#define CONV_MT 2 // 16-voxel tiles per warp iteration

// One CTA: CONV_MT tiles of 16 consecutive voxels x 16 output channels; its
// four warps take every fourth tap (7, 7, 7, 6 of the 27) of the same tile,
// which shortens each warp's chain of dependent gathers fourfold, and their
// FP32 partial sums meet in shared memory (red[3][CONV_MT * 8][32]).
template <bool F32OUT>
__global__ void __launch_bounds__(128) k_conv3(ConvArgs a) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int Cin = a.Ca + a.Cb;
	const int ldw = Cin + 8;
	float *red = reinterpret_cast<float *>(smem_raw);
	bf16 *Ws = reinterpret_cast<bf16 *>(smem_raw + 3 * CONV_MT * 8 * 32 * sizeof(float));
	const int slice = blockIdx.y; // 16 output channels
	// stage the weight slice, 16 bytes per load: Ws[(tap*16 + n) * ldw + k]
	// (Cin is a multiple of 8, so rows of both layouts start on 16 bytes)
	for (int e = threadIdx.x; e < 27 * 16 * (Cin / 8); e += blockDim.x) {
		const int k8 = e % (Cin / 8), row = e / (Cin / 8);
		const int tap = row / 16, n = row % 16;
		const uint4 v = __ldg(reinterpret_cast<const uint4 *>(a.W + ((size_t)tap * a.Cout + slice * 16 + n) * Cin + 8 * k8));
		*reinterpret_cast<uint4 *>(Ws + (size_t)row * ldw + 8 * k8) = v;
	}
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int g = lane >> 2, t4 = lane & 3;
	const long long nvox = (long long)a.nz * a.ny * a.nx;
	const long long ntile = (nvox + 16 * CONV_MT - 1) / (16 * CONV_MT);
	const int nyA = a.ny >> a.upA, nxA = a.nx >> a.upA;
	for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
		// rows handled by this lane: r = mt*16 + g + 8*h
		int vz[CONV_MT][2], vy[CONV_MT][2], vx[CONV_MT][2];
		bool vin[CONV_MT][2];
#pragma unroll
		for (int mt = 0; mt < CONV_MT; mt++)
#pragma unroll
			for (int h = 0; h < 2; h++) {
				const long long v = tile * 16 * CONV_MT + mt * 16 + g + 8 * h;
				vin[mt][h] = v < nvox;
				const long long vv = vin[mt][h] ? v : 0;
				vx[mt][h] = (int)(vv % a.nx);
				vy[mt][h] = (int)((vv / a.nx) % a.ny);
				vz[mt][h] = (int)(vv / ((long long)a.nx * a.ny));
			}
		float acc[CONV_MT][2][4];
#pragma unroll
		for (int mt = 0; mt < CONV_MT; mt++)
#pragma unroll
			for (int j = 0; j < 2; j++)
#pragma unroll
				for (int q = 0; q < 4; q++) acc[mt][j][q] = 0.f;
		for (int tap = warp; tap < 27; tap += 4) {
			const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
			long long ia[CONV_MT][2], ib[CONV_MT][2];
			bool ok[CONV_MT][2];
#pragma unroll
			for (int mt = 0; mt < CONV_MT; mt++)
#pragma unroll
				for (int h = 0; h < 2; h++) {
					const int z = vz[mt][h] + dz, y = vy[mt][h] + dy, x = vx[mt][h] + dx;
					ok[mt][h] = vin[mt][h] && z >= 0 && z < a.nz && y >= 0 && y < a.ny && x >= 0 && x < a.nx;
					const int za = z >> a.upA, ya = y >> a.upA, xa = x >> a.upA;
					ia[mt][h] = ok[mt][h] ? (((long long)za * nyA + ya) * nxA + xa) * a.Ca : 0;
					ib[mt][h] = ok[mt][h] ? (((long long)z * a.ny + y) * a.nx + x) * a.Cb : 0;
				}
			const bf16 *wt = Ws + (size_t)tap * 16 * ldw;
			for (int cb = 0; cb < Cin; cb += 16) {
				const bool fromA = cb < a.Ca;
				const bf16 *src = fromA ? a.A + cb : a.B + (cb - a.Ca);
				unsigned b[2][2];
#pragma unroll
				for (int j = 0; j < 2; j++) {
					const bf16 *wr = wt + (size_t)(j * 8 + g) * ldw + cb + 2 * t4;
					b[j][0] = *reinterpret_cast<const unsigned *>(wr);
					b[j][1] = *reinterpret_cast<const unsigned *>(wr + 8);
				}
#pragma unroll
				for (int mt = 0; mt < CONV_MT; mt++) {
					unsigned af[4];
					const long long i0 = fromA ? ia[mt][0] : ib[mt][0];
					const long long i1 = fromA ? ia[mt][1] : ib[mt][1];
					af[0] = ok[mt][0] ? ld_u32(src + i0 + 2 * t4) : 0u;
					af[1] = ok[mt][1] ? ld_u32(src + i1 + 2 * t4) : 0u;
					af[2] = ok[mt][0] ? ld_u32(src + i0 + 2 * t4 + 8) : 0u;
					af[3] = ok[mt][1] ? ld_u32(src + i1 + 2 * t4 + 8) : 0u;
#pragma unroll
					for (int j = 0; j < 2; j++) mma_bf16(acc[mt][j], af, b[j][0], b[j][1]);
				}
			}
		}
		// warps 1-3 hand their partial sums to warp 0
		if (warp > 0)
#pragma unroll
			for (int mt = 0; mt < CONV_MT; mt++)
#pragma unroll
				for (int j = 0; j < 2; j++)
#pragma unroll
					for (int q = 0; q < 4; q++) red[((warp - 1) * CONV_MT * 8 + (mt * 2 + j) * 4 + q) * 32 + lane] = acc[mt][j][q];
		__syncthreads();
		if (warp == 0) {
#pragma unroll
			for (int w = 0; w < 3; w++)
#pragma unroll
				for (int mt = 0; mt < CONV_MT; mt++)
#pragma unroll
					for (int j = 0; j < 2; j++)
#pragma unroll
						for (int q = 0; q < 4; q++) acc[mt][j][q] += red[(w * CONV_MT * 8 + (mt * 2 + j) * 4 + q) * 32 + lane];
		}
		__syncthreads(); // red is free for the next tile
		if (warp > 0) continue;
		// epilogue (warp 0): rows g / g+8, columns slice*16 + j*8 + 2*t4 + {0,1}
#pragma unroll
		for (int mt = 0; mt < CONV_MT; mt++)
#pragma unroll
			for (int h = 0; h < 2; h++) {
				if (!vin[mt][h]) continue;
				const long long v = tile * 16 * CONV_MT + mt * 16 + g + 8 * h;
#pragma unroll
				for (int j = 0; j < 2; j++) {
					const int co = slice * 16 + j * 8 + 2 * t4;
					const float c0 = acc[mt][j][2 * h], c1 = acc[mt][j][2 * h + 1];
					if (F32OUT) {
						*reinterpret_cast<float2 *>(static_cast<float *>(a.out) + v * a.Cout + co) = make_float2(c0, c1);
					} else {
						*reinterpret_cast<__nv_bfloat162 *>(static_cast<bf16 *>(a.out) + v * a.Cout + co) =
						    __floats2bfloat162_rn(fmaxf(c0, 0.f), fmaxf(c1, 0.f));
					}
				}
			}
	}
}

// ---- shared-memory tiled convolution (grids with nx % 32 == 0) ------------
// A CTA (8 warps) computes a 32 x 4 x 2 brick of output voxels for 16 output
// channels.  Input channels go in chunks of CH (16 or 32): the CTA stages the
// 34 x 6 x 4 halo brick of the chunk and the chunk's weights for all 27 taps
// in shared memory, then every warp (one 32-voxel x-row) runs the 27 taps
// with ldmatrix A / B fragments and mma.sync.  The halo rows are stored with
// their 16-byte pieces XOR-swizzled by the voxel index, so the 8 row
// addresses of an ldmatrix (8 consecutive voxels) hit 8 distinct bank
// groups; weight rows are padded by 8 elements for the same reason.
#define TT_X 32
#define TT_Y 4
#define TT_Z 2
#define TH_X (TT_X + 2)
#define TH_Y (TT_Y + 2)
#define TH_Z (TT_Z + 2)
#define TH_VOX (TH_X * TH_Y * TH_Z)

template <int CH>
__device__ __forceinline__ unsigned halo_off(int hv, int piece) {
	const int swz = CH == 32 ? ((hv >> 1) & 3) : ((hv >> 2) & 1);
	return (unsigned)(hv * CH * 2 + 16 * (piece ^ swz));
}

__device__ __forceinline__ void ldsm_x4(unsigned addr, unsigned &r0, unsigned &r1, unsigned &r2, unsigned &r3) {
	asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
	             : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
	             : "r"(addr));
}

template <bool F32OUT, int CH>
__global__ void __launch_bounds__(256) k_conv3t(ConvArgs a) {
	extern __shared__ __align__(128) unsigned char smem_t[];
	unsigned char *sIn = smem_t;                                   // TH_VOX * CH bf16
	bf16 *sW = reinterpret_cast<bf16 *>(smem_t + TH_VOX * CH * 2); // [27][16][CH + 8]
	const int ldw = CH + 8;
	const int Cin = a.Ca + a.Cb;
	const int slice = blockIdx.y;
	const int tx = a.nx / TT_X, ty = a.ny / TT_Y;
	const int bx = blockIdx.x % tx, by = (blockIdx.x / tx) % ty, bz = blockIdx.x / (tx * ty);
	const int x0 = bx * TT_X, y0 = by * TT_Y, z0 = bz * TT_Z;
	const int nyA = a.ny >> a.upA, nxA = a.nx >> a.upA;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int wy = warp & 3, wz = warp >> 2;
	const int g = lane >> 2, t4 = lane & 3;
	const unsigned sIn_s = (unsigned)__cvta_generic_to_shared(sIn);
	const unsigned sW_s = (unsigned)__cvta_generic_to_shared(sW);
	float acc[2][2][4];
#pragma unroll
	for (int mt = 0; mt < 2; mt++)
#pragma unroll
		for (int j = 0; j < 2; j++)
#pragma unroll
			for (int q = 0; q < 4; q++) acc[mt][j][q] = 0.f;
	for (int c0 = 0; c0 < Cin; c0 += CH) {
		__syncthreads(); // the previous chunk's reads are done
		// halo brick: TH_VOX voxels x CH/8 pieces of 16 bytes
		for (int e = threadIdx.x; e < TH_VOX * (CH / 8); e += blockDim.x) {
			const int piece = e % (CH / 8), hv = e / (CH / 8);
			const int hx = hv % TH_X, hy = (hv / TH_X) % TH_Y, hz = hv / (TH_X * TH_Y);
			const int X = x0 - 1 + hx, Y = y0 - 1 + hy, Z = z0 - 1 + hz;
			uint4 val = make_uint4(0u, 0u, 0u, 0u);
			if (X >= 0 && X < a.nx && Y >= 0 && Y < a.ny && Z >= 0 && Z < a.nz) {
				const int c = c0 + piece * 8;
				const bf16 *src;
				if (c < a.Ca)
					src = a.A + (((long long)(Z >> a.upA) * nyA + (Y >> a.upA)) * nxA + (X >> a.upA)) * a.Ca + c;
				else
					src = a.B + (((long long)Z * a.ny + Y) * a.nx + X) * a.Cb + (c - a.Ca);
				val = __ldg(reinterpret_cast<const uint4 *>(src));
			}
			*reinterpret_cast<uint4 *>(sIn + halo_off<CH>(hv, piece)) = val;
		}
		// weights of the chunk: sW[(tap*16 + n) * ldw + k] = W[tap][slice*16 + n][c0 + k]
		for (int e = threadIdx.x; e < 27 * 16 * (CH / 8); e += blockDim.x) {
			const int piece = e % (CH / 8), row = e / (CH / 8);
			const int tap = row / 16, n = row % 16;
			const uint4 val =
			    __ldg(reinterpret_cast<const uint4 *>(a.W + ((size_t)tap * a.Cout + slice * 16 + n) * Cin + c0 + piece * 8));
			*reinterpret_cast<uint4 *>(sW + (size_t)row * ldw + piece * 8) = val;
		}
		__syncthreads();
		// lane roles in ldmatrix.x4: matrix q = lane / 8, row r = lane % 8
		const int q = lane >> 3, r = lane & 7;
		for (int tap = 0; tap < 27; tap++) {
			const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3; // halo offsets (0..2)
			const int hrow = ((wz + dz) * TH_Y + (wy + dy)) * TH_X + dx;
#pragma unroll
			for (int kc = 0; kc < CH / 16; kc++) {
				unsigned b0, b1, b2, b3;
				{
					const int n = r + 8 * (q >> 1), k = kc * 16 + 8 * (q & 1);
					ldsm_x4(sW_s + (unsigned)(((tap * 16 + n) * ldw + k) * 2), b0, b1, b2, b3);
				}
#pragma unroll
				for (int mt = 0; mt < 2; mt++) {
					const int hv = hrow + mt * 16 + r + 8 * (q & 1);
					unsigned af[4];
					ldsm_x4(sIn_s + halo_off<CH>(hv, kc * 2 + (q >> 1)), af[0], af[1], af[2], af[3]);
					mma_bf16(acc[mt][0], af, b0, b1);
					mma_bf16(acc[mt][1], af, b2, b3);
				}
			}
		}
	}
	// epilogue: rows g / g+8 of m-tile mt are x = 16 mt + g (+8)
	const long long vrow = ((long long)(z0 + wz) * a.ny + (y0 + wy)) * a.nx + x0;
#pragma unroll
	for (int mt = 0; mt < 2; mt++)
#pragma unroll
		for (int h = 0; h < 2; h++) {
			const long long v = vrow + mt * 16 + g + 8 * h;
#pragma unroll
			for (int j = 0; j < 2; j++) {
				const int co = slice * 16 + j * 8 + 2 * t4;
				const float c0v = acc[mt][j][2 * h], c1v = acc[mt][j][2 * h + 1];
				if (F32OUT)
					*reinterpret_cast<float2 *>(static_cast<float *>(a.out) + v * a.Cout + co) = make_float2(c0v, c1v);
				else
					*reinterpret_cast<__nv_bfloat162 *>(static_cast<bf16 *>(a.out) + v * a.Cout + co) =
					    __floats2bfloat162_rn(fmaxf(c0v, 0.f), fmaxf(c1v, 0.f));
			}
		}
}

// 2x2x2 mean, bf16 in / out (dims of the input).
// A thread takes 8 channels of one output voxel (16-byte loads and store; C
// is a multiple of 8); each channel sums its 8 inputs in the order k = 0..7.
__global__ void k_pool(int nz, int ny, int nx, int C, const bf16 *in, bf16 *out) {
	const int oz = nz / 2, oy = ny / 2, ox = nx / 2, G = C / 8;
	const long long n = (long long)oz * oy * ox * G;
	for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
		const int c0 = 8 * (int)(e % G);
		const long long v = e / G;
		const int x = (int)(v % ox), y = (int)((v / ox) % oy), z = (int)(v / ((long long)ox * oy));
		uint4 q[8];
#pragma unroll
		for (int k = 0; k < 8; k++) {
			const long long u = ((long long)(2 * z + (k >> 2)) * ny + 2 * y + ((k >> 1) & 1)) * nx + 2 * x + (k & 1);
			q[k] = __ldg(reinterpret_cast<const uint4 *>(in + u * C + c0));
		}
		float s[8];
#pragma unroll
		for (int c = 0; c < 8; c++) s[c] = 0.f;
#pragma unroll
		for (int k = 0; k < 8; k++) {
			const bf16 *h = reinterpret_cast<const bf16 *>(&q[k]);
#pragma unroll
			for (int c = 0; c < 8; c++) s[c] += __bfloat162float(h[c]);
		}
		__align__(16) bf16 o[8];
#pragma unroll
		for (int c = 0; c < 8; c++) o[c] = __float2bfloat16_rn(s[c] * 0.125f);
		*reinterpret_cast<uint4 *>(out + v * C + c0) = *reinterpret_cast<const uint4 *>(o);
	}
}

// x0 from r (scaled by 1/|r|, |r|^2 in *nrm2) and the log-diagonal channel.
__global__ void k_input(long long n, const double *r, const double *nrm2, const bf16 *logd, bf16 *x0) {
	const double s2 = *nrm2;
	const double inv = s2 > 0.0 ? 1.0 / sqrt(s2) : 0.0;
	for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
		__align__(16) bf16 h[16];
#pragma unroll
		for (int c = 0; c < 16; c++) h[c] = __float2bfloat16_rn(0.f);
		h[0] = __float2bfloat16_rn((float)(r[v] * inv));
		h[1] = logd[v];
		uint4 *dst = reinterpret_cast<uint4 *>(x0 + v * 16);
		dst[0] = reinterpret_cast<const uint4 *>(h)[0];
		dst[1] = reinterpret_cast<const uint4 *>(h)[1];
	}
}

// y = w7 . d0 per voxel (FP32).
__global__ void k_head(long long n, const bf16 *d0, const float *w7, float *y) {
	for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
		const uint4 *p = reinterpret_cast<const uint4 *>(d0 + v * 16);
		const uint4 q[2] = {__ldg(p), __ldg(p + 1)};
		const bf16 *h = reinterpret_cast<const bf16 *>(q);
		float s = 0.f;
#pragma unroll
		for (int c = 0; c < 16; c++) s = fmaf(w7[c], __bfloat162float(h[c]), s);
		y[v] = s;
	}
}

// y as FP64
__global__ void k_widen(long long n, const float *y, double *yd) {
	for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
		yd[v] = (double)y[v];
}
// z += alpha y with alpha = (r . y) / (y . A y) = s[0] / s[1], the step that
// minimises the A-norm of the remaining error; a step that is not finite
// and positive (a non-finite or useless network output) leaves z as the
// plain ILU2 step.
__global__ void k_correct(long long n, const double *yd, const double *s, double *z) {
	const double alpha = s[0] / s[1];
	if (!(alpha > 0.0) || !isfinite(alpha)) return;
	for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
		z[v] = fma(alpha, yd[v], z[v]);
}

// Deterministic sums of NQ products over a fixed grid: block partials, then
// one ordered final pass.  Q = 2: r . yd, yd . ay.  Q = 3 (training): y . t,
// y . y, t . t.
#define RED_BLOCKS 256
__global__ void k_red2(long long n, const double *r, const double *yd, const double *ay, double *part) {
	__shared__ double sh[2][8];
	double a = 0, b = 0;
	// four grid-stride steps a round, loads first, products in loop order
	const long long T = (long long)gridDim.x * blockDim.x;
	long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	for (; v + 3 * T < n; v += 4 * T) {
		double rr[4], yy[4], aa[4];
#pragma unroll
		for (int u = 0; u < 4; u++) rr[u] = r[v + u * T], yy[u] = yd[v + u * T], aa[u] = ay[v + u * T];
#pragma unroll
		for (int u = 0; u < 4; u++) {
			a = fma(rr[u], yy[u], a);
			b = fma(yy[u], aa[u], b);
		}
	}
	for (; v < n; v += T) {
		a = fma(r[v], yd[v], a);
		b = fma(yd[v], ay[v], b);
	}
	a = warp_sum(a);
	b = warp_sum(b);
	if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = a; sh[1][threadIdx.x >> 5] = b; }
	__syncthreads();
	if (threadIdx.x < 2) {
		double q = 0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) q += sh[threadIdx.x][w];
		part[threadIdx.x * RED_BLOCKS + blockIdx.x] = q;
	}
}
__global__ void k_red3(long long n, const float *y, const double *t, double *part) {
	__shared__ double sh[3][8];
	double a = 0, b = 0, c = 0;
	for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
		const double yv = (double)y[v];
		a = fma(yv, t[v], a);
		b = fma(yv, yv, b);
		c = fma(t[v], t[v], c);
	}
	a = warp_sum(a);
	b = warp_sum(b);
	c = warp_sum(c);
	if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = a; sh[1][threadIdx.x >> 5] = b; sh[2][threadIdx.x >> 5] = c; }
	__syncthreads();
	if (threadIdx.x < 3) {
		double q = 0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) q += sh[threadIdx.x][w];
		part[threadIdx.x * RED_BLOCKS + blockIdx.x] = q;
	}
}
__global__ void k_red_final(int nq, const double *part, double *out) {
	if (threadIdx.x < nq) {
		double q = 0;
		for (int b = 0; b < RED_BLOCKS; b++) q += part[threadIdx.x * RED_BLOCKS + b];
		out[threadIdx.x] = q;
	}
}

// r1 = v - t
__global__ void k_sub(long long n, const double *v, const double *t, double *r) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		r[i] = v[i] - t[i];
}

// sum of squares into *out (deterministic: fixed grid, block partials, one
// final block)
#define SQ_BLOCKS 256
__global__ void k_sumsq_part(long long n, const double *x, double *part) {
	__shared__ double sh[8];
	double s = 0;
	// four grid-stride steps a round, loads first, products in loop order
	const long long T = (long long)gridDim.x * blockDim.x;
	long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	for (; i + 3 * T < n; i += 4 * T) {
		double xx[4];
#pragma unroll
		for (int u = 0; u < 4; u++) xx[u] = x[i + u * T];
#pragma unroll
		for (int u = 0; u < 4; u++) s = fma(xx[u], xx[u], s);
	}
	for (; i < n; i += T) s = fma(x[i], x[i], s);
	s = warp_sum(s);
	if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
		part[blockIdx.x] = t;
	}
}
__global__ void k_sum_final(int nb, const double *part, double *out) {
	if (threadIdx.x == 0) {
		double t = 0;
		for (int b = 0; b < nb; b++) t += part[b];
		*out = t;
	}
}

// log |a_ii| (diagonal first in each row of the upper split), then its
// mean and standard deviation, then the bf16 normalised channel.
__global__ void k_logdiag(int n, const int *iu, const double *al, double *ld) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		ld[i] = log(fabs(al[iu[i]]) + 1e-300);
}
__global__ void k_logvec(int n, const double *d, double *ld) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		ld[i] = log(fabs(d[i]) + 1e-300);
}
// mean and standard deviation of ld: block partials over a fixed grid
// (SQ_BLOCKS), then one ordered final pass
__global__ void k_moments_part(int n, const double *ld, double *part) {
	__shared__ double s1[8], s2[8];
	double a = 0, b = 0;
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		a += ld[i];
		b = fma(ld[i], ld[i], b);
	}
	a = warp_sum(a);
	b = warp_sum(b);
	if ((threadIdx.x & 31) == 0) { s1[threadIdx.x >> 5] = a; s2[threadIdx.x >> 5] = b; }
	__syncthreads();
	if (threadIdx.x == 0) {
		double p = 0, q = 0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) { p += s1[w]; q += s2[w]; }
		part[blockIdx.x] = p;
		part[gridDim.x + blockIdx.x] = q;
	}
}
__global__ void k_moments_final(int n, int nb, const double *part, double *out) {
	if (threadIdx.x == 0) {
		double m = 0, q = 0;
		for (int b = 0; b < nb; b++) { m += part[b]; q += part[nb + b]; }
		m /= n;
		q = q / n - m * m;
		out[0] = m;
		out[1] = q > 1e-30 ? sqrt(q) : 1.0;
	}
}
__global__ void k_logd_norm(int n, const double *ld, const double *mom, bf16 *out) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		out[i] = __float2bfloat16_rn((float)((ld[i] - mom[0]) / mom[1]));
}

// ---- training --------------------------------------------------------------

// Loss 1 - cos^2(y, t) (only the direction of y is trained; the step length
// is chosen when the stage is applied) and its gradient in y; s = {y.t, y.y,
// t.t}, the loss goes to s[3].
__global__ void k_cos_grad(long long n, const float *y, const double *t, double *s, float *gy) {
	const double a = s[0], b = s[1], c = s[2];
	const bool ok = b > 0.0 && c > 0.0;
	const double ct = ok ? -2.0 * a / (b * c) : 0.0, cy = ok ? 2.0 * a * a / (b * b * c) : 0.0;
	if (blockIdx.x == 0 && threadIdx.x == 0) s[3] = ok ? 1.0 - a * a / (b * c) : 1.0;
	for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
		gy[v] = (float)(ct * t[v] + cy * (double)y[v]);
}

// dd0 = w7 * gy masked by d0 > 0 (bf16); dw7[c] += sum_v d0[v][c] gy[v]
__global__ void k_head_bwd(long long n, const bf16 *d0, const float *w7, const float *gy, bf16 *dd0, float *dw7) {
	__shared__ float sh[16][33];
	float acc[16];
#pragma unroll
	for (int c = 0; c < 16; c++) acc[c] = 0.f;
	for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
		const float gv = gy[v];
#pragma unroll
		for (int c = 0; c < 16; c++) {
			const float a = __bfloat162float(d0[v * 16 + c]);
			acc[c] = fmaf(a, gv, acc[c]);
			dd0[v * 16 + c] = __float2bfloat16_rn(a > 0.f ? w7[c] * gv : 0.f);
		}
	}
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int c = 0; c < 16; c++) {
		float s = acc[c];
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) sh[c][warp] = s;
	}
	__syncthreads();
	if (threadIdx.x < 16) {
		float s = 0.f;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[threadIdx.x][w];
		atomicAdd(dw7 + threadIdx.x, s);
	}
}

// Gradient of an activation act [v][C] (this level's dims), bf16 out:
//   up_t mode (fine != null): sum over the 8 children of fine[child*fs + fo + c]
//   skip mode: skip[v*ss + so + c] + coarse[parent*C + c] / 8 (coarse may be null)
// times (act > 0).
__global__ void k_grad_act(int nz, int ny, int nx, int C, const float *fine, int fs, int fo, const float *skip, int ss,
                           int so, const float *coarse, const bf16 *act, bf16 *out) {
	const long long n = (long long)nz * ny * nx * C;
	for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
		const int c = (int)(e % C);
		const long long v = e / C;
		const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((long long)nx * ny));
		float s = 0.f;
		if (fine) {
			const int fy = 2 * ny, fx = 2 * nx;
#pragma unroll
			for (int k = 0; k < 8; k++) {
				const long long u = ((long long)(2 * z + (k >> 2)) * fy + 2 * y + ((k >> 1) & 1)) * fx + 2 * x + (k & 1);
				s += fine[u * fs + fo + c];
			}
		} else {
			s = skip[v * ss + so + c];
			if (coarse) {
				const long long p = ((long long)(z >> 1) * (ny >> 1) + (y >> 1)) * (nx >> 1) + (x >> 1);
				s += coarse[p * C + c] * 0.125f;
			}
		}
		out[e] = __float2bfloat16_rn(__bfloat162float(act[e]) > 0.f ? s : 0.f);
	}
}

// dW[tap][co][ci] += sum_v g[v][co] in(v + off(tap))[ci], CUDA cores, FP32.
// Each thread owns (tap, 4 output, 4 input channels) combinations over one
// voxel chunk of the block.
__global__ void __launch_bounds__(256) k_wgrad(ConvArgs a, const bf16 *gr, long long chunk, float *dW) {
	const int Cin = a.Ca + a.Cb, Cout = a.Cout;
	const long long nvox = (long long)a.nz * a.ny * a.nx;
	const long long v0 = blockIdx.x * chunk;
	const long long v1 = v0 + chunk < nvox ? v0 + chunk : nvox;
	const int nci4 = Cin / 4, nco4 = Cout / 4;
	const int ncombo = 27 * nco4 * nci4;
	const int nyA = a.ny >> a.upA, nxA = a.nx >> a.upA;
	for (int e = threadIdx.x; e < ncombo; e += blockDim.x) {
		const int ci4 = e % nci4, co4 = (e / nci4) % nco4, tap = e / (nci4 * nco4);
		const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
		const int ci = ci4 * 4;
		const bool fromA = ci < a.Ca;
		float acc[4][4];
#pragma unroll
		for (int p = 0; p < 4; p++)
#pragma unroll
			for (int q = 0; q < 4; q++) acc[p][q] = 0.f;
		int x = (int)(v0 % a.nx), y = (int)((v0 / a.nx) % a.ny), z = (int)(v0 / ((long long)a.nx * a.ny));
		for (long long v = v0; v < v1; v++) {
			const int zz = z + dz, yy = y + dy, xx = x + dx;
			if (zz >= 0 && zz < a.nz && yy >= 0 && yy < a.ny && xx >= 0 && xx < a.nx) {
				const bf16 *ip;
				if (fromA)
					ip = a.A + (((long long)(zz >> a.upA) * nyA + (yy >> a.upA)) * nxA + (xx >> a.upA)) * a.Ca + ci;
				else
					ip = a.B + (((long long)zz * a.ny + yy) * a.nx + xx) * a.Cb + (ci - a.Ca);
				const uint2 iv = __ldg(reinterpret_cast<const uint2 *>(ip));
				const uint2 gv = __ldg(reinterpret_cast<const uint2 *>(gr + v * Cout + co4 * 4));
				const __nv_bfloat162 i01 = *reinterpret_cast<const __nv_bfloat162 *>(&iv.x);
				const __nv_bfloat162 i23 = *reinterpret_cast<const __nv_bfloat162 *>(&iv.y);
				const __nv_bfloat162 g01 = *reinterpret_cast<const __nv_bfloat162 *>(&gv.x);
				const __nv_bfloat162 g23 = *reinterpret_cast<const __nv_bfloat162 *>(&gv.y);
				const float in4[4] = {__low2float(i01), __high2float(i01), __low2float(i23), __high2float(i23)};
				const float g4[4] = {__low2float(g01), __high2float(g01), __low2float(g23), __high2float(g23)};
#pragma unroll
				for (int p = 0; p < 4; p++)
#pragma unroll
					for (int q = 0; q < 4; q++) acc[p][q] = fmaf(g4[p], in4[q], acc[p][q]);
			}
			if (++x == a.nx) { x = 0; if (++y == a.ny) { y = 0; ++z; } }
		}
#pragma unroll
		for (int p = 0; p < 4; p++)
#pragma unroll
			for (int q = 0; q < 4; q++)
				if (acc[p][q] != 0.f) atomicAdd(dW + ((size_t)tap * Cout + co4 * 4 + p) * Cin + ci + q, acc[p][q]);
	}
}

// Adam on the FP32 master weights; grads are averaged over `count` samples
// and cleared.  W0's padded input channels (ci >= 2) stay zero.
__global__ void k_adam(int n, float *w, float *m, float *v, float *gr, float inv_count, float lr, float b1, float b2,
                       float eps, float c1, float c2, int w0_len) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		float gi = gr[i] * inv_count;
		gr[i] = 0.f;
		if (i < w0_len && (i % 16) >= 2) { w[i] = 0.f; continue; }
		m[i] = b1 * m[i] + (1.f - b1) * gi;
		v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
		const float mh = m[i] / c1, vh = v[i] / c2;
		w[i] -= lr * mh / (sqrtf(vh) + eps);
	}
}

// bf16 copies of the master weights: W [tap][co][ci] and the data-gradient
// form WT [tap][ci][co] = W[26 - tap][co][ci].
__global__ void k_refresh(int len, int cout, int cin, const float *w, bf16 *wb, bf16 *wt) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) {
		const int ci = i % cin, co = (i / cin) % cout, tap = i / (cin * cout);
		const bf16 b = __float2bfloat16_rn(w[i]);
		wb[i] = b;
		wt[((size_t)(26 - tap) * cin + ci) * cout + co] = b;
	}
}
__global__ void k_w7(const float *w, float *w7b) {
	if (threadIdx.x < 16) w7b[threadIdx.x] = __bfloat162float(__float2bfloat16_rn(w[threadIdx.x]));
}

inline int ew(long long n) {
	long long b = (n + 255) / 256;
	return (int)(b < BSG_SMS * 16 ? (b > 0 ? b : 1) : BSG_SMS * 16);
}

// ---- 5th-generation tensor cores (tcgen05) for the level-0 convolutions ----
// Level 0 of the network has 16 output channels and x-lines of 128 voxels.
// For a staged input line (y', z') of 128 voxels the tensor cores compute,
// one MMA per z tap dz and 16-channel K chunk,
//     D[x'][(dy, dx, n)] = sum_cin in[x'][y'][z'][cin] W[dz][dy][dx][n][cin],
// M = 128 voxels, N = 3 x 3 x 16 = 144 (an N = 16 MMA costs as many cycles
// as an N = 48 one; N = 144 runs the tensor cores at full rate).  Line y'
// feeds output rows y' + 1 (dy = 0), y' (dy = 1) and y' - 1 (dy = 2), so
// each output row owns a 48-column accumulator block T[x'][(dx, n)] in
// tensor memory and the blocks of consecutive rows are laid out at
// descending column offsets: the three blocks a line feeds are contiguous,
// and one MMA adds into all of them (two when the ring of 10 blocks wraps).
// The epilogue forms out[x] = T0[x - 1] + T1[x] + T2[x + 1] with warp
// shuffles (the grid's x boundary is the tile's: nx = 128 only).
//
// Warp roles (288 threads, two CTAs per SM):
//   warps 0-3  epilogue: TMEM lanes 32w .. 32w + 31; read a finished row's
//              block, zero it for its next use, shift-add, ReLU, store;
//   warps 4-7  producers: stage the three z lines of each input line y' into
//              a ring of slots.  A 16-channel input at full resolution is one
//              TMA box per z line (4 KB; planes outside the grid read as
//              zeros); an upsampled one is gathered with cp.async;
//   warp 8     one thread issues the MMAs and commits them to mbarriers.
// Each 16-channel part of a staged z line is a 128 x 32-byte K-major tile in
// the 32-byte swizzle (16-byte halves of row r exchanged when bit 2 of r is
// set), the layout TMA writes and the tensor cores read with SWIZZLE_32B
// descriptors.  The weights are K-major without swizzle: core matrices of
// 8 rows x 16 bytes, rows 16 bytes apart, 8-channel chunks LBO bytes apart.  Every wait is an mbarrier wait bounded
// by BSG_SPIN_LIMIT_NS; one that expires raises BSG_ERR_TIMEOUT and makes
// all roles leave their loops.
namespace tc {
constexpr int NB = 5;     // 48-column accumulator blocks in the TMEM ring (256 columns allocated)
constexpr int CTAS = 2;   // CTAs per SM: two pipelines share the tensor cores
constexpr int THREADS = 288;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address, leading (K-chunk) and
// stride (8-row group) byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ unsigned long long sdesc(unsigned addr, unsigned lbo, unsigned sbo) {
	return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
	       ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// descriptor of a 128-row K-major tile of 32-byte rows in the 32-byte swizzle
// (SBO = 8 rows x 32 bytes; the leading offset is unused)
__device__ __forceinline__ unsigned long long sdesc_sw32(unsigned addr) {
	return (unsigned long long)((addr >> 4) & 0x3FFFu) | (1ull << 16) | ((unsigned long long)(256 >> 4) << 32) |
	       (1ull << 46) | (6ull << 61);
}

// instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major, M = 128
__device__ __forceinline__ unsigned idesc(int n) {
	return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma(unsigned tmem, unsigned long long ad, unsigned long long bd, unsigned id) {
	asm volatile("{\n\t.reg .pred p;\n\tsetp.eq.u32 p, 1, 1;\n\t"
	             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
	             "l"(ad), "l"(bd), "r"(id));
}
__device__ __forceinline__ void commit(unsigned mb) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb) : "memory");
}
__device__ __forceinline__ void arrive(unsigned mb) {
	asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(mb) : "memory");
}
__device__ __forceinline__ void arrive_tx(unsigned mb, unsigned bytes) {
	asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(mb), "r"(bytes)
	             : "memory");
}
// TMA: the 128-voxel x 16-channel box at voxel v0 of a 2D [voxel][16] map
__device__ __forceinline__ void tma_line(unsigned dst, const CUtensorMap *map, int v0, unsigned mb) {
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
	             "l"(reinterpret_cast<unsigned long long>(map)), "r"(0), "r"(v0), "r"(mb)
	             : "memory");
}
__device__ __forceinline__ void mbar_init(unsigned mb, int count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mb), "r"(count));
}

// bounded wait on the mbarrier phase `parity`: 1 when it completed, 0 when
// *abort was raised (here on expiry, or by another role).  The timer is read
// only once the phase has not completed after 64 polls.
__device__ __forceinline__ int mbar_wait(unsigned mb, unsigned parity, volatile int *abort) {
	unsigned long long t0 = 0;
	for (unsigned it = 0;; it++) {
		unsigned done;
		asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}\n"
		             : "=r"(done)
		             : "r"(mb), "r"(parity)
		             : "memory");
		if (done) return 1;
		if ((it & 63) == 63) {
			if (*abort) return 0;
			const unsigned long long now = globaltimer_ns();
			if (t0 == 0)
				t0 = now;
			else if (now - t0 > BSG_SPIN_LIMIT_NS) {
				*abort = 1;
				return 0;
			}
		}
	}
}
// TMEM column of the accumulator block of the q-th output row of a CTA
__device__ __forceinline__ unsigned blk_col(long long q) { return 48u * (unsigned)(NB - 1 - (int)(q % NB)); }

// shared-memory plan of k_conv3_tc<CIN>
template <int CIN>
struct Plan {
	static constexpr int NCH = CIN / 8;                 // 16-byte chunks of a voxel
	static constexpr int NK = CIN / 16;                 // 16-channel parts (K steps)
	static constexpr int WDZ = NCH * 144 * 16;          // weights of one z tap: [chunk][(dy,dx,n)][8]
	static constexpr int TILE = 128 * 32;               // one part of one z line (swizzled)
	static constexpr int SLOT = 3 * NK * TILE;          // an input line: [dz][part] tiles
	static constexpr int NSLOT = CIN == 16 ? 6 : 3;     // ring depth (two CTAs per SM either way)
	static constexpr int XCH = 2 * 4 * 2 * 16 * 4;      // warp-edge exchange: [row parity][warp][side][16] floats
	// slots first (1024-byte aligned for the swizzle), then weights, exchange
	static constexpr size_t BYTES = 1024 + (size_t)NSLOT * SLOT + (size_t)3 * WDZ + XCH;
};
} // namespace tc

// tmA / tmB: [voxel][16] maps of the A part (when not upsampled) and the B part
template <int CIN>
__global__ void __launch_bounds__(tc::THREADS, tc::CTAS)
    k_conv3_tc(ConvArgs a, const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               bsg_devstat *st) {
	using PL = tc::Plan<CIN>;
	constexpr int NCH = PL::NCH, NK = PL::NK, NSLOT = PL::NSLOT, NB = tc::NB;
	extern __shared__ __align__(128) unsigned char sm_raw[];
	unsigned char *sl = sm_raw + ((1024u - (tc::smem_u32(sm_raw) & 1023u)) & 1023u);
	unsigned char *sw = sl + (size_t)NSLOT * PL::SLOT;
	float *xch = reinterpret_cast<float *>(sw + 3 * PL::WDZ);
	const bool up = a.upA != 0; // A part gathered with cp.async (else TMA, like B)
	__shared__ __align__(8) unsigned long long bar[2 * NSLOT + 2 * NB + 3];
	__shared__ unsigned tmem_base;
	__shared__ volatile int abort_;
	const unsigned b_full = tc::smem_u32(&bar[0]), b_free = b_full + 8 * NSLOT; // slots
	const unsigned k_full = b_free + 8 * NSLOT, k_free = k_full + 8 * NB;        // accumulator blocks
	const unsigned x_bar = k_free + 8 * NB, f_bar = x_bar + 16;                  // edge exchange, drain
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int ny = a.ny, nz = a.nz;
	// this CTA's share of the level's nz * ny output rows: one contiguous range,
	// walked as one segment [ya, yb) per z plane it touches
	const long long nrow = (long long)nz * ny;
	const long long r0 = nrow * blockIdx.x / gridDim.x, r1 = nrow * (blockIdx.x + 1) / gridDim.x;
	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(tc::smem_u32(&tmem_base)));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
	}
	if (tid == 0) {
		for (int i = 0; i < NSLOT; i++) {
			tc::mbar_init(b_full + 8 * i, 1 + (up ? 128 : 0)); // TMA issuer (+ gatherers)
			tc::mbar_init(b_free + 8 * i, 1);
		}
		for (int i = 0; i < NB; i++) {
			tc::mbar_init(k_full + 8 * i, 1);
			tc::mbar_init(k_free + 8 * i, 128);
		}
		tc::mbar_init(x_bar, 8); // lanes 0 and 31 of the four epilogue warps
		tc::mbar_init(x_bar + 8, 8);
		tc::mbar_init(f_bar, 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		abort_ = 0;
	}
	// weights: sw[dz][chunk][(dy, dx, n)][8] = W[(dz, dy, dx)][n][chunk * 8 ..]
	for (int e = tid; e < 27 * 16 * NCH; e += tc::THREADS) {
		const int ch = e % NCH, r = e / NCH, n = r % 16, tap = r / 16, dz = tap / 9, t9 = tap % 9;
		const uint4 v = __ldg(reinterpret_cast<const uint4 *>(a.W + ((size_t)tap * 16 + n) * CIN + ch * 8));
		*reinterpret_cast<uint4 *>(sw + dz * PL::WDZ + ch * (144 * 16) + (t9 * 16 + n) * 16) = v;
	}
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	const unsigned tmem = tmem_base;

	if (warp < 4) {
		// ---- epilogue ----
		const unsigned lanes = (unsigned)(32 * warp) << 16;
		unsigned zero[16];
#pragma unroll
		for (int i = 0; i < 16; i++) zero[i] = 0u;
		// accumulators start at zero (every MMA accumulates)
		for (int c = 0; c < NB * 48; c += 16)
			asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
			                 tmem + lanes + c),
			             "r"(zero[0]), "r"(zero[1]), "r"(zero[2]), "r"(zero[3]), "r"(zero[4]), "r"(zero[5]), "r"(zero[6]),
			             "r"(zero[7]), "r"(zero[8]), "r"(zero[9]), "r"(zero[10]), "r"(zero[11]), "r"(zero[12]), "r"(zero[13]),
			             "r"(zero[14]), "r"(zero[15]));
		asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
		asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
		for (int i = 0; i < NB; i++) tc::arrive(k_free + 8 * i); // use 0 of every block: free
		long long q = 0;
		bool quit = false; // warp-uniform
		for (long long rs = r0, re; rs < r1 && !quit; rs = re) {
			const int z = (int)(rs / ny), ya = (int)(rs % ny);
			re = min(r1, (long long)(z + 1) * ny);
			const int yb = (int)(re - (long long)z * ny);
			for (int r = ya; r < yb; r++, q++) {
				const int b = (int)(q % NB);
				const bool ok = tc::mbar_wait(k_full + 8 * b, (unsigned)((q / NB) & 1), &abort_);
				if (!__all_sync(0xffffffffu, ok)) {
					quit = true;
					break;
				}
				asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
				const unsigned col = tmem + lanes + tc::blk_col(q);
				float t[3][16];
#pragma unroll
				for (int dx = 0; dx < 3; dx++) {
					unsigned rr[16];
					asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
					             : "=r"(rr[0]), "=r"(rr[1]), "=r"(rr[2]), "=r"(rr[3]), "=r"(rr[4]), "=r"(rr[5]), "=r"(rr[6]),
					               "=r"(rr[7]), "=r"(rr[8]), "=r"(rr[9]), "=r"(rr[10]), "=r"(rr[11]), "=r"(rr[12]), "=r"(rr[13]),
					               "=r"(rr[14]), "=r"(rr[15])
					             : "r"(col + 16 * dx));
					asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
					for (int i = 0; i < 16; i++) t[dx][i] = __uint_as_float(rr[i]);
				}
#pragma unroll
				for (int dx = 0; dx < 3; dx++)
					asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
					                 col + 16 * dx),
					             "r"(zero[0]), "r"(zero[1]), "r"(zero[2]), "r"(zero[3]), "r"(zero[4]), "r"(zero[5]),
					             "r"(zero[6]), "r"(zero[7]), "r"(zero[8]), "r"(zero[9]), "r"(zero[10]), "r"(zero[11]),
					             "r"(zero[12]), "r"(zero[13]), "r"(zero[14]), "r"(zero[15]));
				asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
				asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
				tc::arrive(k_free + 8 * b);
				// warp edges: lane 31's T0 goes to the next warp, lane 0's T2 to the previous
				float *xr = xch + (q & 1) * 128;
				if (lane == 31)
#pragma unroll
					for (int i = 0; i < 16; i++) xr[(warp * 2 + 0) * 16 + i] = t[0][i];
				if (lane == 0)
#pragma unroll
					for (int i = 0; i < 16; i++) xr[(warp * 2 + 1) * 16 + i] = t[2][i];
				if (lane == 0 || lane == 31) tc::arrive(x_bar + 8 * (unsigned)(q & 1));
				const bool xok = tc::mbar_wait(x_bar + 8 * (unsigned)(q & 1), (unsigned)((q >> 1) & 1), &abort_);
				if (!__all_sync(0xffffffffu, xok)) {
					quit = true;
					break;
				}
				// branch-free edges: every lane reads the neighbour warps' values
				// (one broadcast each), lanes 0 and 31 select them
				const float4 *xl = reinterpret_cast<const float4 *>(xr + ((warp > 0 ? warp - 1 : 0) * 2 + 0) * 16);
				const float4 *xg = reinterpret_cast<const float4 *>(xr + ((warp < 3 ? warp + 1 : 3) * 2 + 1) * 16);
				const bool has_l = lane == 0 && warp > 0, has_r = lane == 31 && warp < 3;
				const bool zero_l = lane == 0 && warp == 0, zero_r = lane == 31 && warp == 3;
				float o[16];
#pragma unroll
				for (int i4 = 0; i4 < 4; i4++) {
					const float4 el = xl[i4], er = xg[i4];
					const float ev_l[4] = {el.x, el.y, el.z, el.w}, ev_r[4] = {er.x, er.y, er.z, er.w};
#pragma unroll
					for (int k = 0; k < 4; k++) {
						const int i = 4 * i4 + k;
						float lf = __shfl_up_sync(0xffffffffu, t[0][i], 1);
						float rt = __shfl_down_sync(0xffffffffu, t[2][i], 1);
						lf = has_l ? ev_l[k] : (zero_l ? 0.f : lf);
						rt = has_r ? ev_r[k] : (zero_r ? 0.f : rt);
						o[i] = lf + t[1][i] + rt;
					}
				}
				// ReLU, bf16
				const long long v = ((long long)z * ny + r) * 128 + 32 * warp + lane;
				unsigned pk[8];
#pragma unroll
				for (int k = 0; k < 8; k++) {
					const __nv_bfloat162 h = __floats2bfloat162_rn(fmaxf(o[2 * k], 0.f), fmaxf(o[2 * k + 1], 0.f));
					pk[k] = *reinterpret_cast<const unsigned *>(&h);
				}
				uint4 *op = reinterpret_cast<uint4 *>(static_cast<bf16 *>(a.out) + v * 16);
				op[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
				op[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
			}
		}
	} else if (warp < 8) {
		// ---- producers: thread 128 issues the TMA boxes; with an upsampled A
		// part, thread p also gathers voxel x = p of its three z lines ----
		const int p = tid - 128;
		const bool tma_thread = p == 0;
		const unsigned tx_bytes = 3u * PL::TILE * (unsigned)(NK - (up ? 1 : 0));
		const int nyA = ny >> a.upA, nxA = 128 >> a.upA;
		if (tma_thread) {
			asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(&tmA)) : "memory");
			if (NK == 2) asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(&tmB)) : "memory");
		}
		long long g = 0; // lines staged
		if (up || tma_thread) {
			bool pending = false;
			for (long long rs = r0, re; rs < r1 && !abort_; rs = re) {
				const int z = (int)(rs / ny), ya = (int)(rs % ny);
				re = min(r1, (long long)(z + 1) * ny);
				const int yb = (int)(re - (long long)z * ny);
				const int l0 = max(ya - 1, 0), l1 = min(yb, ny - 1);
				for (int y = l0; y <= l1; y++, g++) {
					const int s = (int)(g % NSLOT);
					const long long k = g / NSLOT;
					if (k >= 1 && !tc::mbar_wait(b_free + 8 * s, (unsigned)((k - 1) & 1), &abort_)) break;
					unsigned char *slot = sl + (size_t)s * PL::SLOT;
					if (tma_thread) {
						tc::arrive_tx(b_full + 8 * s, tx_bytes);
#pragma unroll
						for (int dz = 0; dz < 3; dz++) {
							const int v0 = ((z + dz - 1) * ny + y) * 128; // outside the grid: zeros
							if (!up) tc::tma_line(tc::smem_u32(slot + (dz * NK) * PL::TILE), &tmA, v0, b_full + 8 * s);
							if (NK == 2) tc::tma_line(tc::smem_u32(slot + (dz * NK + 1) * PL::TILE), &tmB, v0, b_full + 8 * s);
						}
					}
					if (up) {
						// row p of part 0, 16-byte halves h stored at h ^ bit 2 of p
#pragma unroll
						for (int dz = 0; dz < 3; dz++) {
							const int Z = z + dz - 1;
							const bool in = Z >= 0 && Z < nz;
							const bf16 *src = in ? a.A + (((long long)(Z >> a.upA) * nyA + (y >> a.upA)) * nxA + (p >> a.upA)) * 16 : a.W;
							unsigned char *row = slot + (dz * NK) * PL::TILE + p * 32;
#pragma unroll
							for (int h = 0; h < 2; h++)
								asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
								                 tc::smem_u32(row + ((h ^ ((p >> 2) & 1)) << 4))),
								             "l"(src + 8 * h), "r"(in ? 16u : 0u)
								             : "memory");
						}
						asm volatile("cp.async.commit_group;" ::: "memory");
						// the previous line's gathers have landed: hand them on
						if (pending) {
							asm volatile("cp.async.wait_group 1;" ::: "memory");
							asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
							tc::arrive(b_full + 8 * (unsigned)((g - 1) % NSLOT));
						}
						pending = true;
					}
				}
			}
			if (up) {
				asm volatile("cp.async.wait_group 0;" ::: "memory");
				asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
				if (pending) tc::arrive(b_full + 8 * (unsigned)((g - 1) % NSLOT));
			}
		}
		// no TMA copy may still be in flight when the CTA leaves: wait (bounded)
		// for the last lines' slots
		if (tma_thread)
			for (long long h = g > NSLOT ? g - NSLOT : 0; h < g; h++) {
				volatile int never = 0;
				tc::mbar_wait(b_full + 8 * (unsigned)(h % NSLOT), (unsigned)((h / NSLOT) & 1), &never);
			}
	} else if (lane == 0) {
		// ---- MMA issue (warp 8, one thread) ----
		// descriptors of slot 0 / z tap 0 / K chunk 0; offsets add to the start field
		const unsigned long long adesc0 = tc::sdesc_sw32(tc::smem_u32(sl));
		const unsigned long long bdesc0 = tc::sdesc(tc::smem_u32(sw), 144 * 16, 128);
		int q0 = 0, gs = 0;   // rows of earlier units; slot of the current line
		unsigned gph = 0;     // phase parity of that slot
		bool issued = false, ok = true;
		for (long long rs = r0, re; rs < r1 && ok; rs = re) {
			const int z = (int)(rs / ny), ya = (int)(rs % ny);
			re = min(r1, (long long)(z + 1) * ny);
			const int yb = (int)(re - (long long)z * ny);
			const int l0 = max(ya - 1, 0), l1 = min(yb, ny - 1);
			int acq = ya, done = ya; // next row to acquire / to release
			for (int y = l0; y <= l1; y++) {
				const int rlo = max(y - 1, ya), rhi = min(y + 1, yb - 1); // rows this line feeds
				// the epilogue frees blocks in row order: the newest row's block
				// being free implies the blocks of the rows before it are
				if (acq <= rhi) {
					const int q = q0 + (rhi - ya);
					ok = tc::mbar_wait(k_free + 8 * (unsigned)(q % NB), (unsigned)((q / NB) & 1), &abort_);
					acq = rhi + 1;
				}
				if (!ok || !(ok = tc::mbar_wait(b_full + 8 * (unsigned)gs, gph, &abort_))) break;
				asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
				// rows rhi, rhi - 1, .., rlo take dy = jlo, jlo + 1, ..; their blocks
				// (one less each) sit at ascending columns up to block 0, then the
				// rest starts again at column 0 (block NB - 1)
				const int jlo = y + 1 - rhi, nrow = rhi - rlo + 1;
				const int b0 = (q0 + (rhi - ya)) % NB;
				const int n1 = min(nrow, b0 + 1), n2 = nrow - n1;
				const unsigned c1 = tmem + 48u * (unsigned)(NB - 1 - b0);
				const unsigned id1 = tc::idesc(48 * n1), id2 = tc::idesc(48 * max(n2, 1));
				const unsigned long long ad = adesc0 + (unsigned)(gs * (PL::SLOT >> 4));
				const unsigned long long bd1 = bdesc0 + (unsigned)(jlo * 48), bd2 = bdesc0 + (unsigned)((jlo + n1) * 48);
				// straight-line issue (the issuing thread's instructions between
				// MMAs cost tensor-core time at this size)
				if (n2 == 0) {
#pragma unroll
					for (int dz = 0; dz < 3; dz++)
#pragma unroll
						for (int kc = 0; kc < NK; kc++)
							tc::mma(c1, ad + (unsigned)(((dz * NK + kc) * PL::TILE) >> 4),
							        bd1 + (unsigned)((dz * PL::WDZ + kc * 2 * 2304) >> 4), id1);
				} else {
#pragma unroll
					for (int dz = 0; dz < 3; dz++)
#pragma unroll
						for (int kc = 0; kc < NK; kc++) {
							const unsigned ao = (unsigned)(((dz * NK + kc) * PL::TILE) >> 4);
							const unsigned bo = (unsigned)((dz * PL::WDZ + kc * 2 * 2304) >> 4);
							tc::mma(c1, ad + ao, bd1 + bo, id1);
							tc::mma(tmem, ad + ao, bd2 + bo, id2);
						}
				}
				tc::commit(b_free + 8 * (unsigned)gs);
				issued = true;
				if (++gs == NSLOT) {
					gs = 0;
					gph ^= 1u;
				}
				// rows whose last input line this was
				const int last = y == l1 ? yb - 1 : y - 1;
				for (; done <= last; done++) tc::commit(k_full + 8 * (unsigned)((q0 + (done - ya)) % NB));
			}
			q0 += yb - ya;
		}
		if (issued) { // drain before the accumulators are released
			tc::commit(f_bar);
			volatile int never = 0;
			tc::mbar_wait(f_bar, 0, &never);
		}
	}
	__syncwarp();
	if (abort_ && tid == 0) devstat_fail(st, BSG_ERR_TIMEOUT, (int)blockIdx.x, 30);
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
	if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem_base));
}

} // namespace

// ---- the network object ------------------------------------------------------
struct bsg_unet {
	bsg_ctx *ctx;
	const bsg_mat *mat;
	int nz, ny, nx;
	long long nv[4];            // voxels per level
	int woff[NW + 1];           // offsets of W0..W6 in the flat parameter vector (w7 at woff[NW])
	int nparam;
	float *master, *adam_m, *adam_v, *grad;
	bf16 *wb[NW], *wt[NW];
	float *w7b;                 // bf16-rounded head weights as FP32
	bf16 *logd;                 // normalised log-diagonal channel [R0]
	double *ld, *mom;           // log-diagonal scratch, its moments
	// activations
	bf16 *x0, *e0, *p1, *e1, *p2, *e2, *p3, *e3, *d2, *d1, *d0;
	float *y, *gy;
	double *r1, *t1, *ay;       // residual after the ILU2 step, SpMV scratch, A y
	double *sc;                 // scalars: [0] |r|^2, [4..7] reductions of the step / the loss
	double *part;               // reduction partials (3 x RED_BLOCKS)
	// training buffers
	bf16 *dd0, *gd1, *gd2, *ge3, *ge2, *ge1, *ge0;
	float *gi6, *gi5, *gi4, *gp3, *gp2, *gp1;
	int count;
	double loss_sum;
	bool train;
};

namespace {

template <class T>
int dalloc(bsg_ctx *c, T **p, size_t n) {
	if (cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess)
		return bsg_set_error(BSG_ERR_NOMEM, "U-Net buffers");
	(void)c;
	return BSG_OK;
}

template <bool F32OUT, int CH>
int conv_tiled(const ConvArgs &a, cudaStream_t s) {
	const size_t smem = (size_t)TH_VOX * CH * 2 + (size_t)27 * 16 * (CH + 8) * 2;
	BSG_CUDA(cudaFuncSetAttribute(k_conv3t<F32OUT, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	dim3 grid((unsigned)((a.nx / TT_X) * (a.ny / TT_Y) * (a.nz / TT_Z)), a.Cout / 16);
	k_conv3t<F32OUT, CH><<<grid, 256, smem, s>>>(a);
	return BSG_OK;
}

// cuTensorMapEncodeTiled, through the runtime's driver entry point
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	static bool tried = false;
	if (!tried) {
		tried = true;
		void *f = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
		    q == cudaDriverEntryPointSuccess)
			fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
	}
	return fn;
}

// 2D map of a [nv][16] bf16 array: boxes of 128 voxels x 16 channels in the
// 32-byte swizzle; boxes outside [0, nv) read as zeros
int tmap_lines(CUtensorMap *m, const bf16 *p, long long nv) {
	const PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
	if (!enc) return bsg_set_error(BSG_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
	const cuuint64_t dim[2] = {16, (cuuint64_t)nv};
	const cuuint64_t stride[1] = {16 * sizeof(bf16)};
	const cuuint32_t box[2] = {16, 128}, estride[2] = {1, 1};
	if (enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(p), dim, stride, box, estride,
	        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
	        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
		return bsg_set_error(BSG_ERR_CUDA, "cuTensorMapEncodeTiled failed");
	return BSG_OK;
}

// the tensor-core (tcgen05) convolution: a persistent grid, two CTAs per SM;
// A has 16 channels (full or half resolution), B none or 16; ReLU, bf16 out
template <int CIN>
int conv_tc(const ConvArgs &a, bsg_ctx *c) {
	constexpr size_t smem = tc::Plan<CIN>::BYTES;
	const long long nv = (long long)a.nz * a.ny * a.nx;
	CUtensorMap ta, tb;
	int rc;
	// an upsampled A is gathered instead; its map is only a valid placeholder
	if ((rc = tmap_lines(&ta, a.A, a.upA ? nv >> (3 * a.upA) : nv))) return rc;
	if (CIN == 32) {
		if ((rc = tmap_lines(&tb, a.B, nv))) return rc;
	} else {
		tb = ta;
	}
	BSG_CUDA(cudaFuncSetAttribute(k_conv3_tc<CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	const long long nrow = (long long)a.nz * a.ny;
	const long long cap = (long long)BSG_SMS * tc::CTAS;
	const long long grid = nrow < cap ? nrow : cap;
	k_conv3_tc<CIN><<<(unsigned)grid, tc::THREADS, smem, c->stream>>>(a, ta, tb, c->d_stat);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

int conv_launch(bsg_unet *u, int lvl, const bf16 *A, int Ca, int upA, const bf16 *B, int Cb, const bf16 *W, int Cout,
                void *out, bool f32out) {
	cudaStream_t s = u->ctx->stream;
	ConvArgs a;
	a.nz = u->nz >> lvl; a.ny = u->ny >> lvl; a.nx = u->nx >> lvl;
	a.A = A; a.Ca = Ca; a.upA = upA; a.B = B; a.Cb = Cb; a.W = W; a.Cout = Cout; a.out = out;
	const int Cin = Ca + Cb;
	BSG_COUNT(1);
	// 16 outputs from 16 or 32 inputs on x-lines of 128 voxels: tcgen05 (TMA
	// line coordinates are 32-bit voxel indices)
	if (Cout == 16 && !f32out && a.nx == 128 && Ca == 16 && (Cb == 0 || Cb == 16) && upA <= 1 &&
	    (long long)a.nz * a.ny * 128 < (1ll << 31))
		return Cin == 16 ? conv_tc<16>(a, u->ctx) : conv_tc<32>(a, u->ctx);
	if (a.nx % TT_X == 0 && a.ny % TT_Y == 0 && a.nz % TT_Z == 0) {
		int rc;
		if (Cin % 32 == 0)
			rc = f32out ? conv_tiled<true, 32>(a, s) : conv_tiled<false, 32>(a, s);
		else
			rc = f32out ? conv_tiled<true, 16>(a, s) : conv_tiled<false, 16>(a, s);
		if (rc) return rc;
		BSG_CUDA(cudaGetLastError());
		return BSG_OK;
	}
	const size_t smem = (size_t)3 * CONV_MT * 8 * 32 * sizeof(float) + (size_t)27 * 16 * (Cin + 8) * sizeof(bf16);
	const long long ntile = (u->nv[lvl] + 16 * CONV_MT - 1) / (16 * CONV_MT);
	long long bx = ntile;
	const long long cap = (long long)BSG_SMS * 8 / (Cout / 16);
	if (bx > cap) bx = cap;
	if (bx < 1) bx = 1;
	dim3 grid((unsigned)bx, Cout / 16);
	if (f32out) {
		BSG_CUDA(cudaFuncSetAttribute(k_conv3<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
		k_conv3<true><<<grid, 128, smem, s>>>(a);
	} else {
		BSG_CUDA(cudaFuncSetAttribute(k_conv3<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
		k_conv3<false><<<grid, 128, smem, s>>>(a);
	}
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

int wgrad_launch(bsg_unet *u, int lvl, const bf16 *A, int Ca, int upA, const bf16 *B, int Cb, int Cout, const bf16 *g,
                 float *dW) {
	ConvArgs a;
	a.nz = u->nz >> lvl; a.ny = u->ny >> lvl; a.nx = u->nx >> lvl;
	a.A = A; a.Ca = Ca; a.upA = upA; a.B = B; a.Cb = Cb; a.W = nullptr; a.Cout = Cout; a.out = nullptr;
	const long long nvox = u->nv[lvl];
	long long chunk = (nvox + 2 * BSG_SMS - 1) / (2 * BSG_SMS);
	if (chunk < 64) chunk = 64;
	const int blocks = (int)((nvox + chunk - 1) / chunk);
	BSG_COUNT(1);
	k_wgrad<<<blocks, 256, 0, u->ctx->stream>>>(a, g, chunk, dW);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

int pool_launch(bsg_unet *u, int lvl, int C, const bf16 *in, bf16 *out) {
	BSG_COUNT(1);
	k_pool<<<ew(u->nv[lvl + 1] * (C / 8)), 256, 0, u->ctx->stream>>>(u->nz >> lvl, u->ny >> lvl, u->nx >> lvl, C, in, out);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

int sumsq(bsg_unet *u, long long n, const double *x, double *out) {
	BSG_COUNT(2);
	k_sumsq_part<<<SQ_BLOCKS, 256, 0, u->ctx->stream>>>(n, x, u->part);
	k_sum_final<<<1, 32, 0, u->ctx->stream>>>(SQ_BLOCKS, u->part, out);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// Forward pass from r (FP64, |r|^2 already in u->sc[0]) to y (FP32).
int forward(bsg_unet *u, const double *r) {
	cudaStream_t s = u->ctx->stream;
	int rc;
	BSG_COUNT(1);
	k_input<<<ew(u->nv[0]), 256, 0, s>>>(u->nv[0], r, u->sc, u->logd, u->x0);
	if ((rc = conv_launch(u, 0, u->x0, 16, 0, nullptr, 0, u->wb[0], 16, u->e0, false))) return rc;
	if ((rc = pool_launch(u, 0, 16, u->e0, u->p1))) return rc;
	if ((rc = conv_launch(u, 1, u->p1, 16, 0, nullptr, 0, u->wb[1], 32, u->e1, false))) return rc;
	if ((rc = pool_launch(u, 1, 32, u->e1, u->p2))) return rc;
	if ((rc = conv_launch(u, 2, u->p2, 32, 0, nullptr, 0, u->wb[2], 64, u->e2, false))) return rc;
	if ((rc = pool_launch(u, 2, 64, u->e2, u->p3))) return rc;
	if ((rc = conv_launch(u, 3, u->p3, 64, 0, nullptr, 0, u->wb[3], 64, u->e3, false))) return rc;
	if ((rc = conv_launch(u, 2, u->e3, 64, 1, u->e2, 64, u->wb[4], 32, u->d2, false))) return rc;
	if ((rc = conv_launch(u, 1, u->d2, 32, 1, u->e1, 32, u->wb[5], 16, u->d1, false))) return rc;
	if ((rc = conv_launch(u, 0, u->d1, 16, 1, u->e0, 16, u->wb[6], 16, u->d0, false))) return rc;
	BSG_COUNT(1);
	k_head<<<ew(u->nv[0]), 256, 0, s>>>(u->nv[0], u->d0, u->w7b, u->y);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// Backward pass from gy; accumulates into u->grad.
int backward(bsg_unet *u) {
	cudaStream_t s = u->ctx->stream;
	float *G = u->grad;
	const int *o = u->woff;
	int rc;
	const int R[4][3] = {{u->nz, u->ny, u->nx}, {u->nz >> 1, u->ny >> 1, u->nx >> 1},
	                     {u->nz >> 2, u->ny >> 2, u->nx >> 2}, {u->nz >> 3, u->ny >> 3, u->nx >> 3}};
	BSG_COUNT(1);
	k_head_bwd<<<ew(u->nv[0]), 256, 0, s>>>(u->nv[0], u->d0, u->w7b, u->gy, u->dd0, G + o[NW]);
	// W6: in = [up d1, e0]
	if ((rc = wgrad_launch(u, 0, u->d1, 16, 1, u->e0, 16, 16, u->dd0, G + o[6]))) return rc;
	if ((rc = conv_launch(u, 0, u->dd0, 16, 0, nullptr, 0, u->wt[6], 32, u->gi6, true))) return rc;
	BSG_COUNT(1);
	k_grad_act<<<ew(u->nv[1] * 16), 256, 0, s>>>(R[1][0], R[1][1], R[1][2], 16, u->gi6, 32, 0, nullptr, 0, 0, nullptr,
	                                            u->d1, u->gd1);
	// W5: in = [up d2, e1]
	if ((rc = wgrad_launch(u, 1, u->d2, 32, 1, u->e1, 32, 16, u->gd1, G + o[5]))) return rc;
	if ((rc = conv_launch(u, 1, u->gd1, 16, 0, nullptr, 0, u->wt[5], 64, u->gi5, true))) return rc;
	BSG_COUNT(1);
	k_grad_act<<<ew(u->nv[2] * 32), 256, 0, s>>>(R[2][0], R[2][1], R[2][2], 32, u->gi5, 64, 0, nullptr, 0, 0, nullptr,
	                                            u->d2, u->gd2);
	// W4: in = [up e3, e2]
	if ((rc = wgrad_launch(u, 2, u->e3, 64, 1, u->e2, 64, 32, u->gd2, G + o[4]))) return rc;
	if ((rc = conv_launch(u, 2, u->gd2, 32, 0, nullptr, 0, u->wt[4], 128, u->gi4, true))) return rc;
	BSG_COUNT(1);
	k_grad_act<<<ew(u->nv[3] * 64), 256, 0, s>>>(R[3][0], R[3][1], R[3][2], 64, u->gi4, 128, 0, nullptr, 0, 0, nullptr,
	                                            u->e3, u->ge3);
	// W3: in = p3
	if ((rc = wgrad_launch(u, 3, u->p3, 64, 0, nullptr, 0, 64, u->ge3, G + o[3]))) return rc;
	if ((rc = conv_launch(u, 3, u->ge3, 64, 0, nullptr, 0, u->wt[3], 64, u->gp3, true))) return rc;
	BSG_COUNT(1);
	k_grad_act<<<ew(u->nv[2] * 64), 256, 0, s>>>(R[2][0], R[2][1], R[2][2], 64, nullptr, 0, 0, u->gi4, 128, 64, u->gp3,
	                                            u->e2, u->ge2);
	// W2: in = p2
	if ((rc = wgrad_launch(u, 2, u->p2, 32, 0, nullptr, 0, 64, u->ge2, G + o[2]))) return rc;
	if ((rc = conv_launch(u, 2, u->ge2, 64, 0, nullptr, 0, u->wt[2], 32, u->gp2, true))) return rc;
	BSG_COUNT(1);
	k_grad_act<<<ew(u->nv[1] * 32), 256, 0, s>>>(R[1][0], R[1][1], R[1][2], 32, nullptr, 0, 0, u->gi5, 64, 32, u->gp2,
	                                            u->e1, u->ge1);
	// W1: in = p1
	if ((rc = wgrad_launch(u, 1, u->p1, 16, 0, nullptr, 0, 32, u->ge1, G + o[1]))) return rc;
	if ((rc = conv_launch(u, 1, u->ge1, 32, 0, nullptr, 0, u->wt[1], 16, u->gp1, true))) return rc;
	BSG_COUNT(1);
	k_grad_act<<<ew(u->nv[0] * 16), 256, 0, s>>>(R[0][0], R[0][1], R[0][2], 16, nullptr, 0, 0, u->gi6, 32, 16, u->gp1,
	                                            u->e0, u->ge0);
	// W0: in = x0
	if ((rc = wgrad_launch(u, 0, u->x0, 16, 0, nullptr, 0, 16, u->ge0, G + o[0]))) return rc;
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

int refresh(bsg_unet *u) {
	cudaStream_t s = u->ctx->stream;
	for (int k = 0; k < NW; k++) {
		const int len = 27 * CIN[k] * COUT[k];
		BSG_COUNT(1);
		k_refresh<<<ew(len), 256, 0, s>>>(len, COUT[k], CIN[k], u->master + u->woff[k], u->wb[k], u->wt[k]);
	}
	BSG_COUNT(1);
	k_w7<<<1, 32, 0, s>>>(u->master + u->woff[NW], u->w7b);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

} // namespace

extern "C" int bsg_unet_free(bsg_unet *u);

extern "C" int bsg_unet_create(bsg_ctx *c, int nx, int ny, int nz, int train, bsg_unet **out) {
	if (!c || !out) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_create: null argument");
	*out = nullptr;
	if (nx < 8 || ny < 8 || nz < 8 || nx % 8 || ny % 8 || nz % 8)
		return bsg_set_error(BSG_ERR_ARG, "bsg_unet_create: grid sides must be multiples of 8 (three poolings)");
	BSG_CUDA(cudaSetDevice(c->device));
	bsg_unet *u = new bsg_unet();
	std::memset(u, 0, sizeof(*u));
	u->ctx = c;
	u->nz = nz; u->ny = ny; u->nx = nx;
	for (int l = 0; l < 4; l++) u->nv[l] = (long long)(nz >> l) * (ny >> l) * (nx >> l);
	u->train = train != 0;
	int off = 0;
	for (int k = 0; k < NW; k++) { u->woff[k] = off; off += 27 * CIN[k] * COUT[k]; }
	u->woff[NW] = off;
	u->nparam = off + 16;
	int rc = BSG_OK;
	auto A = [&](auto **p, size_t n) { if (!rc) rc = dalloc(c, p, n); };
	A(&u->master, u->nparam);
	A(&u->adam_m, u->nparam);
	A(&u->adam_v, u->nparam);
	A(&u->grad, u->nparam);
	for (int k = 0; k < NW; k++) {
		A(&u->wb[k], (size_t)27 * CIN[k] * COUT[k]);
		A(&u->wt[k], (size_t)27 * CIN[k] * COUT[k]);
	}
	A(&u->w7b, 16);
	const long long *nv = u->nv;
	A(&u->logd, nv[0]); A(&u->ld, nv[0]); A(&u->mom, 2);
	A(&u->x0, nv[0] * 16); A(&u->e0, nv[0] * 16); A(&u->p1, nv[1] * 16); A(&u->e1, nv[1] * 32);
	A(&u->p2, nv[2] * 32); A(&u->e2, nv[2] * 64); A(&u->p3, nv[3] * 64); A(&u->e3, nv[3] * 64);
	A(&u->d2, nv[2] * 32); A(&u->d1, nv[1] * 16); A(&u->d0, nv[0] * 16);
	A(&u->y, nv[0]); A(&u->gy, nv[0]);
	A(&u->r1, nv[0]); A(&u->t1, nv[0]); A(&u->ay, nv[0]); A(&u->sc, 8); A(&u->part, 3 * RED_BLOCKS);
	if (u->train) {
		A(&u->dd0, nv[0] * 16); A(&u->gd1, nv[1] * 16); A(&u->gd2, nv[2] * 32); A(&u->ge3, nv[3] * 64);
		A(&u->ge2, nv[2] * 64); A(&u->ge1, nv[1] * 32); A(&u->ge0, nv[0] * 16);
		A(&u->gi6, nv[0] * 32); A(&u->gi5, nv[1] * 64); A(&u->gi4, nv[2] * 128);
		A(&u->gp3, nv[3] * 64); A(&u->gp2, nv[2] * 32); A(&u->gp1, nv[1] * 16);
	}
	if (!rc && cudaMemset(u->grad, 0, sizeof(float) * u->nparam) != cudaSuccess) rc = BSG_ERR_CUDA;
	if (!rc && cudaMemset(u->adam_m, 0, sizeof(float) * u->nparam) != cudaSuccess) rc = BSG_ERR_CUDA;
	if (!rc && cudaMemset(u->adam_v, 0, sizeof(float) * u->nparam) != cudaSuccess) rc = BSG_ERR_CUDA;
	if (!rc && cudaMemset(u->logd, 0, sizeof(bf16) * nv[0]) != cudaSuccess) rc = BSG_ERR_CUDA;
	if (rc) {
		bsg_unet_free(u);
		return rc;
	}
	*out = u;
	return BSG_OK;
}

extern "C" int bsg_unet_free(bsg_unet *u) {
	if (!u) return BSG_OK;
	void *ps[] = {u->master, u->adam_m, u->adam_v, u->grad, u->w7b, u->logd, u->ld, u->mom, u->x0, u->e0, u->p1,
	              u->e1, u->p2, u->e2, u->p3, u->e3, u->d2, u->d1, u->d0, u->y, u->gy, u->r1, u->t1, u->sc, u->part,
	              u->ay, u->dd0, u->gd1, u->gd2, u->ge3, u->ge2, u->ge1, u->ge0, u->gi6, u->gi5, u->gi4, u->gp3,
	              u->gp2, u->gp1};
	cudaStreamSynchronize(u->ctx->stream);
	for (void *p : ps)
		if (p) cudaFree(p);
	for (int k = 0; k < NW; k++) {
		if (u->wb[k]) cudaFree(u->wb[k]);
		if (u->wt[k]) cudaFree(u->wt[k]);
	}
	delete u;
	return BSG_OK;
}

extern "C" int bsg_unet_nparam(const bsg_unet *u) {
	return u ? u->nparam : bsg_set_error(BSG_ERR_ARG, "bsg_unet_nparam: null network");
}

// Weights in the flat FP32 layout W0..W6 ([tap][cout][cin] each), then w7.
extern "C" int bsg_unet_set_weights(bsg_unet *u, const float *w) {
	if (!u || !w) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_set_weights: null argument");
	BSG_CUDA(cudaMemcpyAsync(u->master, w, sizeof(float) * u->nparam, cudaMemcpyHostToDevice, u->ctx->stream));
	int rc = refresh(u);
	if (!rc) BSG_CUDA(cudaStreamSynchronize(u->ctx->stream));
	return rc;
}
extern "C" int bsg_unet_get_weights(bsg_unet *u, float *w) {
	if (!u || !w) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_get_weights: null argument");
	BSG_CUDA(cudaMemcpyAsync(w, u->master, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost, u->ctx->stream));
	BSG_CUDA(cudaStreamSynchronize(u->ctx->stream));
	return BSG_OK;
}
extern "C" int bsg_unet_get_grads(bsg_unet *u, float *g) {
	if (!u || !g) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_get_grads: null argument");
	BSG_CUDA(cudaMemcpyAsync(g, u->grad, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost, u->ctx->stream));
	BSG_CUDA(cudaStreamSynchronize(u->ctx->stream));
	return BSG_OK;
}

// The operator whose diagonal feeds the second input channel, and whose
// product forms the residual after the ILU2 step inside FGMRES.  Point
// matrices on an nx x ny x nz grid in natural order.
extern "C" int bsg_unet_set_matrix(bsg_unet *u, const bsg_mat *m) {
	if (!u || !m) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_set_matrix: null argument");
	if (m->bs != 1 || (long long)m->n != u->nv[0])
		return bsg_set_error(BSG_ERR_ARG, "bsg_unet_set_matrix: matrix size does not match the grid");
	u->mat = m;
	cudaStream_t s = u->ctx->stream;
	BSG_COUNT(4);
	k_logdiag<<<ew(m->n), 256, 0, s>>>(m->n, m->d_iu, m->d_al, u->ld);
	k_moments_part<<<SQ_BLOCKS, 256, 0, s>>>(m->n, u->ld, u->part);
	k_moments_final<<<1, 32, 0, s>>>(m->n, SQ_BLOCKS, u->part, u->mom);
	k_logd_norm<<<ew(m->n), 256, 0, s>>>(m->n, u->ld, u->mom, u->logd);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// The second input channel from a device vector of diagonal values (the
// matrix's diagonal), without binding a matrix: training switches between
// instances this way.
extern "C" int bsg_unet_set_diag(bsg_unet *u, const double *d_diag) {
	if (!u || !d_diag) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_set_diag: null argument");
	cudaStream_t s = u->ctx->stream;
	const int n = (int)u->nv[0];
	BSG_COUNT(4);
	k_logvec<<<ew(n), 256, 0, s>>>(n, d_diag, u->ld);
	k_moments_part<<<SQ_BLOCKS, 256, 0, s>>>(n, u->ld, u->part);
	k_moments_final<<<1, 32, 0, s>>>(n, SQ_BLOCKS, u->part, u->mom);
	k_logd_norm<<<ew(n), 256, 0, s>>>(n, u->ld, u->mom, u->logd);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// y_out = N(r / |r|) (FP64), the network's output direction for residual r.
extern "C" int bsg_unet_forward_dev(bsg_unet *u, const double *r, double *y_out) {
	if (!u || !r || !y_out) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_forward_dev: null argument");
	int rc = sumsq(u, u->nv[0], r, u->sc);
	if (!rc) rc = forward(u, r);
	if (rc) return rc;
	BSG_COUNT(1);
	k_widen<<<ew(u->nv[0]), 256, 0, u->ctx->stream>>>(u->nv[0], u->y, y_out);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// One training sample: input residual r, target correction t (both FP64 on
// the device).  Accumulates the weight gradients of 1 - cos^2(N(r/|r|), t);
// *loss (may be NULL) gets the sample's loss.
extern "C" int bsg_unet_train_sample(bsg_unet *u, const double *r, const double *t, double *loss) {
	if (!u || !r || !t) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_train_sample: null argument");
	if (!u->train) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_train_sample: network created without training buffers");
	cudaStream_t s = u->ctx->stream;
	int rc = sumsq(u, u->nv[0], r, u->sc);
	if (!rc) rc = forward(u, r);
	if (rc) return rc;
	BSG_COUNT(3);
	k_red3<<<RED_BLOCKS, 256, 0, s>>>(u->nv[0], u->y, t, u->part);
	k_red_final<<<1, 32, 0, s>>>(3, u->part, u->sc + 4);
	k_cos_grad<<<ew(u->nv[0]), 256, 0, s>>>(u->nv[0], u->y, t, u->sc + 4, u->gy);
	if ((rc = backward(u))) return rc;
	u->count++;
	if (loss) {
		BSG_CUDA(cudaMemcpyAsync(loss, u->sc + 7, sizeof(double), cudaMemcpyDeviceToHost, s));
		BSG_CUDA(cudaStreamSynchronize(s));
	}
	return BSG_OK;
}

// Adam step with the gradients accumulated since the last step (averaged).
extern "C" int bsg_unet_adam(bsg_unet *u, float lr, float beta1, float beta2, float eps, int step) {
	if (!u || step < 1) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_adam: bad argument");
	const float inv = u->count > 0 ? 1.f / (float)u->count : 0.f;
	const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
	BSG_COUNT(1);
	k_adam<<<ew(u->nparam), 256, 0, u->ctx->stream>>>(u->nparam, u->master, u->adam_m, u->adam_v, u->grad, inv, lr,
	                                                 beta1, beta2, eps, c1, c2, u->woff[1]);
	BSG_CUDA(cudaGetLastError());
	u->count = 0;
	return refresh(u);
}

extern "C" int bsg_unet_zero_grads(bsg_unet *u) {
	if (!u) return bsg_set_error(BSG_ERR_ARG, "bsg_unet_zero_grads: null network");
	BSG_CUDA(cudaMemsetAsync(u->grad, 0, sizeof(float) * u->nparam, u->ctx->stream));
	u->count = 0;
	return BSG_OK;
}

// FGMRES learned stage: z holds the ILU2 step M^{-1} v on entry; the
// network's direction y = N(r1/|r1|) for the remaining error, r1 = v - A z,
// is added with the step alpha = (r1 . y) / (y . A y) that minimises the
// A-norm of that error.  A step that is not finite and positive leaves z as
// the plain ILU2 step.  `work` is unused (own buffers).  All on the device
// stream, no host synchronisation.
int bsg_unet_apply(void *net, bsg_ctx *c, const double *v, double *z, double *work) {
	(void)work;
	bsg_unet *u = static_cast<bsg_unet *>(net);
	if (!u || !u->mat) return bsg_set_error(BSG_ERR_ARG, "learned stage: network has no matrix");
	if (u->ctx != c) return bsg_set_error(BSG_ERR_ARG, "learned stage: network belongs to another context");
	cudaStream_t s = c->stream;
	const long long n = u->nv[0];
	int rc = bsg_spmm_launch(u->mat, 1, z, u->t1, n, s);
	if (rc) return bsg_set_error(rc, "learned stage: SpMV failed");
	BSG_COUNT(1);
	k_sub<<<ew(n), 256, 0, s>>>(n, v, u->t1, u->r1);
	if ((rc = sumsq(u, n, u->r1, u->sc))) return rc;
	if ((rc = forward(u, u->r1))) return rc;
	BSG_COUNT(1);
	k_widen<<<ew(n), 256, 0, s>>>(n, u->y, u->t1);
	if ((rc = bsg_spmm_launch(u->mat, 1, u->t1, u->ay, n, s))) return bsg_set_error(rc, "learned stage: SpMV failed");
	BSG_COUNT(3);
	k_red2<<<RED_BLOCKS, 256, 0, s>>>(n, u->r1, u->t1, u->ay, u->part);
	k_red_final<<<1, 32, 0, s>>>(2, u->part, u->sc + 4);
	k_correct<<<ew(n), 256, 0, s>>>(n, u->t1, u->sc + 4, z);
	BSG_CUDA(cudaGetLastError());
	return BSG_OK;
}

// this unit's copy of the spin-wait bound (bsg_set_spin_limit_ns)
int bsg_spin_limit_set_unet(unsigned long long ns) {
	return bsg_spin_limit_set_here(ns) == cudaSuccess ? BSG_OK : BSG_ERR_CUDA;
}
