// Internal declarations of the B200 solver library (libbsg.so).
// Everything here is sm_100a device code or host glue around it; the public
// C ABI lives in include/bslib_gpu.h.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include "../../include/bslib_gpu.h"

#define BSG_WARP 32
#define BSG_SMS 148

// ---- error handling -------------------------------------------------------
#define BSG_CUDA(call)                                                        \
	do {                                                                      \
		cudaError_t e_ = (call);                                              \
		if (e_ != cudaSuccess) return bsg_set_cuda_error(e_, #call, __FILE__, __LINE__); \
	} while (0)

int bsg_set_cuda_error(cudaError_t e, const char *what, const char *file, int line);
int bsg_set_error(int code, const char *msg);

// Device-side status word written by kernels that can fail (pivot, workspace,
// spin-wait limit).  The first failure wins (atomicCAS from 0).
struct bsg_devstat {
	int code;  // 0 = ok, else a BSG_ERR_* value
	int where; // row / index that failed
	int pad[2];
};

// ---- device helpers -------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
	for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
	return v;
}
__device__ __forceinline__ int ld_acquire(const int *p) {
	int v;
	asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
	asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
	unsigned long long v;
	asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
	asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_volatile_u64(const void *p) {
	unsigned long long v;
	asm volatile("ld.volatile.global.b64 %0, [%1];" : "=l"(v) : "l"(p));
	return v;
}
__device__ __forceinline__ void st_volatile_f64(double *p, double v) {
	asm volatile("st.volatile.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}
__device__ __forceinline__ void devstat_fail(bsg_devstat *st, int code, int where, int site = 0) {
	if (atomicCAS(&st->code, 0, code) == 0) {
		st->where = where;
		st->pad[0] = site;
	}
}

// Bit pattern that no arithmetic result carries (a signalling NaN payload);
// marks "not yet solved" entries in the sync-free triangular solves.
#define BSG_PENDING 0x7FF4DEADBEEF0001ull

// Spin-wait bound: every device wait on another warp's result gives up after
// this many nanoseconds of globaltimer time, reports BSG_ERR_TIMEOUT and
// returns.  The default, two seconds, is far above any legitimate wait;
// bsg_set_spin_limit_ns() changes it.  Every translation unit with waits
// keeps its own copy in constant memory (static), set through
// bsg_spin_limit_set_here() from that unit, for the current device.
#define BSG_SPIN_LIMIT_DEFAULT_NS 2000000000ull
static __constant__ unsigned long long c_bsg_spin_limit_ns = BSG_SPIN_LIMIT_DEFAULT_NS;
#define BSG_SPIN_LIMIT_NS c_bsg_spin_limit_ns
static inline __attribute__((unused)) cudaError_t bsg_spin_limit_set_here(unsigned long long ns) {
	return cudaMemcpyToSymbol(c_bsg_spin_limit_ns, &ns, sizeof ns);
}

// ---- device-resident objects ---------------------------------------------
struct bsg_ctx {
	int device;
	cudaStream_t stream;
	bool own_stream;
	bsg_devstat *d_stat;     // device status word
	double *d_scalars;       // small device scratch for reductions / Krylov scalars
	double *d_partials;      // block partial sums
	unsigned int *d_counters;
	double *h_pinned;        // pinned host mirror of a few scalars
	int n_partials;
	cudaEvent_t ev0, ev1;
	int spmv_group;          // autotuned sub-warp size for CSR SpMV (0 = choose per matrix)
};

// SELL-8: slices of 8 rows, entries column-major inside a slice (k_sell.cu).
struct bsg_sell {
	int n = 0;
	int fp32 = 0;
	long long entries = 0;   // stored entries including padding
	long long *off = nullptr; // slice offsets [nslices + 1]
	int *col = nullptr;
	void *val = nullptr;      // float or double
	int *perm = nullptr;      // slot -> row when rows are sorted by length in windows (SELL-C-sigma)
	// Tiled form (FP32 sweeps): tiles of 256 slots; tile t reads x only in the
	// 32-float blocks tb[tb_off[t] .. tb_off[t+1]), staged in shared memory,
	// and its columns are 16-bit indices into that staging, two per word in
	// cpair (slice widths even).  ntile == 0: no tiled form.
	int ntile = 0;
	int tmax = 0;             // most blocks of one tile
	int tgrid = 0;            // persistent grid of the tiled sweep
	int *tb_off = nullptr;
	int *tb = nullptr;
	unsigned *cpair = nullptr;
	// Long rows (more than SELL_LONG entries; none in the tiled form) are left
	// out of the slices -- their slots hold padding and bit l of lmask[slice]
	// marks them -- and kept as CSR: rows lrow[0 .. nvlong) (more than
	// SELL_VLONG entries) are summed by a whole block each, the rest of
	// lrow[0 .. nlong) by one warp each, so no slice waits on one lane walking
	// a row of thousands of entries.
	int nlong = 0, nvlong = 0;
	int *lrow = nullptr;
	long long *loff = nullptr; // [nlong + 1]
	int *lcol = nullptr;
	void *lval = nullptr;      // float or double, as val
	unsigned char *lmask = nullptr;
};
// sigma > 0: sort rows by length inside windows of sigma rows first;
// tiled != 0 (FP32 only, sigma dividing 256): also build the tiled form when
// every tile's x blocks fit the staging limit
int bsg_sell_build(bsg_ctx *c, int n, const int *rp, const int *ci, const double *v, int skip, int fp32,
                   bsg_sell *out, int sigma = 0, int tiled = 0);
void bsg_sell_free(bsg_sell *m, cudaStream_t s);
int bsg_sell_spmv(cudaStream_t s, const bsg_sell *m, const double *x, double *y);
int bsg_sell_sweep(cudaStream_t s, const bsg_sell *m, const double *x, const double *dinv, const double *yin,
                   int scaled_in, double *yout);
int bsg_sell_sweeps32(cudaStream_t s, const bsg_sell *m, const double *x, const double *dinv, int nsweeps,
                      float *work32, double *yout);
int bsg_sell_sweep32_pass(cudaStream_t s, const bsg_sell *m, const double *x, const double *dinv, const float *x32,
                          double *yout);
// The same for nr vectors at stride n, the matrix read once per 8 vectors;
// every vector gets the bits of a single-vector call.  work32: 2 n nr floats.
int bsg_sell_sweep_multi(cudaStream_t s, const bsg_sell *m, int nr, const double *x, const double *dinv,
                         const double *yin, int scaled_in, double *yout);
int bsg_sell_sweeps32_multi(cudaStream_t s, const bsg_sell *m, int nr, const double *x, const double *dinv,
                            int nsweeps, float *work32, double *yout);

// Block SELL of 3 x 3 blocks (k_bsell.cu): slices of 8 block rows, block k
// of slot l at off_s + 8 k + l (column: block column), its 9 values row-major
// in planes: value p at 9 off_s + 72 k + 8 p + l.  Block rows of more than
// 64 blocks are kept out of the slices as block CSR (lrow / loff / lcol /
// lval, 9 values a block), summed by a warp each, or by a block of 256
// threads beyond 1024 blocks (the first nvlong of them).
struct bsg_bsell {
	int nb = 0;
	int fp32 = 0;
	long long blocks = 0;     // stored blocks, padding and long rows included
	long long *off = nullptr; // slice offsets in blocks [nslices + 1]
	int *col = nullptr;
	void *val = nullptr;      // float or double
	int nlong = 0, nvlong = 0;
	int *lrow = nullptr;
	long long *loff = nullptr;
	int *lcol = nullptr;
	void *lval = nullptr;
	unsigned char *lmask = nullptr;
};
// From the point CSR of a strict block part (every block's 9 entries stored,
// blocks in column order in each point row).
int bsg_bsell_build(bsg_ctx *c, int nb, const int *rp, const int *ci, const double *v, int fp32, bsg_bsell *out);
void bsg_bsell_free(bsg_bsell *m, cudaStream_t s);
// Block Jacobi sweeps for nr vectors at stride 3 nb: y0 = D x, then
// nsweeps - 1 passes y <- D (x - N y) (D: nb column-major 3 x 3 blocks), one
// kernel a pass, the factor read once per 8 vectors; work: 3 nb nr doubles
// (nsweeps > 1).  With scr (bsg_bsell_scratch(nb, nr) doubles, 16-byte
// aligned) several vectors keep their intermediate iterates interleaved there
// and work is not used.  Every vector gets the bits of a single-vector call.
int bsg_bsell_sweeps(cudaStream_t s, const bsg_bsell *m, const double *d, int nsweeps, int nr, const double *x,
                     double *y, double *work, double *scr = nullptr);
size_t bsg_bsell_scratch(int nb, int nr);

struct bsg_mat {
	bsg_ctx *ctx;
	int n;        // rows (point) or block rows
	int bs;       // block size
	int nnz;      // stored entries / blocks in the full (both triangles) matrix
	int symm;     // 1 if created from an upper-triangle symmetric input
	int *d_ia, *d_ja;
	double *d_a;  // point values, or bs*bs row-major blocks for bs > 1
	// upper pattern with diagonal first (factorisation input) and its
	// transpose (the static contributor lists of each row)
	int nnz_up;
	int *d_iu, *d_ju;
	double *d_al, *d_au;  // ILU2 split values (al == au for symmetric input)
	int *d_it, *d_jt;     // transpose of the strict upper pattern: rows k < i with (k,i) stored
	int group;            // CSR SpMV sub-warp size
	bsg_sell sell;        // SELL-8 copy of a point matrix (single-vector SpMV)
	bsg_sell sellT;       // SELL-8 copy of A^T, built on first use (transposed products)
};

struct bsg_fct {
	bsg_ctx *ctx;
	int n, bs;
	int kind;      // 0 IC2, 1 ILU2
	int nnz;       // entries of U including the diagonal
	int fp32;      // 1 if off-diagonal values are stored in FP32
	// U by rows (reference layout, diagonal = inverse pivot first), FP64
	int *d_iu, *d_ju;
	double *d_u;   // U values
	double *d_l;   // L values by columns (== d_u for IC2)
	// solve-ready forms: strict parts + inverse pivots
	double *d_dinv_l, *d_dinv_u;  // inverse pivots (FP64)
	int *d_ur_i, *d_ur_j;         // strict U rows
	int *d_lr_i, *d_lr_j;         // strict L rows (transpose of the column storage)
	double *d_ur_v, *d_lr_v;      // FP64 strict values
	float *d_ur_f, *d_lr_f;       // FP32 strict values
	int nnz_strict;
	int *d_perm;                  // rows by (forward-solve level, index): claim order of the solves
	bsg_sell sl, su;              // SELL-32 strict L / U rows (Jacobi sweeps), FP64 or FP32
	int levels_l, levels_u;       // dependency depth
	double density, density2;
	// transposed solves (U^T: the L-row pattern with U's values; L^T: U's
	// pattern with L's values), built on first use for ILU2 factors
	int has_t;
	double *d_utr_v;
	float *d_utr_f, *d_l_f;
	bsg_sell slt, sut;
	// block factor (k_bfact.cu): nb block rows, nnz = blocks; 3x3 column-major
	// blocks, pivot block first; the strict parts' point rows live in
	// d_lr_* / d_ur_* and sl / su, the diagonal action of the solves in
	// d_bdl (L_ii^T) / d_bdu (U_ii)
	int nb;
	int *d_bia, *d_bja;
	double *d_bl, *d_bu;
	double *d_bdl, *d_bdu, *d_ones;
	bsg_bsell bsl, bsu;           // block SELL copies of the strict L / U block rows (sweeps)
	// two interleaved iterates of the several-vector block sweeps, grown on
	// first use outside graph capture
	double *d_swscr;
	size_t swscr_n;
};

// ---- launch accounting ------------------------------------------------------
// Every kernel launch of the library adds to this process-wide counter
// (bsg_launch_count() in the C ABI), so a benchmark can state how many of
// its own kernels ran in a timed region.
extern unsigned long long g_bsg_launches;
#define BSG_COUNT(k) (g_bsg_launches += (unsigned long long)(k))

// ---- internal entry points shared between translation units --------------
int bsg_prepare_upper(bsg_mat *m);                       // builds d_iu/d_ju/d_al/d_au/d_it/d_jt
int bsg_spmv_launch(const bsg_mat *m, const double *x, double *y, cudaStream_t s);
int bsg_dot_launch(bsg_ctx *c, int n, const double *x, const double *y, double *d_out);
int bsg_fact_run(bsg_ctx *c, bsg_mat *m, int kind, const bsg_param *p, bsg_fct **out);
int bsg_trisolve_launch(bsg_ctx *c, const bsg_fct *f, int lower, int mode, int nsweeps, const double *x, double *y,
                        double *work);
// Solve with U^T (which 0) or L^T (which 1), the transposed preconditioner of
// the two-sided Lanczos; builds the transposed forms on first use.
int bsg_trisolve_t_launch(bsg_ctx *c, bsg_fct *f, int which, int mode, int nsweeps, const double *x, double *y,
                          double *work);
int bsg_check_devstat(bsg_ctx *c);
// block ILU2 / IC2 of a 3x3 block matrix (k_bfact.cu) and its solves
int bsg_bfact_run(bsg_ctx *c, bsg_mat *m, int sym, const bsg_param *p, bsg_fct **out);
int bsg_bfact_make_fp32(bsg_fct *f);
int bsg_btrisolve_launch(bsg_ctx *c, const bsg_fct *f, int lower, int mode, int nsweeps, const double *x, double *y,
                         double *work);
// nr triangular solves with one factor, vectors at stride n (work: n nr
// doubles); sweeps read the factor once for up to 8 vectors.
int bsg_trisolve_multi(bsg_ctx *c, const bsg_fct *f, int lower, int mode, int nsweeps, int nr, const double *x,
                       double *y, double *work);
int bsg_btrisolve_multi(bsg_ctx *c, const bsg_fct *f, int lower, int mode, int nsweeps, int nr, const double *x,
                        double *y, double *work);
// Strict upper part of a CSR pattern transposed: for every column, the rows
// above it that hold an entry there (k_format.cu).
int bsg_strict_transpose(bsg_ctx *c, int n, const int *ia, const int *ja, int nnz, int **it_o, int **jt_o,
                         int **perm_o, int *nnz_o);
// Block IC2 / ILU2 rows with the dynamic schedule (k_fact.cu).
int bsg_bfact_dyn(bsg_ctx *c, int nb, int sym, const bsg_param *p, const int *bia, const int *bja, int nnzb,
                  const double *bal, const double *bau, const double *scll, const double *sclu, const double *diagg,
                  int **ig_o, int **jg_o, double **gl_o, double **gu_o, unsigned long long *nstored);
