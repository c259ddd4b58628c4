// 3 x 3 block helpers (column-major: entry (r, c) at r + 3 c, as CSMatrixRS
// keeps its blocks), shared by the block factorisations.
#pragma once

namespace {

// out = p q with p given by strides: p(r, k) at p[r * pr + k * pc]; q(k, c)
// at q[k * qr + c * qc]; sums in k order from zero
__device__ __forceinline__ void mm3(const double *p, int pr, int pc, const double *q, int qr, int qc, double *out) {
#pragma unroll
	for (int r = 0; r < 3; r++)
#pragma unroll
		for (int c = 0; c < 3; c++) {
			double s = 0.0;
#pragma unroll
			for (int k = 0; k < 3; k++) s += p[r * pr + k * pc] * q[k * qr + c * qc];
			out[r + 3 * c] = s;
		}
}

// A = U diag(s) V^T of a 3 x 3 matrix (column-major), s descending, U and V
// orthogonal: one-sided Jacobi (Hestenes), rotating column pairs of W = A V
// until they are orthogonal; U = the normalised columns of W, completed to an
// orthonormal basis (Gram-Schmidt of unit vectors) where a singular value
// vanishes.
__device__ void svd3(const double *a, double *u, double *s, double *v) {
	double w[9], vw[9];
	for (int k = 0; k < 9; k++) {
		w[k] = a[k];
		vw[k] = (k % 4) == 0 ? 1.0 : 0.0;
	}
	for (int sweep = 0; sweep < 30; sweep++) {
		double off2 = 0.0; // largest ga^2 / (al be) of the sweep
		for (int pq = 0; pq < 3; pq++) {
			const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
			double al = 0.0, be = 0.0, ga = 0.0;
			for (int r = 0; r < 3; r++) {
				al += w[r + 3 * p] * w[r + 3 * p];
				be += w[r + 3 * q] * w[r + 3 * q];
				ga += w[r + 3 * p] * w[r + 3 * q];
			}
			// columns already orthogonal to 1e-16 relative: no rotation (the
			// test on squares keeps a square root and a division off the chain)
			const double ab = al * be, g2 = ga * ga;
			if (ab == 0.0 || g2 <= 1e-32 * ab) continue;
			off2 = fmax(off2, g2 / ab);
			const double zeta = (be - al) / (2.0 * ga);
			const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
			const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
			for (int r = 0; r < 3; r++) {
				const double wp = w[r + 3 * p], wq = w[r + 3 * q];
				w[r + 3 * p] = cs * wp - sn * wq;
				w[r + 3 * q] = sn * wp + cs * wq;
				const double vp = vw[r + 3 * p], vq = vw[r + 3 * q];
				vw[r + 3 * p] = cs * vp - sn * vq;
				vw[r + 3 * q] = sn * vp + cs * vq;
			}
		}
		if (off2 <= 1e-30) break;
	}
	double sv[3];
	for (int c = 0; c < 3; c++) sv[c] = sqrt(w[3 * c] * w[3 * c] + w[1 + 3 * c] * w[1 + 3 * c] + w[2 + 3 * c] * w[2 + 3 * c]);
	int o[3] = {0, 1, 2}; // descending order
	if (sv[o[0]] < sv[o[1]]) { const int t = o[0]; o[0] = o[1]; o[1] = t; }
	if (sv[o[1]] < sv[o[2]]) { const int t = o[1]; o[1] = o[2]; o[2] = t; }
	if (sv[o[0]] < sv[o[1]]) { const int t = o[0]; o[0] = o[1]; o[1] = t; }
	const double smax = sv[o[0]];
	int good[3];
	for (int c = 0; c < 3; c++) {
		const int k = o[c];
		s[c] = sv[k];
		good[c] = sv[k] > 1e-300 && sv[k] > 1e-14 * smax;
		for (int r = 0; r < 3; r++) {
			u[r + 3 * c] = good[c] ? w[r + 3 * k] / sv[k] : 0.0;
			v[r + 3 * c] = vw[r + 3 * k];
		}
	}
	for (int c = 0; c < 3; c++) {
		if (good[c]) continue;
		for (int e = 0; e < 3; e++) {
			double x[3] = {e == 0 ? 1.0 : 0.0, e == 1 ? 1.0 : 0.0, e == 2 ? 1.0 : 0.0};
			for (int d = 0; d < 3; d++) {
				if (d == c || !good[d]) continue;
				const double pr = u[3 * d] * x[0] + u[1 + 3 * d] * x[1] + u[2 + 3 * d] * x[2];
				for (int r = 0; r < 3; r++) x[r] -= pr * u[r + 3 * d];
			}
			const double nx = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
			if (nx > 0.5) {
				for (int r = 0; r < 3; r++) u[r + 3 * c] = x[r] / nx;
				good[c] = 1;
				break;
			}
		}
	}
}

} // namespace
