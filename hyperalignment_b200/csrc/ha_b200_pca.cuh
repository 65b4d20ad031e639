// ha_b200_pca.cuh -- searchlight PCA template (src/hyperalignment/searchlight.py:215-236 with
// compute_template(kind="pca", max_npc=n, common_topography=True, demean=False),
// src/hyperalignment/local_template.py:224-248, :72-78, :11-53), float64 throughout.
//
// Per searchlight s with vertices sl (n of them, n <= nt) and ns subjects D_j (nt x nv):
//   X = [D_1[:, sl], ..., D_ns[:, sl]]                     nt x ns n
//   the top n singular pairs of X from the smaller Gram (m = min(nt, ns n) <= 512):
//     time side   (m = nt):   X X^T = U diag(lambda) U^T,   tmpl = U_n diag(sqrt(lambda_n)) / sqrt(ns)
//     vertex side (m = ns n): X^T X = W diag(lambda) W^T,   tmpl = X W_n / sqrt(ns)
//   both by the pivoted Cholesky factor of the Gram and the eigenvector-mode Jacobi (k_pchol,
//   k_jacobi); then M = sum_j D_j[:, sl], R = polar(tmpl^T M) by the float64 Jacobi polar, and
//   template[:, sl] += (tmpl R) diag(w_s) with the searchlight weights, reduced per vertex in
//   searchlight order.
// tmpl R depends only on the top-n singular subspace of X (signs and rotations inside a degenerate
// eigenspace cancel in tmpl polar(tmpl^T M)), so this exact route agrees with the reference's
// randomized SVD wherever that subspace is separated from the rest.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ha_b200_kernels.cuh"

namespace hab200 {

constexpr int kPcaMaxM = 512;  // Gram order limit (the pivoted Cholesky's shared rank arrays)

// Per-searchlight scratch of the PCA template (float64 elements from the searchlight's base):
// tmpl (nt x n), M (nt x n), then a work area that first holds the gathered X (nt x m) and the
// selected eigenvectors (m x n, vertex side) and finally C = tmpl R (nt x n).  All column-major.
struct PcaLayout {
	int64_t tmpl, M, work, wsel, total;
	__host__ __device__ static PcaLayout make(int nt, int n, int m, bool vertex_side) {
		PcaLayout L;
		const int64_t tn = (int64_t)nt * n;
		L.tmpl = 0;
		L.M = tn;
		L.work = 2 * tn;
		L.wsel = L.work + (int64_t)nt * m;
		const int64_t w = vertex_side ? (int64_t)nt * m + (int64_t)m * n : tn;
		L.total = (L.work + (w > tn ? w : tn) + 31) & ~(int64_t)31;
		return L;
	}
};

// Column offsets of X: column k = j n + a is subject j's vertex sl[a].
__device__ __forceinline__ int64_t pca_col(const int32_t *sl, int n, int64_t plane, int nt, int k) {
	const int j = k / n;
	return (int64_t)j * plane + (int64_t)sl[k - j * n] * nt;
}

// The Gram of every searchlight of a batch into the V scratch at wm.aofs (m x m, leading dimension
// m, wm.n = m): X X^T (m = nt, reduction over the ns n columns) or X^T X (m = ns n < nt, reduction
// over time).  64 x 64 output tiles, the reduction staged KT at a time, loads along time.
template <int KT>
__global__ void __launch_bounds__(256) k_pca_gram(const SlWork *__restrict__ wm, const int32_t *__restrict__ sl_idx,
                                                  const int32_t *__restrict__ off, const double *__restrict__ D,
                                                  int ns, int nt, int nv, double *__restrict__ Gscr) {
	const SlWork w = wm[blockIdx.x];
	const int n = off[w.s + 1] - off[w.s];
	const int m = w.n;
	const bool tside = (m == nt);
	const int32_t *sl = sl_idx + off[w.s];
	double *G = Gscr + w.aofs;
	const int64_t plane = (int64_t)nt * nv;
	const int K = tside ? ns * n : nt;  // reduction length
	__shared__ double xs[KT][64 + 1];
	__shared__ double zs[KT][64 + 1];
	__shared__ int64_t cofs[kPcaMaxM];  // vertex side: the m column offsets; time side: KT of them
	const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
	if (!tside)
		for (int k = threadIdx.x; k < m; k += blockDim.x) cofs[k] = pca_col(sl, n, plane, nt, k);
	for (int i0 = 0; i0 < m; i0 += 64) {
		for (int j0 = 0; j0 < m; j0 += 64) {
			double acc[4][4];
#pragma unroll
			for (int a = 0; a < 4; a++)
#pragma unroll
				for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
			for (int k0 = 0; k0 < K; k0 += KT) {
				__syncthreads();
				if (tside) {
					if (threadIdx.x < KT) {
						const int k = k0 + threadIdx.x;
						cofs[threadIdx.x] = k < K ? pca_col(sl, n, plane, nt, k) : -1;
					}
					__syncthreads();
					// xs[kk][r] = X(i0 + r, k0 + kk): consecutive threads read consecutive times
					for (int e = threadIdx.x; e < KT * 64; e += 256) {
						const int kk = e >> 6, r = e & 63;
						const int64_t c = cofs[kk];
						const int ti = i0 + r, tj = j0 + r;
						xs[kk][r] = (c >= 0 && ti < m) ? D[c + ti] : 0.0;
						zs[kk][r] = (c >= 0 && tj < m) ? D[c + tj] : 0.0;
					}
				} else {
					// xs[kk][r] = X(k0 + kk, i0 + r): consecutive threads read consecutive times
					for (int e = threadIdx.x; e < KT * 64; e += 256) {
						const int r = e / KT, kk = e - r * KT;
						const int t = k0 + kk, pi = i0 + r, pj = j0 + r;
						xs[kk][r] = (t < K && pi < m) ? D[cofs[pi] + t] : 0.0;
						zs[kk][r] = (t < K && pj < m) ? D[cofs[pj] + t] : 0.0;
					}
				}
				__syncthreads();
#pragma unroll 4
				for (int kk = 0; kk < KT; kk++) {
					double a[4], b[4];
#pragma unroll
					for (int q = 0; q < 4; q++) {
						a[q] = xs[kk][ty + 16 * q];
						b[q] = zs[kk][tx + 16 * q];
					}
#pragma unroll
					for (int p = 0; p < 4; p++)
#pragma unroll
						for (int q = 0; q < 4; q++) acc[p][q] += a[p] * b[q];
				}
			}
#pragma unroll
			for (int p = 0; p < 4; p++) {
				const int i = i0 + ty + 16 * p;
				if (i >= m) continue;
#pragma unroll
				for (int q = 0; q < 4; q++) {
					const int j = j0 + tx + 16 * q;
					if (j < m) G[(int64_t)j * m + i] = acc[p][q];
				}
			}
		}
	}
}

// The template of every searchlight of a batch and B = tmpl^T M, the matrix whose polar factor
// rotates it.  Eigenvectors (V scratch at wm.aofs, column-major, leading dimension m) and
// eigenvalues (uv + wm.uvofs) from the eigenvector-mode Jacobi; the n largest eigenvalues (ties:
// the lower column) are taken in decreasing order.  wm and wn (the polar work items) are in slot
// order; B (n x n) goes to the polar solve's A region at wn.aofs with the padding columns of its
// block layout zero.
__global__ void __launch_bounds__(256) k_pca_tmpl(const SlWork *__restrict__ wm, const SlWork *__restrict__ wn,
                                                  const int32_t *__restrict__ sl_idx, const double *__restrict__ D,
                                                  int ns, int nt, int nv, const double *__restrict__ Vscr,
                                                  const double *__restrict__ uv, const int64_t *__restrict__ pofs,
                                                  double *__restrict__ Pscr, double *__restrict__ Ascr) {
	const SlWork em = wm[blockIdx.x];
	const SlWork ep = wn[blockIdx.x];
	const int n = ep.n, m = em.n;
	const bool tside = (m == nt);
	const int32_t *sl = sl_idx + ep.sofs;
	const double *U = Vscr + em.aofs;
	const double *lam = uv + em.uvofs;
	const PcaLayout L = PcaLayout::make(nt, n, m, !tside);
	double *base = Pscr + pofs[ep.slot];
	double *tmpl = base + L.tmpl;
	double *M = base + L.M;
	__shared__ int sel[kPcaMaxM];
	__shared__ double ps[16][65], qs[16][65];
	for (int c = threadIdx.x; c < m; c += blockDim.x) {
		const double lc = lam[c];
		int rank = 0;
		for (int c2 = 0; c2 < m; c2++) {
			const double l2 = lam[c2];
			rank += (l2 > lc || (l2 == lc && c2 < c)) ? 1 : 0;
		}
		if (rank < n) sel[rank] = c;
	}
	__syncthreads();
	const double inv_ns = rsqrt((double)ns);
	const int64_t plane = (int64_t)nt * nv;
	for (int64_t e = threadIdx.x; e < (int64_t)nt * n; e += blockDim.x) {
		const int r = (int)(e / nt), t = (int)(e - (int64_t)r * nt);
		if (tside) {
			const int c = sel[r];
			tmpl[e] = U[(int64_t)c * m + t] * sqrt(fmax(lam[c], 0.0)) * inv_ns;
		}
		double s = 0.0;
		for (int j = 0; j < ns; j++) s += D[(int64_t)j * plane + (int64_t)sl[r] * nt + t];
		M[e] = s;
	}
	if (!tside) {
		// tmpl = X W_sel / sqrt(ns): X gathered (nt x m) and the selected eigenvectors (m x n)
		double *Xg = base + L.work;
		double *Ws = base + L.wsel;
		for (int64_t e = threadIdx.x; e < (int64_t)nt * m; e += blockDim.x) {
			const int k = (int)(e / nt), t = (int)(e - (int64_t)k * nt);
			Xg[e] = D[pca_col(sl, n, plane, nt, k) + t];
		}
		for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) {
			const int r = (int)(e / m), k = (int)(e - (int64_t)r * m);
			Ws[e] = U[(int64_t)sel[r] * m + k];
		}
		__syncthreads();
		// tmpl(t, r) = sum_k Xg(t, k) Ws(k, r) / sqrt(ns)
		GemmArgs<double, double> g;
		g.M = nt; g.N = n; g.K = m;
		g.P = Xg; g.pk = nt; g.pi = 1;
		g.Q = Ws; g.qk = 1; g.qj = m;
		g.d = nullptr; g.alpha = inv_ns;
		g.E = nullptr; g.ei = 0; g.ej = 0; g.beta = 0.0;
		g.C = tmpl; g.ci = 1; g.cj = nt;
		block_gemm(g, ps, qs);
	}
	__syncthreads();
	// B(r, c) = sum_t tmpl(t, r) M(t, c)
	GemmArgs<double, double> g;
	g.M = n; g.N = n; g.K = nt;
	g.P = tmpl; g.pk = 1; g.pi = nt;
	g.Q = M; g.qk = 1; g.qj = nt;
	g.d = nullptr; g.alpha = 1.0;
	g.E = nullptr; g.ei = 0; g.ej = 0; g.beta = 0.0;
	double *A = Ascr + ep.aofs;
	g.C = A; g.ci = 1; g.cj = n;
	block_gemm(g, ps, qs);
	const int ncol = ep.nblk * ep.bsz;
	for (int64_t e = (int64_t)n * n + threadIdx.x; e < (int64_t)n * ncol; e += blockDim.x) A[e] = 0.0;
}

// C = tmpl R (nt x n, into the work area) from the polar factor R (float, column-major in the T
// scratch at wn.tofs), R staged as float64 in the M block.  wn in slot order; m of the slot's
// Gram from wm (slot order).
__global__ void __launch_bounds__(256) k_pca_contrib(const SlWork *__restrict__ wm, const SlWork *__restrict__ wn,
                                                     const float *__restrict__ Tscr, int nt,
                                                     const int64_t *__restrict__ pofs, double *__restrict__ Pscr) {
	const SlWork ep = wn[blockIdx.x];
	const int n = ep.n, m = wm[blockIdx.x].n;
	const PcaLayout L = PcaLayout::make(nt, n, m, m != nt);
	double *base = Pscr + pofs[ep.slot];
	const double *tmpl = base + L.tmpl;
	double *Rd = base + L.M;  // M is no longer needed
	double *C = base + L.work;
	const float *R = Tscr + ep.tofs;
	__shared__ double ps[16][65], qs[16][65];
	for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) Rd[e] = (double)R[e];
	__syncthreads();
	// C(t, j) = sum_i tmpl(t, i) R(i, j)
	GemmArgs<double, double> g;
	g.M = nt; g.N = n; g.K = n;
	g.P = tmpl; g.pk = nt; g.pi = 1;
	g.Q = Rd; g.qk = 1; g.qj = n;
	g.d = nullptr; g.alpha = 1.0;
	g.E = nullptr; g.ei = 0; g.ej = 0; g.beta = 0.0;
	g.C = C; g.ci = 1; g.cj = nt;
	block_gemm(g, ps, qs);
}

// template[:, v] += sum over the searchlights s of [s_lo, s_hi) holding v (member a), in
// searchlight order, of w_s[a] C_s[:, a] (w = 1 without weights).  One CTA per vertex, threads
// over time; pofs and the Gram orders mg are per slot s - s_lo.
__global__ void __launch_bounds__(256) k_pca_reduce(const int64_t *__restrict__ vl_ptr, const int2 *__restrict__ vl_ent,
                                                    const int32_t *__restrict__ off, const double *__restrict__ wts,
                                                    const int64_t *__restrict__ pofs, const int32_t *__restrict__ mg,
                                                    const double *__restrict__ Pscr, int nt, int s_lo, int s_hi,
                                                    double *__restrict__ tpl) {
	const int v = blockIdx.x;
	double *out = tpl + (int64_t)v * nt;
	for (int64_t k = vl_ptr[v]; k < vl_ptr[v + 1]; k++) {
		const int2 e = vl_ent[k];
		if (e.x < s_lo || e.x >= s_hi) continue;
		const int n = off[e.x + 1] - off[e.x];
		const double wv = wts ? wts[off[e.x] + e.y] : 1.0;
		const PcaLayout L = PcaLayout::make(nt, n, mg[e.x - s_lo], mg[e.x - s_lo] != nt);
		const double *C = Pscr + pofs[e.x - s_lo] + L.work + (int64_t)e.y * nt;
		for (int t = threadIdx.x; t < nt; t += blockDim.x) out[t] += wv * C[t];
	}
}

}  // namespace hab200
