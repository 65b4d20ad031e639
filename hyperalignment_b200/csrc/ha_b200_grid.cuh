// ha_b200_grid.cuh -- per-searchlight ridge grid search with cross-validated ensembles.  The grid
// kernels are templated on the arithmetic type Real: double for the float64 search, float for the
// plain FP32 form (inputs, alphas and the output betas stay float64).
//
// Composition of the reference's ha_ridge_grid (csrc/ha_ridge.c:97-227) and ha_ensemble_ridge
// (csrc/ha_ridge.c:229-345) applied to every searchlight: X = X[:, sl] and the searchlight's n
// target columns Y[:, sl], with the prediction cost summed over the targets (one winner per
// searchlight).  For CV model m with training rows tr_m (bootstrap, duplicates kept) and test
// rows te_m:
//   G = X_tr^T X_tr = V diag(lambda) V^T   (X_tr = U diag(s) V^T, lambda = s^2),
//   Q = V^T X_tr^T Y_tr,  component k contributes v_k q_k^T / (alpha + lambda_k)
// which is the reference's V diag(s / (alpha + s^2)) U^T Y per component.  Components are taken
// in decreasing lambda (the SVD's order), the PC chunks [npcs[p-1], npcs[p]) are clipped at
// K = min(rows, n) and summed cumulatively over p (csrc/ha_ridge.c:185-220, also for non-monotone
// npcs).  Test predictions of model m are X_te V diag(c) Q; every tested time point averages the
// predictions of the models that test it (csrc/ha_ridge.c:262-303), and the cost of a grid point
// is the squared error over all time points and targets (csrc/ha_ridge.c:305-319; untested time
// points predict zero).  The winner is the first grid point with the smallest cost (g = a * n_npcs
// + p, csrc/ha_ridge.c:322-327); its model-averaged beta is written like the ridge solve's.
#pragma once

#include "ha_b200_kernels.cuh"

namespace hab200 {

constexpr int kGridMaxN = 512;  // searchlight size limit of the grid kernels (shared rank arrays)

struct GridModel {
	int32_t tr_ofs, tr_n;  // training rows: rows[tr_ofs .. tr_ofs + tr_n)
	int32_t te_ofs, te_n;  // test rows: rows[te_ofs .. te_ofs + te_n); union positions tpos[te_ofs ..]
};

struct GridParams {
	int models, mte, ntu, n_alphas, n_npcs, nt, n_untested;
	const double *alphas;      // n_alphas
	const int32_t *npcs;       // n_npcs
	const GridModel *mdl;      // models
	const int32_t *rows;       // concatenated training and test row lists
	const int32_t *tpos;       // per test-list entry: position in the union of tested rows
	const double *winv;        // per union position: 1 / (number of models that test it)
	const int32_t *urows;      // union of tested rows, ntu
	const int32_t *untested;   // rows no model tests, n_untested
	const int64_t *gbase;      // per work slot: base offset of the searchlight's grid scratch
};

// Per-searchlight layout of the grid scratch (Real elements from the searchlight's base).
// Per model: V and Q with components in decreasing-lambda order (V column r = r-th component,
// Q row r), lambda in that order and E = X_te V (mte x n, column-major, ld mte).  Per alpha (the
// grid evaluation runs one CTA per searchlight and alpha): the models' cumulative test predictions
// Pm (models x mte x n) and the averaged predictions P on the union of tested rows (ntu x n,
// column-major; alpha 0's block is also the n x n beta accumulator of the winner).  Yu holds the
// targets on the tested rows, C the cross-covariance of the current model.
struct GridLayout {
	int64_t C, Vst, Qst, Lst, Est, Yu, Xte, cost, PA, pa_stride, total;
	__host__ __device__ static GridLayout make(int n, int models, int mte, int ntu, int n_alphas, int grid) {
		GridLayout L;
		const int64_t n2 = (int64_t)n * n, mn = (int64_t)mte * n;
		int64_t o = 0;
		L.C = o; o += n2;
		L.Vst = o; o += (int64_t)models * n2;
		L.Qst = o; o += (int64_t)models * n2;
		L.Lst = o; o += (int64_t)models * n;
		L.Est = o; o += (int64_t)models * mn;
		L.Yu = o; o += (int64_t)ntu * n;
		L.Xte = o; o += mn;
		L.cost = o; o += grid;
		L.pa_stride = (((int64_t)models * mn + (int64_t)(ntu > n ? ntu : n) * n) + 31) & ~(int64_t)31;
		L.PA = (o + 31) & ~(int64_t)31;
		o = L.PA + (int64_t)n_alphas * L.pa_stride;
		L.total = (o + 31) & ~(int64_t)31;
		return L;
	}
	// per-alpha blocks: Pm at PA + a * pa_stride, P right after it
	__host__ __device__ int64_t Pm(int a) const { return PA + (int64_t)a * pa_stride; }
	__host__ __device__ int64_t P(int a, int models, int mte, int n) const {
		return Pm(a) + (int64_t)models * mte * n;
	}
};

__device__ __forceinline__ GridLayout grid_layout(const GridParams &gp, int n) {
	return GridLayout::make(n, gp.models, gp.mte, gp.ntu, gp.n_alphas, gp.n_alphas * gp.n_npcs);
}

// A_s = X[rows, sl]^T Z[rows, sl] (Z = X for the Gram, Y for the cross-covariance) over one row
// list with duplicates, in Real, the k_xcov tiling with gathered rows.  Output column-major:
// mode 0 at Ascr + w.aofs with ncol columns (padding columns zero), mode 1 into the searchlight's
// grid C block, mode 2 at Ascr + w.tofs (n x n).
template <int KT, typename Real>
__global__ void __launch_bounds__(256) k_xcov_rows(const SlWork *__restrict__ work, const int32_t *__restrict__ sl_idx,
                                                   const double *__restrict__ X, const double *__restrict__ Z, int nt,
                                                   const int32_t *__restrict__ rows, int nrows, Real *__restrict__ Ascr,
                                                   Real *__restrict__ Gscr, GridParams gp, int mode) {
	const SlWork w = work[blockIdx.x];
	const int n = w.n;
	const int ncol = w.nblk * w.bsz;
	const int32_t *sl = sl_idx + w.sofs;
	Real *A = mode == 1 ? Gscr + gp.gbase[w.slot] + grid_layout(gp, n).C : Ascr + (mode == 2 ? w.tofs : w.aofs);
	__shared__ Real xs[KT][64 + 1];
	__shared__ Real zs[KT][64 + 1];
	__shared__ int32_t vi[64], vj[64];
	__shared__ int32_t rt[KT];
	const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
	for (int i0 = 0; i0 < n; i0 += 64) {
		for (int j0 = 0; j0 < n; j0 += 64) {
			__syncthreads();
			if (threadIdx.x < 64) {
				const int i = i0 + threadIdx.x;
				vi[threadIdx.x] = (i < n) ? sl[i] : -1;
			} else if (threadIdx.x < 128) {
				const int j = j0 + threadIdx.x - 64;
				vj[threadIdx.x - 64] = (j < n) ? sl[j] : -1;
			}
			Real acc[4][4];
#pragma unroll
			for (int a = 0; a < 4; a++)
#pragma unroll
				for (int b = 0; b < 4; b++) acc[a][b] = Real(0);
			for (int t0 = 0; t0 < nrows; t0 += KT) {
				__syncthreads();
				if (threadIdx.x < KT) rt[threadIdx.x] = (t0 + threadIdx.x < nrows) ? rows[t0 + threadIdx.x] : -1;
				__syncthreads();
				for (int e = threadIdx.x; e < 64 * KT; e += 256) {
					const int r = e / KT, t = e - r * KT;
					const int tt = rt[t];
					const int v = vi[r], u = vj[r];
					xs[t][r] = (v >= 0 && tt >= 0) ? (Real)X[(int64_t)v * nt + tt] : Real(0);
					zs[t][r] = (u >= 0 && tt >= 0) ? (Real)Z[(int64_t)u * nt + tt] : Real(0);
				}
				__syncthreads();
#pragma unroll 4
				for (int t = 0; t < KT; t++) {
					Real a[4], b[4];
#pragma unroll
					for (int q = 0; q < 4; q++) {
						a[q] = xs[t][ty + 16 * q];
						b[q] = zs[t][tx + 16 * q];
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
				if (i >= n) continue;
#pragma unroll
				for (int q = 0; q < 4; q++) {
					const int j = j0 + tx + 16 * q;
					if (j < n) A[(int64_t)j * n + i] = acc[p][q];
				}
			}
		}
	}
	if (mode == 0)
		for (int64_t e = (int64_t)n * n + threadIdx.x; e < (int64_t)n * ncol; e += 256) A[e] = Real(0);
}

// Pivoted Cholesky G = sum_k r_k r_k^T (pivot = largest remaining diagonal, ties to the smaller
// vertex index), stopped when the largest remaining diagonal is at most n * eps * max(diag G).
// Panels of kPcholNb columns: inside a panel each new column is corrected by the panel's earlier
// columns (kept in shared memory, indexed by vertex) and the diagonal is updated per column; the
// trailing Schur complement in G (column-major, ld n, at Gscr + w.aofs) is updated once per panel.
// r_k (original vertex order, zero at earlier pivots) becomes column k of Rt (ld n, ncol columns,
// the rest zero), so G = Rt Rt^T; the number of columns (the numerical rank) goes to the stats.
// The one-sided Jacobi rotations then run on Rt: its columns come in decreasing, graded norms and
// only rank(G) of them are nonzero, which takes fewer sweeps than rotating G itself and needs no
// accumulated rotations.  Dynamic shared memory: kPcholNb * 32 * RPL elements (>= kPcholNb * n).
constexpr int kPcholNb = 16;

template <typename Real>
__global__ void __launch_bounds__(256) k_pchol(const SlWork *__restrict__ work, Real *__restrict__ Gscr,
                                               Real *__restrict__ Rscr, SlStats *__restrict__ stats) {
	extern __shared__ __align__(16) unsigned char pan_raw[];
	Real *pan = reinterpret_cast<Real *>(pan_raw);  // [kPcholNb][n], indexed by vertex
	__shared__ int rem[kGridMaxN];                  // vertices not yet pivoted (positions 0 .. m-1)
	__shared__ Real dg[kGridMaxN];                // current Schur diagonal, by vertex
	__shared__ Real rv[32];
	__shared__ int ri[32], rpos[32];
	__shared__ Real s_tol, s_piv;
	__shared__ int s_pos;
	const SlWork w = work[blockIdx.x];
	const int n = w.n, ncol = w.nblk * w.bsz;
	Real *S = Gscr + w.aofs;
	Real *Rt = Rscr + w.aofs;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	for (int i = threadIdx.x; i < n; i += blockDim.x) {
		rem[i] = i;
		dg[i] = S[(int64_t)i * n + i];
	}
	for (int64_t e = threadIdx.x; e < (int64_t)n * ncol; e += blockDim.x) Rt[e] = Real(0);
	__syncthreads();
	{
		Real mx = Real(0);
		for (int i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, dg[i]);
		for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
		if (lane == 0) rv[warp] = mx;
		__syncthreads();
		if (threadIdx.x == 0) {
			Real t = Real(0);
			for (int q = 0; q < nwarp; q++) t = fmax(t, rv[q]);
			s_tol = (Real)n * Eps<Real>::v() * t;
		}
		__syncthreads();
	}
	int m = n, k = 0;
	bool stop = false;
	while (k < n && !stop) {
		int nbk = 0;  // columns of the current panel
		for (; nbk < kPcholNb && k < n; nbk++, k++) {
			// pivot: largest remaining diagonal (ties: smaller vertex index)
			Real bv = Real(-1);
			int bi = 0x7fffffff, bpos = 0;
			for (int a = threadIdx.x; a < m; a += blockDim.x) {
				const int v = rem[a];
				const Real d = dg[v];
				if (d > bv || (d == bv && v < bi)) { bv = d; bi = v; bpos = a; }
			}
			for (int o = 16; o > 0; o >>= 1) {
				const Real ov = __shfl_xor_sync(0xffffffffu, bv, o);
				const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
				const int op = __shfl_xor_sync(0xffffffffu, bpos, o);
				if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; bpos = op; }
			}
			if (lane == 0) { rv[warp] = bv; ri[warp] = bi; rpos[warp] = bpos; }
			__syncthreads();
			if (threadIdx.x == 0) {
				Real v = rv[0];
				int vi = ri[0], pos = rpos[0];
				for (int q = 1; q < nwarp; q++)
					if (rv[q] > v || (rv[q] == v && ri[q] < vi)) { v = rv[q]; vi = ri[q]; pos = rpos[q]; }
				s_piv = v;
				s_pos = pos;
			}
			__syncthreads();
			if (!(s_piv > s_tol)) {
				stop = true;
				break;
			}
			const int a = s_pos, p = rem[a];
			const Real rp = sqrt(s_piv);
			Real *rk = pan + (int64_t)nbk * n;
			for (int b = threadIdx.x; b < m; b += blockDim.x) {
				const int v = rem[b];
				Real r = rp;
				if (b != a) {
					Real x = S[(int64_t)p * n + v];
					for (int j = 0; j < nbk; j++) x -= pan[(int64_t)j * n + p] * pan[(int64_t)j * n + v];
					r = x / rp;
					dg[v] -= r * r;
				}
				rk[v] = r;
				Rt[(int64_t)k * n + v] = r;
			}
			__syncthreads();
			if (threadIdx.x == 0) rem[a] = rem[m - 1];
			m--;
			__syncthreads();
		}
		if (stop || m == 0) break;
		// Schur complement on the remaining vertices with the panel's nbk columns
		for (int c = warp; c < m; c += nwarp) {
			const int u = rem[c];
			Real *Su = S + (int64_t)u * n;
			for (int b = lane; b < m; b += 32) {
				const int v = rem[b];
				Real acc = Real(0);
				for (int j = 0; j < nbk; j++) acc += pan[(int64_t)j * n + v] * pan[(int64_t)j * n + u];
				Su[v] -= acc;
			}
		}
		__syncthreads();
	}
	if (threadIdx.x == 0) stats[w.slot].ncols = max(k, 1);
}

// Rank of every component by decreasing lambda (ties by index): order[r] = k.
__device__ __forceinline__ void rank_desc(const double *lam, int n, int *order) {
	for (int k = threadIdx.x; k < n; k += blockDim.x) {
		const double lk = lam[k];
		int r = 0;
		for (int l = 0; l < n; l++) {
			const double ll = lam[l];
			r += (ll > lk) || (ll == lk && l < k);
		}
		order[r] = k;
	}
}

// One CV model of every searchlight: the eigenvectors (column-major, ld n) in the V scratch and
// lambda in the u/v buffer come from the Jacobi kernel (in Real) in eigenvector mode run on the
// pivoted Cholesky factor of the Gram; C is in the grid scratch.
// Stores V, lambda in decreasing-lambda order, Q = V^T C and E = X_te V for the model.
template <typename Real>
__global__ void __launch_bounds__(256) k_grid_model(const SlWork *__restrict__ work, const int32_t *__restrict__ sl_idx,
                                                    const double *__restrict__ X, const double *__restrict__ Y,
                                                    const Real *__restrict__ Vscr, const double *__restrict__ uvbuf,
                                                    int model, Real *__restrict__ Gscr, GridParams gp) {
	__shared__ Real ps[16][65], qs[16][65];
	__shared__ int order[kGridMaxN];
	const SlWork w = work[blockIdx.x];
	const int n = w.n;
	const GridLayout L = grid_layout(gp, n);
	Real *base = Gscr + gp.gbase[w.slot];
	const Real *V = Vscr + w.aofs;
	const double *lam = uvbuf + w.uvofs;
	const int32_t *sl = sl_idx + w.sofs;
	const GridModel md = gp.mdl[model];
	const int m = md.te_n;
	const int64_t n2 = (int64_t)n * n, mn = (int64_t)gp.mte * n;
	Real *Vst = base + L.Vst + model * n2;
	Real *Qst = base + L.Qst + model * n2;
	Real *Lst = base + L.Lst + (int64_t)model * n;
	Real *Est = base + L.Est + model * mn;
	Real *Xte = base + L.Xte;
	const Real *C = base + L.C;
	const int32_t *te = gp.rows + md.te_ofs;
	if (model == 0)  // the targets on the tested rows, for the grid evaluation
		for (int64_t e = threadIdx.x; e < (int64_t)gp.ntu * n; e += blockDim.x) {
			const int j = (int)(e / gp.ntu), u = (int)(e - (int64_t)j * gp.ntu);
			base[L.Yu + e] = (Real)Y[(int64_t)sl[j] * gp.nt + gp.urows[u]];
		}
	rank_desc(lam, n, order);
	__syncthreads();
	for (int64_t e = threadIdx.x; e < n2; e += blockDim.x) {
		const int r = (int)(e / n), i = (int)(e - (int64_t)r * n);
		Vst[e] = V[(int64_t)order[r] * n + i];
	}
	for (int r = threadIdx.x; r < n; r += blockDim.x) Lst[r] = (Real)lam[order[r]];
	// test rows of X, column-major by vertex: Xte[v * m + t]
	for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) {
		const int v = (int)(e / m), t = (int)(e - (int64_t)v * m);
		Xte[e] = (Real)X[(int64_t)sl[v] * gp.nt + te[t]];
	}
	__syncthreads();
	GemmArgs<Real, Real> g;
	g.d = nullptr; g.alpha = Real(1); g.E = nullptr; g.ei = 0; g.ej = 0; g.beta = Real(0);
	// Q(r, j) = sum_k Vst(k, r) C(k, j), column-major ld n
	g.M = n; g.N = n; g.K = n;
	g.P = Vst; g.pk = 1; g.pi = n;
	g.Q = C; g.qk = 1; g.qj = n;
	g.C = Qst; g.ci = 1; g.cj = n;
	block_gemm(g, ps, qs);
	if (m > 0) {
		// E(t, r) = sum_v Xte(t, v) Vst(v, r), column-major ld m
		g.M = m; g.N = n; g.K = n;
		g.P = Xte; g.pk = m; g.pi = 1;
		g.Q = Vst; g.qk = 1; g.qj = n;
		g.C = Est; g.ci = 1; g.cj = m;
		block_gemm(g, ps, qs);
	}
}

// First and one-past-last component of PC chunk p of a model with K usable components, or an
// empty range (csrc/ha_ridge.c:187-210).
__device__ __forceinline__ void pc_chunk(const int32_t *npcs, int p, int K, int &r0, int &r1) {
	const int lo = p ? npcs[p - 1] : 0;
	const int hi = npcs[p];
	r0 = lo;
	r1 = lo;
	if (hi - lo > 0 && lo < K) r1 = min(hi, K);
}

// Block-wide sum of one value per thread (256 threads), result in every thread.
template <typename Real>
__device__ __forceinline__ Real grid_block_sum(Real v, Real *red) {
	v = warp_sum(v);
	__syncthreads();
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
	__syncthreads();
	Real tot = Real(0);
	for (int q = 0; q < (int)(blockDim.x >> 5); q++) tot += red[q];
	return tot;
}

// The grid evaluation after all models, one CTA per (searchlight, alpha = blockIdx.y): the models'
// cumulative test predictions over the PC chunks, their average per tested row and the squared
// error over the tested rows and the targets, cost[alpha * n_npcs + p] (without the untested
// rows, which k_grid_final adds).
template <typename Real>
__global__ void __launch_bounds__(256) k_grid_eval(const SlWork *__restrict__ work, Real *__restrict__ Gscr,
                                                   GridParams gp) {
	__shared__ Real ps[16][65], qs[16][65];
	__shared__ Real cval[kGridMaxN];
	__shared__ Real red[32];
	const SlWork w = work[blockIdx.x];
	const int a = blockIdx.y;
	const int n = w.n;
	const GridLayout L = grid_layout(gp, n);
	Real *base = Gscr + gp.gbase[w.slot];
	const int64_t n2 = (int64_t)n * n, mn = (int64_t)gp.mte * n;
	const int ntu = gp.ntu;
	Real *Pma = base + L.Pm(a);
	Real *P = base + L.P(a, gp.models, gp.mte, n);
	const Real *Yu = base + L.Yu;
	Real *cost = base + L.cost;
	const Real al = (Real)gp.alphas[a];
	GemmArgs<Real, Real> g;
	g.alpha = Real(1);
	g.beta = Real(1);
	for (int64_t e = threadIdx.x; e < gp.models * mn; e += blockDim.x) Pma[e] = Real(0);
	__syncthreads();
	for (int p = 0; p < gp.n_npcs; p++) {
		// Pm += E[:, r0:r1] diag(1 / (alpha + lambda)) Q[r0:r1, :] for every model
		for (int mo = 0; mo < gp.models; mo++) {
			const GridModel md = gp.mdl[mo];
			const int m = md.te_n;
			int r0, r1;
			pc_chunk(gp.npcs, p, min(md.tr_n, n), r0, r1);
			if (r1 <= r0 || m == 0) continue;
			const Real *lam = base + L.Lst + (int64_t)mo * n;
			__syncthreads();
			for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) cval[r] = Real(1) / (al + lam[r]);
			__syncthreads();
			const Real *E = base + L.Est + mo * mn;
			const Real *Q = base + L.Qst + mo * n2;
			Real *Pm = Pma + mo * mn;
			g.M = m; g.N = n; g.K = r1 - r0;
			g.P = E + (int64_t)r0 * m; g.pk = m; g.pi = 1;
			g.Q = Q + r0; g.qk = 1; g.qj = n;
			g.d = cval + r0;
			g.E = Pm; g.ei = 1; g.ej = m;
			g.C = Pm; g.ci = 1; g.cj = m;
			block_gemm(g, ps, qs);
		}
		// average over the models that test each row, then the squared error
		__syncthreads();
		for (int64_t e = threadIdx.x; e < (int64_t)ntu * n; e += blockDim.x) P[e] = Real(0);
		for (int mo = 0; mo < gp.models; mo++) {
			const GridModel md = gp.mdl[mo];
			const int m = md.te_n;
			const Real *Pm = Pma + mo * mn;
			const int32_t *tp = gp.tpos + md.te_ofs;
			__syncthreads();
			for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) {
				const int j = (int)(e / m), i = (int)(e - (int64_t)j * m);
				const int u = tp[i];
				P[(int64_t)j * ntu + u] += (Real)gp.winv[u] * Pm[e];
			}
		}
		__syncthreads();
		Real s = Real(0);
		for (int64_t e = threadIdx.x; e < (int64_t)ntu * n; e += blockDim.x) {
			const Real d = Yu[e] - P[e];
			s += d * d;
		}
		s = grid_block_sum(s, red);
		if (threadIdx.x == 0) cost[a * gp.n_npcs + p] = s;
	}
}

// Winner per searchlight (first minimum of the summed cost, csrc/ha_ridge.c:322-327) and its
// model-averaged beta, written float64 in the T layout (row-major for CSR output, column-major for
// CSC), plus the cost row (cost_out may be null) with the untested rows' squared targets added
// (their prediction is zero, csrc/ha_ridge.c:297-319).
template <typename Real>
__global__ void __launch_bounds__(256) k_grid_final(const SlWork *__restrict__ work, const int32_t *__restrict__ sl_idx,
                                                    const double *__restrict__ Y, Real *__restrict__ Gscr,
                                                    GridParams gp, double *__restrict__ Bout, int t_rowmajor,
                                                    int32_t *__restrict__ best_out, double *__restrict__ cost_out) {
	__shared__ Real ps[16][65], qs[16][65];
	__shared__ Real cval[kGridMaxN];
	__shared__ Real red[32];
	__shared__ int best;
	const SlWork w = work[blockIdx.x];
	const int n = w.n;
	const int grid = gp.n_alphas * gp.n_npcs;
	const GridLayout L = grid_layout(gp, n);
	Real *base = Gscr + gp.gbase[w.slot];
	const int32_t *sl = sl_idx + w.sofs;
	const int64_t n2 = (int64_t)n * n;
	const Real *cost = base + L.cost;
	Real yc = Real(0);
	for (int64_t e = threadIdx.x; e < (int64_t)gp.n_untested * n; e += blockDim.x) {
		const int j = (int)(e / gp.n_untested), t = (int)(e - (int64_t)j * gp.n_untested);
		const Real y = (Real)Y[(int64_t)sl[j] * gp.nt + gp.untested[t]];
		yc += y * y;
	}
	const Real yconst = grid_block_sum(yc, red);
	if (threadIdx.x == 0) {
		int b = 0;
		for (int gi = 1; gi < grid; gi++)
			if (cost[gi] < cost[b]) b = gi;
		best = b;
		best_out[w.s] = b;
	}
	__syncthreads();
	if (cost_out)
		for (int gi = threadIdx.x; gi < grid; gi += blockDim.x) cost_out[(int64_t)w.s * grid + gi] = (double)(cost[gi] + yconst);
	// beta of the winner: the cumulative PC chunks up to p of every model, averaged
	const int ba = best / gp.n_npcs, bp = best % gp.n_npcs;
	const Real al = (Real)gp.alphas[ba];
	Real *acc = base + L.P(0, gp.models, gp.mte, n);  // n x n accumulator (column-major)
	for (int64_t e = threadIdx.x; e < n2; e += blockDim.x) acc[e] = Real(0);
	GemmArgs<Real, Real> g;
	g.alpha = Real(1);
	g.beta = Real(1);
	for (int mo = 0; mo < gp.models; mo++) {
		const GridModel md = gp.mdl[mo];
		const Real *V = base + L.Vst + mo * n2;
		const Real *Q = base + L.Qst + mo * n2;
		const Real *lam = base + L.Lst + (int64_t)mo * n;
		for (int p = 0; p <= bp; p++) {
			int r0, r1;
			pc_chunk(gp.npcs, p, min(md.tr_n, n), r0, r1);
			if (r1 <= r0) continue;
			__syncthreads();
			for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) cval[r] = Real(1) / (al + lam[r]);
			__syncthreads();
			// acc(i, j) += sum_r V(i, r) c_r Q(r, j)
			g.M = n; g.N = n; g.K = r1 - r0;
			g.P = V + (int64_t)r0 * n; g.pk = n; g.pi = 1;
			g.Q = Q + r0; g.qk = 1; g.qj = n;
			g.d = cval + r0;
			g.E = acc; g.ei = 1; g.ej = n;
			g.C = acc; g.ci = 1; g.cj = n;
			block_gemm(g, ps, qs);
		}
	}
	__syncthreads();
	double *Bo = Bout + w.tofs;
	const int64_t ti = t_rowmajor ? n : 1, tj = t_rowmajor ? 1 : n;
	for (int64_t e = threadIdx.x; e < n2; e += blockDim.x) {
		const int j = (int)(e / n), i = (int)(e - (int64_t)j * n);
		Bo[i * ti + j * tj] = (double)(acc[e] / (Real)gp.models);
	}
}

// ---------------------------------------------------------------------------------------------
// learned proposal: features and the single fit at the proposed grid point
// ---------------------------------------------------------------------------------------------

constexpr int kFeatSv = 64;  // singular values per feature vector (then log n)

// Features of every searchlight from its eigen decomposition (lambda in the u/v buffer): the 64
// largest singular values sqrt(lambda) divided by the largest (zero-padded), then log n.
__global__ void __launch_bounds__(256) k_features(const SlWork *__restrict__ work, const double *__restrict__ uvbuf,
                                                  float *__restrict__ feat) {
	__shared__ int order[kGridMaxN];
	const SlWork w = work[blockIdx.x];
	const int n = w.n;
	const double *lam = uvbuf + w.uvofs;
	rank_desc(lam, n, order);
	__syncthreads();
	const double s1 = sqrt(fmax(lam[order[0]], 0.0));
	float *f = feat + (int64_t)w.s * (kFeatSv + 1);
	for (int k = threadIdx.x; k < kFeatSv; k += blockDim.x)
		f[k] = (k < n && s1 > 0.0) ? (float)(sqrt(fmax(lam[order[k]], 0.0)) / s1) : 0.0f;
	if (threadIdx.x == 0) f[kFeatSv] = logf((float)n);
}

// beta = sum_k v_k q_k^T mult_k / (alpha + lambda_k) at grid point g = cls[w.s] for the
// searchlights whose proposal probability is at least min_prob: the reference's ha_ridge_grid
// (csrc/ha_ridge.c:97-227) restricted to one (alpha, PC count), with mult_k the number of PC
// chunks up to p that contain component k's rank (clipped at K = min(rows, n)).  V (eigenvectors,
// column-major ld n) and lambda come from the eigenvector-mode Jacobi, C = X_fit^T Y_fit is at
// Cin + w.tofs; beta goes to Bout + w.tofs (float64, T layout; Cin may be Bout: C is read first);
// Q = V^T C goes to the A scratch.  Real is the arithmetic type of the products.
template <typename Real>
__global__ void __launch_bounds__(256) k_proposed_fit(const SlWork *__restrict__ work, const Real *__restrict__ Vscr,
                                                      const double *__restrict__ uvbuf, Real *__restrict__ Ascr,
                                                      const Real *Cin, double *Bout, const int32_t *__restrict__ cls,
                                                      const float *__restrict__ prob, float min_prob,
                                                      const double *__restrict__ alphas, const int32_t *__restrict__ npcs,
                                                      int n_npcs, int rows, int t_rowmajor) {
	__shared__ Real ps[16][65], qs[16][65];
	__shared__ int order[kGridMaxN];
	__shared__ Real cval[kGridMaxN];
	const SlWork w = work[blockIdx.x];
	if (prob[w.s] < min_prob) return;
	const int n = w.n;
	const Real *V = Vscr + w.aofs;
	const double *lam = uvbuf + w.uvofs;
	Real *Q = Ascr + w.aofs;
	const Real *Cs = Cin + w.tofs;
	double *B = Bout + w.tofs;
	const int g = cls[w.s];
	const int a = g / n_npcs, p = g - a * n_npcs;
	const Real al = (Real)alphas[a];
	const int K = min(rows, n);
	rank_desc(lam, n, order);
	__syncthreads();
	for (int r = threadIdx.x; r < n; r += blockDim.x) {
		int mult = 0;
		for (int pp = 0; pp <= p; pp++) {
			int r0, r1;
			pc_chunk(npcs, pp, K, r0, r1);
			mult += (r >= r0 && r < r1);
		}
		const int k = order[r];
		cval[k] = mult ? (Real)mult / (al + (Real)lam[k]) : Real(0);
	}
	GemmArgs<Real, Real> gm;
	gm.d = nullptr; gm.alpha = Real(1); gm.E = nullptr; gm.ei = 0; gm.ej = 0; gm.beta = Real(0);
	// Q(k, j) = sum_i V(i, k) C(i, j)
	gm.M = n; gm.N = n; gm.K = n;
	gm.P = V; gm.pk = 1; gm.pi = n;
	gm.Q = Cs; gm.qk = 1; gm.qj = n;
	gm.C = Q; gm.ci = 1; gm.cj = n;
	block_gemm(gm, ps, qs);
	__syncthreads();  // every read of C (which may share memory with beta) is done
	// beta(i, j) = sum_k V(i, k) c_k Q(k, j), in the T layout
	gm.P = V; gm.pk = n; gm.pi = 1;
	gm.Q = Q; gm.qk = 1; gm.qj = n;
	gm.d = cval;
	GemmArgs<Real, double> gb;
	gb.M = gm.M; gb.N = gm.N; gb.K = gm.K; gb.P = gm.P; gb.pk = gm.pk; gb.pi = gm.pi; gb.Q = gm.Q; gb.qk = gm.qk;
	gb.qj = gm.qj; gb.d = gm.d; gb.alpha = Real(1); gb.E = nullptr; gb.ei = 0; gb.ej = 0; gb.beta = Real(0);
	gb.C = B; gb.ci = t_rowmajor ? n : 1; gb.cj = t_rowmajor ? 1 : n;
	block_gemm(gb, ps, qs);
}

}  // namespace hab200
