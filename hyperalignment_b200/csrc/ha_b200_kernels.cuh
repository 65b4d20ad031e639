// ha_b200_kernels.cuh -- sm_100a kernels of the searchlight alignment path.
//
// Data layout in HBM (one call, one hemisphere):
//   X32, Y32   float  [nv][ntp]   vertex-major time series, ntp = nt rounded up to 32, zero padded
//   X64, Y64   double [nv][nt]    the caller's column-major float64 input (vertex-major already)
//   A scratch  Real   per searchlight: n rows x ncol columns, column-major (column c contiguous),
//              ncol = nblk * bsz >= n (padding columns are zero)
//   V scratch  Real   same shape as A (right singular vectors, accumulated rotations)
//   T scratch  float  per searchlight: n x n local transform, row-major (CSR output) or
//              column-major (CSC output), so the row the reduction needs is contiguous
//   values     double the symmetric CSC/CSR pattern's entries, accumulated in place
//
// Reference anchors: local Procrustes csrc/ha_procrustes.c:17-127 and its
// column-major workspace twin csrc/ha_searchlight.c:578-659; scatter-add
// csrc/ha_searchlight.c:1073-1085 (dense) and csrc/ha_sparse.c:128-142 (CSC);
// pattern csrc/ha_sparse.c:31-112.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hab200 {

// ---------------------------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------------------------

template <typename Real> struct Eps;
template <> struct Eps<float> { static __device__ __forceinline__ float v() { return 1.1920928955078125e-7f; } };
template <> struct Eps<double> { static __device__ __forceinline__ double v() { return 2.220446049250313e-16; } };

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

__device__ __forceinline__ float real_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double real_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float real_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double real_abs(double x) { return fabs(x); }

// Per-searchlight work item of a size bucket.
struct SlWork {
	int32_t s;        // searchlight index
	int32_t n;        // size
	int32_t bsz;      // columns per Jacobi block
	int32_t nblk;     // number of column blocks (even, >= 2); 2 means the matrix stays in shared memory
	int64_t aofs;     // element offset of A / V in the scratch (n * nblk * bsz elements each)
	int64_t tofs;     // element offset of T in the T scratch (n * n)
	int32_t sofs;     // flat offset of the searchlight in sl_indices
	int32_t slot;     // index within the current chunk (stats, uv)
	int64_t uvofs;    // element offset (double) of the saved u_min / v_min vectors (2 n)
};

// Per-searchlight results of the solve.
struct SlStats {
	double s_sum;     // sum of singular values (sign-flipped smallest one when reflection was removed)
	double s_min;     // smallest singular value
	double s_max;     // largest singular value
	int32_t k_min;    // column of the smallest singular value
	int32_t flags;    // bit 0: unconverged, bit 1: ill-conditioned (re-solved in FP64), bit 2: reflected
	int32_t sweeps;   // Jacobi sweeps of the last solve
	int32_t ncols;    // eigenvector mode: the nonzero columns of A lead and number ncols (0: all)
};

enum : int32_t { kFlagUnconverged = 1, kFlagIllCond = 2, kFlagReflected = 4, kFlagFP64 = 8, kFlagCompleted = 16 };

// ---------------------------------------------------------------------------------------------
// layout conversion
// ---------------------------------------------------------------------------------------------

// col-major float64 (vertex v at X[v*nt]) -> vertex-major float32 [nv][ntp], zero padded.
__global__ void k_to_f32_vertex_major(const double *__restrict__ X, int nt, int nv, int ntp,
                                      float *__restrict__ out) {
	int64_t total = (int64_t)nv * ntp;
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
	     e += (int64_t)gridDim.x * blockDim.x) {
		int64_t v = e / ntp;
		int t = (int)(e - v * ntp);
		out[e] = (t < nt) ? (float)X[v * nt + t] : 0.0f;
	}
}

// row-major float64 (X[t*nv + v]) -> column-major float64 (X[v*nt + t]); 32x32 tiles.
__global__ void k_transpose_f64(const double *__restrict__ in, int nt, int nv, double *__restrict__ out) {
	__shared__ double tile[32][33];
	int v0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
	for (int r = threadIdx.y; r < 32; r += blockDim.y) {
		int t = t0 + r, v = v0 + threadIdx.x;
		tile[r][threadIdx.x] = (t < nt && v < nv) ? in[(int64_t)t * nv + v] : 0.0;
	}
	__syncthreads();
	for (int r = threadIdx.y; r < 32; r += blockDim.y) {
		int v = v0 + r, t = t0 + threadIdx.x;
		if (v < nv && t < nt) out[(int64_t)v * nt + t] = tile[threadIdx.x][r];
	}
}

// Population variance / nt of every vertex column, the two-pass loop of
// csrc/ha_searchlight.c:640-652 (mean, then sum of squared deviations), with
// rounded operations so the float64 result does not depend on FMA contraction.
__global__ void k_col_var_over_nt(const double *__restrict__ X, int nt, int nv, double *__restrict__ out) {
	int v = blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= nv) return;
	const double *x = X + (int64_t)v * nt;
	double mean = 0.0;
	for (int i = 0; i < nt; i++) mean = __dadd_rn(mean, x[i]);
	mean = mean / nt;
	double var = 0.0;
	for (int i = 0; i < nt; i++) {
		double d = __dsub_rn(x[i], mean);
		var = __dadd_rn(var, __dmul_rn(d, d));
	}
	out[v] = var / nt;
}

// ---------------------------------------------------------------------------------------------
// cross-covariance  A_s = X[:, sl]^T Y[:, sl]   (csrc/ha_searchlight.c:581-582)
// ---------------------------------------------------------------------------------------------
// One CTA per searchlight, 64x64 output tiles, 16x16 threads with 4x4 register tiles,
// K (time) staged through shared memory in chunks of KT.  Output column-major with
// ncol = nblk*bsz columns; padding columns are written as zeros.

template <typename Real, int KT>
__global__ void __launch_bounds__(256) k_xcov(const SlWork *__restrict__ work, const int32_t *__restrict__ sl_idx,
                                              const Real *__restrict__ Xv, const Real *__restrict__ Yv, int ld,
                                              int nt, Real *__restrict__ Ascr,
                                              const SlStats *__restrict__ stats, int only_flagged) {
	const SlWork w = work[blockIdx.x];
	if (only_flagged && !(stats[w.slot].flags & kFlagIllCond)) return;
	const int n = w.n;
	const int ncol = w.nblk * w.bsz;
	const int32_t *sl = sl_idx + w.sofs;
	Real *A = Ascr + w.aofs;

	__shared__ Real xs[KT][64 + 1];
	__shared__ Real ys[KT][64 + 1];
	__shared__ int32_t vi[64], vj[64];

	const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
	for (int i0 = 0; i0 < n; i0 += 64) {
		for (int j0 = 0; j0 < n; j0 += 64) {
			__syncthreads();
			if (threadIdx.x < 64) {
				int i = i0 + threadIdx.x;
				vi[threadIdx.x] = (i < n) ? sl[i] : -1;
			} else if (threadIdx.x < 128) {
				int j = j0 + threadIdx.x - 64;
				vj[threadIdx.x - 64] = (j < n) ? sl[j] : -1;
			}
			Real acc[4][4];
#pragma unroll
			for (int a = 0; a < 4; a++)
#pragma unroll
				for (int b = 0; b < 4; b++) acc[a][b] = 0;
			for (int t0 = 0; t0 < nt; t0 += KT) {
				__syncthreads();
				// load: 64 vertices x KT samples for X and for Y
				for (int e = threadIdx.x; e < 64 * KT; e += 256) {
					int r = e / KT, t = e - r * KT;
					int tt = t0 + t;
					int v = vi[r], u = vj[r];
					xs[t][r] = (v >= 0 && tt < nt) ? Xv[(int64_t)v * ld + tt] : Real(0);
					ys[t][r] = (u >= 0 && tt < nt) ? Yv[(int64_t)u * ld + tt] : Real(0);
				}
				__syncthreads();
#pragma unroll 4
				for (int t = 0; t < KT; t++) {
					Real a[4], b[4];
#pragma unroll
					for (int q = 0; q < 4; q++) {
						a[q] = xs[t][ty + 16 * q];
						b[q] = ys[t][tx + 16 * q];
					}
#pragma unroll
					for (int p = 0; p < 4; p++)
#pragma unroll
						for (int q = 0; q < 4; q++) acc[p][q] += a[p] * b[q];
				}
			}
#pragma unroll
			for (int p = 0; p < 4; p++) {
				int i = i0 + ty + 16 * p;
				if (i >= n) continue;
#pragma unroll
				for (int q = 0; q < 4; q++) {
					int j = j0 + tx + 16 * q;
					if (j < n) A[(int64_t)j * n + i] = acc[p][q];
				}
			}
		}
	}
	// zero padding columns
	for (int64_t e = (int64_t)n * n + threadIdx.x; e < (int64_t)n * ncol; e += 256) A[e] = 0;
}

// ---------------------------------------------------------------------------------------------
// one-sided Jacobi (Hestenes) on the columns of A, accumulating V
// ---------------------------------------------------------------------------------------------
// A V = B with orthogonal columns; sigma_c = ||B[:, c]||, U = B diag(1/sigma), T = U V^T
// (the polar factor of A, csrc/ha_searchlight.c:593-609).  Parallel ordering: the
// circle-method round robin over m columns (m - 1 rounds of m/2 disjoint pairs).
// Squared column norms are cached in shared memory (recomputed exactly at the start of
// every sweep or staging, updated by alpha' = alpha - t gamma, beta' = beta + t gamma after a
// rotation), so a pair needs one dot product; each warp takes up to JP pairs of a round at
// once so their reductions overlap.  A pair is rotated when |cos| > tol_rot; a sweep whose
// largest |cos| is <= tol_conv ends the iteration.  Columns whose norm is below zero_thr
// (numerically zero, e.g. rank-deficient A) are not rotated; they are completed to an
// orthonormal basis at the end.
//
// Resident mode (nblk == 2): A and V live in shared memory for every sweep.
// Blocked mode (nblk > 2): A and V stay in the global scratch (L2 resident); a sweep visits
// the block pairs in row-cyclic order with two staging slots in shared memory (A and V columns),
// block I in slot 0 for its whole row and block J in slot 1.  Block 0 meets every block first:
// (0, 1) runs the full round robin over both blocks, (0, J) the round robin inside block J and
// then the cross pairs, later pairs only the cross pairs, so one sweep visits every column pair
// exactly once.  Blocks have an even width.

// Pairs processed together by one warp (their reductions overlap), by rows per lane.  The float
// instances with 8 and 10 rows per lane run at most 384 threads (their blocked buckets use 12 and
// 10 warps), which leaves 80 registers a thread: no spills, and two pairs per warp at 10 rows.
template <typename Real, int RPL>
struct PairsPerWarp {
	static constexpr int value = RPL <= 4 ? 4 : ((RPL <= 8 || (sizeof(Real) == 4 && RPL == 10)) ? 2 : 1);
};

template <typename Real, int RPL>
struct JacobiBounds {
	static constexpr int threads = (sizeof(Real) == 4 && (RPL == 8 || RPL == 10)) ? 384 : 512;
	static constexpr int blocks = sizeof(Real) == 4 ? 2 : 1;
};

// circle method: pair k of round r among m players (m even); no integer division
__device__ __forceinline__ void rr_pair(int m, int r, int k, int &p, int &q) {
	if (k == 0) {
		p = m - 1;
		q = r;
	} else {
		const int mm = m - 1;
		p = r + k;
		if (p >= mm) p -= mm;
		q = r - k;
		if (q < 0) q += mm;
	}
}

// Rotation parameters: the hardware reciprocal square root and fast division in float32 (a
// rotation only needs c^2 + s^2 = 1 to working precision, which c = rsqrt(1 + t^2), s = c t
// keeps); IEEE operations in float64.
__device__ __forceinline__ float rot_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rot_rsqrt(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ float rot_div(float a, float b) { return __fdividef(a, b); }
// c = 1 / sqrt(x) to full float32 precision (hardware estimate + one Newton step), so that
// c^2 + s^2 = 1 holds to rounding and V stays orthogonal over thousands of rotations
__device__ __forceinline__ float rot_cos(float x) {
	const float y = rsqrtf(x);
	return y * fmaf(-0.5f * x * y, y, 1.5f);
}
__device__ __forceinline__ double rot_cos(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ double rot_div(double a, double b) { return a / b; }

template <typename Real>
struct JacobiTol {
	Real rot;    // rotate when |cos| > rot
	Real zero2;  // squared norm at or below which a column counts as zero
};

// Rows a lane owns in a column of LD = 32*RPL rows: chunks of VW consecutive rows, chunk c of lane l
// at row c*32*VW + l*VW, with VW as many rows as 16 bytes hold when RPL allows.  Every row has one
// owner and the rows keep their natural order in shared memory, so a lane moves its chunk with one
// 16-byte load or store and consecutive lanes touch consecutive 16-byte words (no bank conflicts).
template <typename Real, int VW> struct VecOf { using T = Real; };
template <> struct VecOf<float, 4> { using T = float4; };
template <> struct VecOf<float, 2> { using T = float2; };
template <> struct VecOf<double, 2> { using T = double2; };

template <typename Real, int RPL>
struct LaneRows {
	static constexpr int W16 = 16 / (int)sizeof(Real);
	static constexpr int VW = (RPL % W16 == 0) ? W16 : ((RPL % 2 == 0) ? 2 : 1);
	static constexpr int NC = RPL / VW;
	using V = typename VecOf<Real, VW>::T;
	static __device__ __forceinline__ int ofs(int lane, int c) { return c * 32 * VW + lane * VW; }
	static __device__ __forceinline__ void load(const Real *col, int lane, Real (&x)[RPL]) {
#pragma unroll
		for (int c = 0; c < NC; c++) {
			const V v = *reinterpret_cast<const V *>(col + ofs(lane, c));
			const Real *e = reinterpret_cast<const Real *>(&v);
#pragma unroll
			for (int q = 0; q < VW; q++) x[c * VW + q] = e[q];
		}
	}
	static __device__ __forceinline__ void store(Real *col, int lane, const Real (&x)[RPL]) {
#pragma unroll
		for (int c = 0; c < NC; c++) {
			V v;
			Real *e = reinterpret_cast<Real *>(&v);
#pragma unroll
			for (int q = 0; q < VW; q++) e[q] = x[c * VW + q];
			*reinterpret_cast<V *>(col + ofs(lane, c)) = v;
		}
	}
};

// sqrt(x) for x >= 1 in the rotation tangent: hardware reciprocal square root in float32 (the
// tangent only steers the rotation; c and s = c t stay orthogonal through rot_cos), IEEE in float64.
__device__ __forceinline__ float rot_sqrt(float x) { return x * rsqrtf(x); }
__device__ __forceinline__ double rot_sqrt(double x) { return sqrt(x); }

// Sum of each of the JPW per-lane partial dot products over the warp, reduce-scatter style: pair k's
// total ends up in the lanes of group k (32 / JPW consecutive lanes), with log2(JPW) fewer shuffles
// per pair than one butterfly per pair.
template <typename Real, int JPW>
__device__ __forceinline__ Real pair_sums(const Real (&g)[JPW], int lane) {
	if constexpr (JPW == 4) {
		const bool hi = lane & 16, h8 = lane & 8;
		const Real r0 = __shfl_xor_sync(0xffffffffu, hi ? g[0] : g[2], 16);
		const Real r1 = __shfl_xor_sync(0xffffffffu, hi ? g[1] : g[3], 16);
		const Real a0 = (hi ? g[2] : g[0]) + r0, a1 = (hi ? g[3] : g[1]) + r1;
		Real v = (h8 ? a1 : a0) + __shfl_xor_sync(0xffffffffu, h8 ? a0 : a1, 8);
#pragma unroll
		for (int o = 4; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
		return v;
	} else if constexpr (JPW == 2) {
		const bool hi = lane & 16;
		Real v = (hi ? g[1] : g[0]) + __shfl_xor_sync(0xffffffffu, hi ? g[0] : g[1], 16);
#pragma unroll
		for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
		return v;
	} else {
		return warp_sum(g[0]);
	}
}

// Rotate JPW pairs (p[k], q[k]) of columns stored at B + c*LD (and V + c*LD) in shared memory,
// LD = 32*RPL rows with rows >= n zero, so every lane handles exactly RPL rows and no row test
// is needed.  Unused pair slots point at two zero columns and are skipped like any zero column.
// nrm[] holds the cached squared norms.  The columns of B stay in registers between the dot
// products and the rotation; the first lane of group k computes pair k's rotation and
// broadcasts it.  Returns the largest |cos| seen.
template <typename Real, int RPL>
__device__ __forceinline__ Real jacobi_pairs(Real *B, Real *V, Real *nrm, const int *p, const int *q,
                                             const JacobiTol<Real> &tol, int lane, bool &rotated) {
	constexpr int JPW = PairsPerWarp<Real, RPL>::value;
	constexpr int LD = 32 * RPL;
	constexpr int GRP = 32 / JPW;  // lanes per pair group
	using LR = LaneRows<Real, RPL>;
	Real x[JPW][RPL], y[JPW][RPL], g[JPW];
#pragma unroll
	for (int k = 0; k < JPW; k++) {
		LR::load(B + p[k] * LD, lane, x[k]);
		LR::load(B + q[k] * LD, lane, y[k]);
		Real g0 = 0, g1 = 0;  // two partial sums halve the dependency chain
#pragma unroll
		for (int r = 0; r < RPL; r++) {
			if (r & 1)
				g1 += x[k][r] * y[k][r];
			else
				g0 += x[k][r] * y[k][r];
		}
		g[k] = g0 + g1;
	}
	const Real gk = pair_sums<Real, JPW>(g, lane);
	const int kk = lane / GRP;
	Real mycos = 0, myc = 1, mys = 0;
	int mydo = 0;
	if ((lane & (GRP - 1)) == 0) {
		int pk = p[0], qk = q[0];
#pragma unroll
		for (int k = 1; k < JPW; k++)
			if (kk == k) { pk = p[k]; qk = q[k]; }
		const Real al = nrm[pk], be = nrm[qk];
		if (al > tol.zero2 && be > tol.zero2) {
			mycos = real_abs(gk) * rot_rsqrt(al) * rot_rsqrt(be);
			if (mycos > tol.rot) {
				const Real zeta = rot_div(be - al, 2 * gk);
				const Real t = rot_div((zeta >= 0) ? Real(1) : Real(-1), real_abs(zeta) + rot_sqrt(Real(1) + zeta * zeta));
				myc = rot_cos(Real(1) + t * t);
				mys = myc * t;
				mydo = 1;
				nrm[pk] = al - t * gk;
				nrm[qk] = be + t * gk;
			}
		}
	}
#pragma unroll
	for (int k = 0; k < JPW; k++) {
		if (!__shfl_sync(0xffffffffu, mydo, k * GRP)) continue;
		const Real c = __shfl_sync(0xffffffffu, myc, k * GRP);
		const Real s = __shfl_sync(0xffffffffu, mys, k * GRP);
#pragma unroll
		for (int r = 0; r < RPL; r++) {
			const Real a = x[k][r], b2 = y[k][r];
			x[k][r] = c * a - s * b2;
			y[k][r] = s * a + c * b2;
		}
		LR::store(B + p[k] * LD, lane, x[k]);
		LR::store(B + q[k] * LD, lane, y[k]);
		if (V) {  // null when the rotations are not accumulated (eigenvector mode); x, y reused
			LR::load(V + p[k] * LD, lane, x[k]);
			LR::load(V + q[k] * LD, lane, y[k]);
#pragma unroll
			for (int r = 0; r < RPL; r++) {
				const Real a = x[k][r], b2 = y[k][r];
				x[k][r] = c * a - s * b2;
				y[k][r] = s * a + c * b2;
			}
			LR::store(V + p[k] * LD, lane, x[k]);
			LR::store(V + q[k] * LD, lane, y[k]);
		}
		rotated = true;
	}
	__syncwarp();
	return mycos;
}

// exact squared norms of columns [0, m) (stride LD) into nrm[]
template <typename Real, int RPL>
__device__ __forceinline__ void column_norms(const Real *B, Real *nrm, int m) {
	constexpr int LD = 32 * RPL;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	for (int c = warp; c < m; c += nwarp) {
		Real x[RPL];
		LaneRows<Real, RPL>::load(B + c * LD, lane, x);
		Real ss = 0;
#pragma unroll
		for (int r = 0; r < RPL; r++) ss += x[r] * x[r];
		ss = warp_sum(ss);
		if (lane == 0) nrm[c] = ss;
	}
	__syncthreads();
}

// Full round robin (m - 1 rounds) over m columns; columns m and m+1 are the zero pair used to
// pad a warp's last group.  Returns this thread's max |cos|.
template <typename Real, int RPL>
__device__ __forceinline__ Real jacobi_full_rr(Real *B, Real *V, Real *nrm, int m, const JacobiTol<Real> &tol,
                                               bool &rotated) {
	constexpr int JPW = PairsPerWarp<Real, RPL>::value;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	Real mc = 0;
	const int npairs = m / 2;
	for (int r = 0; r < m - 1; r++) {
		for (int k0 = warp * JPW; k0 < npairs; k0 += nwarp * JPW) {
			int p[JPW], q[JPW];
#pragma unroll
			for (int k = 0; k < JPW; k++) {
				if (k0 + k < npairs) {
					rr_pair(m, r, k0 + k, p[k], q[k]);
				} else {
					p[k] = m;
					q[k] = m + 1;
				}
			}
			Real c = jacobi_pairs<Real, RPL>(B, V, nrm, p, q, tol, lane, rotated);
			mc = c > mc ? c : mc;
		}
		__syncthreads();
	}
	return mc;
}

// Cross pairs only between column halves [0, h) and [h, 2h): h rounds of h pairs; columns 2h and
// 2h+1 are the zero padding pair.
template <typename Real, int RPL>
__device__ __forceinline__ Real jacobi_cross(Real *B, Real *V, Real *nrm, int h, const JacobiTol<Real> &tol,
                                             bool &rotated) {
	constexpr int JPW = PairsPerWarp<Real, RPL>::value;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	Real mc = 0;
	for (int r = 0; r < h; r++) {
		for (int k0 = warp * JPW; k0 < h; k0 += nwarp * JPW) {
			int p[JPW], q[JPW];
#pragma unroll
			for (int k = 0; k < JPW; k++) {
				if (k0 + k < h) {
					p[k] = k0 + k;
					int qq = k0 + k + r;
					if (qq >= h) qq -= h;
					q[k] = h + qq;
				} else {
					p[k] = 2 * h;
					q[k] = 2 * h + 1;
				}
			}
			Real c = jacobi_pairs<Real, RPL>(B, V, nrm, p, q, tol, lane, rotated);
			mc = c > mc ? c : mc;
		}
		__syncthreads();
	}
	return mc;
}

// block-wide maximum of a non-negative value (all threads get the result)
template <typename Real>
__device__ Real block_max_nonneg(Real v, Real *scratch32) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		Real w = __shfl_xor_sync(0xffffffffu, v, o);
		v = w > v ? w : v;
	}
	__syncthreads();
	if (lane == 0) scratch32[warp] = v;
	__syncthreads();
	Real m = 0;
	for (int q = 0; q < nwarp; q++) m = scratch32[q] > m ? scratch32[q] : m;
	__syncthreads();
	return m;
}

// ---------------------------------------------------------------------------------------------
// generic small GEMM:  C(i, j) = alpha * sum_k P(k, i) d(k) Q(k, j) + beta * E(i, j)
// ---------------------------------------------------------------------------------------------
// Operands are addressed through strides, P(k, i) = P[k*pk + i*pi] etc., so the same routine
// serves every layout used here; tiles of 64x64 outputs per pass, K staged in chunks of 16.
template <typename Real, typename OutT = Real>
struct GemmArgs {
	int M, N, K;
	const Real *P;
	int64_t pk, pi;
	const Real *Q;
	int64_t qk, qj;
	const Real *d;  // optional K scales (nullptr = 1)
	Real alpha;
	const Real *E;  // optional addend (nullptr = none)
	int64_t ei, ej;
	Real beta;
	OutT *C;
	int64_t ci, cj;
};

template <typename Real, typename OutT>
__device__ void block_gemm(const GemmArgs<Real, OutT> &g, Real (*ps)[65], Real (*qs)[65]) {
	constexpr int KC = 16;
	const int tx = threadIdx.x & 15, ty = (threadIdx.x >> 4) & 15;
	const int nthr = blockDim.x;  // 256 assumed for the compute mapping
	for (int i0 = 0; i0 < g.M; i0 += 64) {
		for (int j0 = 0; j0 < g.N; j0 += 64) {
			Real acc[4][4];
#pragma unroll
			for (int a = 0; a < 4; a++)
#pragma unroll
				for (int b = 0; b < 4; b++) acc[a][b] = 0;
			for (int k0 = 0; k0 < g.K; k0 += KC) {
				__syncthreads();
				for (int e = threadIdx.x; e < KC * 64; e += nthr) {
					int kk = e >> 6, ii = e & 63;
					int k = k0 + kk;
					int i = i0 + ii, j = j0 + ii;
					Real dk = (k < g.K && g.d) ? g.d[k] : Real(1);
					ps[kk][ii] = (k < g.K && i < g.M) ? g.P[k * g.pk + i * g.pi] * dk : Real(0);
					qs[kk][ii] = (k < g.K && j < g.N) ? g.Q[k * g.qk + j * g.qj] : Real(0);
				}
				__syncthreads();
				if (threadIdx.x < 256) {
#pragma unroll
					for (int kk = 0; kk < KC; kk++) {
						Real a[4], b[4];
#pragma unroll
						for (int q = 0; q < 4; q++) {
							a[q] = ps[kk][ty + 16 * q];
							b[q] = qs[kk][tx + 16 * q];
						}
#pragma unroll
						for (int p = 0; p < 4; p++)
#pragma unroll
							for (int q = 0; q < 4; q++) acc[p][q] += a[p] * b[q];
					}
				}
			}
			if (threadIdx.x < 256) {
#pragma unroll
				for (int p = 0; p < 4; p++) {
					int i = i0 + ty + 16 * p;
					if (i >= g.M) continue;
#pragma unroll
					for (int q = 0; q < 4; q++) {
						int j = j0 + tx + 16 * q;
						if (j >= g.N) continue;
						Real v = g.alpha * acc[p][q];
						if (g.E) v += g.beta * g.E[i * g.ei + j * g.ej];
						g.C[i * g.ci + j * g.cj] = (OutT)v;
					}
				}
			}
		}
	}
	__syncthreads();
}

// ---------------------------------------------------------------------------------------------
// Jacobi polar kernel
// ---------------------------------------------------------------------------------------------
// Per searchlight: run sweeps until converged (or max_sweeps), take sigma_c = ||B[:, c]||,
// form T = B diag(1/sigma) V^T into the T scratch (row-major when t_rowmajor, else
// column-major), and record the singular-value statistics and the singular pair of the
// smallest singular value (for the reflection fix).  Numerically zero columns get an
// orthonormal completion so T stays orthogonal.

struct JacobiParams {
	int max_sweeps;
	int t_rowmajor;
	double ill_ratio;  // sigma_min / sigma_max below this -> kFlagIllCond
	double weak;       // columns with sigma <= weak * eps * sigma_max are re-orthogonalised / completed
	int eig;           // eigenvector mode (A A^T = G): no V; write u_c = b_c / sigma_c (column-major, ld n,
	                   // zero for numerically zero columns) to the V scratch and sigma_c^2 to uvbuf
	int only_flagged;  // process only searchlights whose stats carry kFlagIllCond (FP64 re-solve)
	int keep_v;        // write V (column-major, ld n) to the V scratch for searchlights this solve flags
	int warm;          // start from the rotations V in the V scratch (A already multiplied by V)
	double stop_cos;   // also stop after a sweep whose largest |cos| is at most this (0: off)
};

template <typename Real, int RPL>
__global__ void __launch_bounds__(JacobiBounds<Real, RPL>::threads, JacobiBounds<Real, RPL>::blocks) k_jacobi(const SlWork *__restrict__ work, Real *__restrict__ Ascr,
                                                   Real *__restrict__ Vscr, float *__restrict__ Tscr,
                                                   SlStats *__restrict__ stats, double *__restrict__ uvbuf,
                                                   JacobiParams prm) {
	constexpr int LD = 32 * RPL;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	Real *sm = reinterpret_cast<Real *>(smem_raw);
	const SlWork w = work[blockIdx.x];
	if (prm.only_flagged && !(stats[w.slot].flags & kFlagIllCond)) return;
	const int n = w.n, bsz = w.bsz, nblk = w.nblk;
	const int ncol = nblk * bsz;
	const int mst = 2 * bsz + 2;  // staged columns: two blocks plus the zero padding pair
	Real *Ag = Ascr + w.aofs;
	Real *Vg = Vscr + w.aofs;
	const Real eps = Eps<Real>::v();
	const Real sqn = real_sqrt(Real(n));
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;

	// shared: Bs[mst][LD], Vs[mst][LD], nrm[mst], then GEMM tiles (resident mode); eigenvector
	// mode has no Vs (nrm follows Bs)
	Real *Bs = sm;
	Real *Vs = sm + mst * LD;
	Real *nrm = prm.eig ? Vs : Vs + mst * LD;
	__shared__ Real red[32];
	__shared__ double frob2;

	const bool resident = (nblk == 2);
	// ||A||_F^2 (invariant under the rotations) sets the zero threshold
	{
		Real ss = 0;
		for (int e = threadIdx.x; e < n * n; e += blockDim.x) ss += Ag[e] * Ag[e];
		ss = warp_sum(ss);
		if (threadIdx.x == 0) frob2 = 0;
		__syncthreads();
		if (lane == 0) atomicAdd(&frob2, (double)ss);
		__syncthreads();
	}
	JacobiTol<Real> tol;
	tol.rot = eps * sqn;
	tol.zero2 = (Real)(frob2 * (double)(eps * sqn) * (double)(eps * sqn));
	// Rotations converge quadratically: a sweep that starts with every |cos| below stop_cos leaves the
	// columns orthogonal to working precision, so the sweep that would only confirm it is skipped.
	const Real tol_conv = fmax(Real(4) * eps * sqn, (Real)prm.stop_cos);

	bool converged = false;
	int sweep = 0;
	if (resident) {
		for (int e = threadIdx.x; e < mst * LD; e += blockDim.x) {
			const int c = e / LD, i = e - c * LD;
			Bs[e] = (c < ncol && i < n) ? Ag[c * n + i] : Real(0);
			if (!prm.eig)
				Vs[e] = prm.warm ? ((c < n && i < n) ? Vg[c * n + i] : Real(0)) : ((c == i && c < n) ? Real(1) : Real(0));
		}
		__syncthreads();
		for (sweep = 0; sweep < prm.max_sweeps; sweep++) {
			column_norms<Real, RPL>(Bs, nrm, mst);
			bool rot = false;
			Real mc = jacobi_full_rr<Real, RPL>(Bs, prm.eig ? nullptr : Vs, nrm, 2 * bsz, tol, rot);
			mc = block_max_nonneg(mc, red);
			if (mc <= tol_conv) {
				converged = true;
				sweep++;
				break;
			}
		}
	} else {
		if (!prm.eig && !prm.warm)
			for (int e = threadIdx.x; e < ncol * n; e += blockDim.x) {
				const int c = e / n, i = e - c * n;
				Vg[e] = (c == i) ? Real(1) : Real(0);
			}
		Real *Vst = prm.eig ? nullptr : Vs;
		for (int e = threadIdx.x; e < mst * LD; e += blockDim.x) {
			Bs[e] = Real(0);
			if (Vst) Vs[e] = Real(0);
		}
		__syncthreads();
		// only the blocks holding the leading nonzero columns take part (eigenvector mode)
		int nb = nblk;
		if (prm.eig && stats[w.slot].ncols > 0) {
			nb = max(2, (stats[w.slot].ncols + bsz - 1) / bsz);
			nb += nb & 1;
			nb = min(nb, nblk);
		}
		// block b of the scratch <-> staging slot (columns slot*bsz ..): each element is moved by the
		// same thread in both directions, so a slot can be written back and refilled without a barrier
		auto unstage = [&](int blk, int slot) {
			for (int e = threadIdx.x; e < bsz * n; e += blockDim.x) {
				const int c = e / n, i = e - c * n;
				const int gc = blk * bsz + c, sc = slot * bsz + c;
				Ag[gc * n + i] = Bs[sc * LD + i];
				if (Vst) Vg[gc * n + i] = Vs[sc * LD + i];
			}
		};
		auto stage = [&](int blk, int slot) {
			for (int e = threadIdx.x; e < bsz * n; e += blockDim.x) {
				const int c = e / n, i = e - c * n;
				const int gc = blk * bsz + c, sc = slot * bsz + c;
				Bs[sc * LD + i] = Ag[gc * n + i];
				if (Vst) Vs[sc * LD + i] = Vg[gc * n + i];
			}
		};
		// pull the next block to be staged (A and V columns) towards L2 while the current pair rotates
		auto prefetch = [&](int blk) {
			const int lines = bsz * n * (int)sizeof(Real) / 128;  // every prefetched address inside the block
			const char *a = reinterpret_cast<const char *>(Ag + blk * bsz * n);
			const char *v = reinterpret_cast<const char *>(Vg + blk * bsz * n);
			for (int l = threadIdx.x; l < lines; l += blockDim.x) {
				asm volatile("prefetch.global.L2 [%0];" ::"l"(a + 128 * l));
				if (Vst) asm volatile("prefetch.global.L2 [%0];" ::"l"(v + 128 * l));
			}
		};
		// Block pairs in row-cyclic order (0,1), (0,2), .., (0,nb-1), (1,2), ..: block I stays staged
		// while J streams past, so each pair stages one block.  Each block's internal pairs run when
		// it first meets block 0 (block 0's own with block 1), so a sweep visits every pair once.
		for (sweep = 0; sweep < prm.max_sweeps; sweep++) {
			Real mc = 0;
			bool rot = false;
			for (int I = 0; I < nb - 1; I++) {
				for (int J = I + 1; J < nb; J++) {
					if (J == I + 1) {
						if (I > 0) {
							unstage(I - 1, 0);
							unstage(nb - 1, 1);
						}
						stage(I, 0);
					} else {
						unstage(J - 1, 1);
					}
					stage(J, 1);
					if (J + 1 < nb)
						prefetch(J + 1);
					else if (I + 2 < nb)
						prefetch(I + 2);
					__syncthreads();
					column_norms<Real, RPL>(Bs, nrm, mst);
					Real c;
					if (I == 0 && J == 1) {
						c = jacobi_full_rr<Real, RPL>(Bs, Vst, nrm, 2 * bsz, tol, rot);
					} else {
						c = 0;
						if (I == 0)
							c = jacobi_full_rr<Real, RPL>(Bs + bsz * LD, Vst ? Vs + bsz * LD : nullptr, nrm + bsz, bsz,
							                             tol, rot);
						const Real c2 = jacobi_cross<Real, RPL>(Bs, Vst, nrm, bsz, tol, rot);
						c = c2 > c ? c2 : c;
					}
					mc = c > mc ? c : mc;
				}
			}
			unstage(nb - 2, 0);
			unstage(nb - 1, 1);
			__syncthreads();
			mc = block_max_nonneg(mc, red);
			if (mc <= tol_conv) {
				converged = true;
				sweep++;
				break;
			}
		}
	}

	// from here on: B, V with column stride ldb (shared, LD, or global, n)
	Real *B = resident ? Bs : Ag;
	Real *V = resident ? Vs : Vg;
	const int ldb = resident ? LD : n;
	// column norms (sigma) -> sg[] (resident: the nrm area; blocked: the staging area)
	Real *sg = resident ? nrm : Bs;
	for (int c = warp; c < ncol; c += nwarp) {
		const Real *bc = B + c * ldb;
		Real ss = 0;
		for (int i = lane; i < n; i += 32) ss += bc[i] * bc[i];
		ss = warp_sum(ss);
		if (lane == 0) sg[c] = (c < n) ? real_sqrt(ss) : Real(0);
	}
	__syncthreads();
	// statistics over the n real columns
	__shared__ double red_sum[32], red_max[32], red_min[32];
	__shared__ int red_kmin[32];
	{
		double ssum = 0, smax = 0, smin = 1e308;
		int kmin = 0;
		for (int c = threadIdx.x; c < n; c += blockDim.x) {
			double v = (double)sg[c];
			ssum += v;
			smax = fmax(smax, v);
			if (v < smin) { smin = v; kmin = c; }
		}
		ssum = warp_sum(ssum);
		for (int o = 16; o > 0; o >>= 1) {
			smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
			double om = __shfl_xor_sync(0xffffffffu, smin, o);
			int ok = __shfl_xor_sync(0xffffffffu, kmin, o);
			if (om < smin || (om == smin && ok < kmin)) { smin = om; kmin = ok; }
		}
		if (lane == 0) { red_sum[warp] = ssum; red_max[warp] = smax; red_min[warp] = smin; red_kmin[warp] = kmin; }
		__syncthreads();
		if (threadIdx.x == 0) {
			double a = 0, mx = 0, mn = 1e308;
			int km = 0;
			for (int q = 0; q < nwarp; q++) {
				a += red_sum[q];
				mx = fmax(mx, red_max[q]);
				if (red_min[q] < mn || (red_min[q] == mn && red_kmin[q] < km)) { mn = red_min[q]; km = red_kmin[q]; }
			}
			SlStats st = stats[w.slot];
			int fl = (sizeof(Real) == 8) ? kFlagFP64 : 0;
			if (prm.only_flagged) fl |= (st.flags & kFlagIllCond);
			if (!converged) fl |= kFlagUnconverged;
			if (!prm.only_flagged && prm.ill_ratio > 0 && (!converged || mx == 0.0 || mn < prm.ill_ratio * mx))
				fl |= kFlagIllCond;
			st.s_sum = a;
			st.s_max = mx;
			st.s_min = mn;
			st.k_min = km;
			st.flags = fl;
			st.sweeps = sweep;
			stats[w.slot] = st;
		}
		__syncthreads();
	}
	// keep V of a searchlight handed to the float64 re-solve (its warm start)
	if (prm.keep_v && resident && (stats[w.slot].flags & kFlagIllCond))
		for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
			const int c = e / n, i = e - c * n;
			Vg[e] = Vs[c * LD + i];
		}
	// eigenvector mode: A W = B with orthogonal columns, so G = A A^T = B B^T has the eigenvectors
	// b_c / sigma_c and the eigenvalues sigma_c^2
	if (prm.eig) {
		for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
			const int c = e / n, i = e - c * n;
			const Real sc = sg[c];
			Vg[e] = (sc * sc > tol.zero2) ? B[c * ldb + i] / sc : Real(0);
		}
		for (int k = threadIdx.x; k < n; k += blockDim.x) {
			const double sk = (double)sg[k];
			uvbuf[w.uvofs + k] = (sg[k] * sg[k] > tol.zero2) ? sk * sk : 0.0;
		}
		return;
	}
	// normalise columns: u_c = b_c / sigma_c (in place)
	for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
		const int c = e / n, i = e - c * n;
		const Real s = sg[c];
		B[c * ldb + i] = (s > 0) ? B[c * ldb + i] / s : Real(0);
	}
	__syncthreads();
	// Weak columns (sigma <= 1e3 eps sigma_max) carry directions that the rotations cannot make
	// orthogonal to working precision, and exactly null ones carry none.  Each is re-orthogonalised
	// (two Gram-Schmidt passes) against the strong columns and the weak ones before it; if little
	// of it is left it is replaced by an orthonormal completion: the unit vector e_i with the
	// largest remainder after the same projection.  The complement of the other columns has at
	// least one dimension, so some e_i keeps a squared remainder >= 1/n; any remainder above
	// 1/(2n) is accepted, else the best one.  Executed by warp 0.
	{
		const Real smax = (Real)stats[w.slot].s_max;
		const Real weak = smax * Real(prm.weak) * eps;
		if (warp == 0) {
			for (int c = 0; c < n; c++) {
				if (sg[c] > weak) continue;
				Real *uc = B + c * ldb;
				Real best = -1;
				int best_cand = 0;
				for (int cand = -1; cand <= n; cand++) {
					const int use = (cand == n) ? best_cand : cand;  // final pass: rebuild the best
					if (cand >= 0)
						for (int i = lane; i < n; i += 32) uc[i] = (i == use) ? Real(1) : Real(0);
					__syncwarp();
					for (int pass = 0; pass < 2; pass++) {
						for (int o = 0; o < n; o++) {
							if (o == c || (o > c && sg[o] <= weak)) continue;
							const Real *uo = B + o * ldb;
							Real dp = 0;
							for (int i = lane; i < n; i += 32) dp += uo[i] * uc[i];
							dp = warp_sum(dp);
							for (int i = lane; i < n; i += 32) uc[i] -= dp * uo[i];
							__syncwarp();
						}
					}
					Real nn = 0;
					for (int i = lane; i < n; i += 32) nn += uc[i] * uc[i];
					nn = warp_sum(nn);
					const Real accept = (cand < 0) ? Real(0.25) : Real(0.5) / Real(n);
					if (nn > accept || (cand == n && nn > 0)) {
						Real inv = Real(1) / real_sqrt(nn);
						for (int i = lane; i < n; i += 32) uc[i] *= inv;
						__syncwarp();
						break;
					}
					if (cand >= 0 && cand < n && nn > best) {
						best = nn;
						best_cand = cand;
					}
				}
			}
		}
	}
	__syncthreads();
	// save u_min, v_min for the reflection fix
	{
		const int km = stats[w.slot].k_min;
		double *uv = uvbuf + w.uvofs;
		for (int i = threadIdx.x; i < n; i += blockDim.x) {
			uv[i] = (double)B[km * ldb + i];
			uv[n + i] = (double)V[km * ldb + i];
		}
	}
	// T = U V^T :  T(i, j) = sum_c U[c][i] V[c][j], written as float32 (resident mode; the
	// blocked mode forms T in k_form_t_global)
	if (resident) {
		GemmArgs<Real, float> g;
		g.M = n; g.N = n; g.K = n;
		g.P = B; g.pk = LD; g.pi = 1;
		g.Q = V; g.qk = LD; g.qj = 1;
		g.d = nullptr; g.alpha = Real(1);
		g.E = nullptr; g.ei = 0; g.ej = 0; g.beta = 0;
		g.C = Tscr + w.tofs;
		g.ci = prm.t_rowmajor ? n : 1;
		g.cj = prm.t_rowmajor ? 1 : n;
		Real (*ps)[65] = reinterpret_cast<Real (*)[65]>(nrm + mst + 2);
		Real (*qs)[65] = ps + 16;
		block_gemm(g, ps, qs);
	}
}

// Warm start of the float64 re-solve of a searchlight the float32 solve flagged, part 1: the
// float32 rotations V32 (column-major, ld n, in the V scratch, same bytes as the float64 V) become
// float64 and get one Newton-Schulz step, V = V32 (3I - V32^T V32) / 2, which takes their
// orthogonality error (~1e-6) to float64 level.  The A scratch and the float64 T scratch are
// temporaries (A is computed after this).  Padding columns of V are zero.
__global__ void __launch_bounds__(256) k_warm_v(const SlWork *__restrict__ work, double *__restrict__ Ascr,
                                                double *__restrict__ Vscr, double *__restrict__ Tmp,
                                                const SlStats *__restrict__ stats) {
	__shared__ double ps[16][65], qs[16][65];
	const SlWork w = work[blockIdx.x];
	if (!(stats[w.slot].flags & kFlagIllCond)) return;
	const int n = w.n, ncol = w.nblk * w.bsz;
	const int64_t n2 = (int64_t)n * n;
	const float *V32 = reinterpret_cast<const float *>(Vscr + w.aofs);
	double *W = Ascr + w.aofs;
	double *G = Tmp + w.tofs;
	double *V = Vscr + w.aofs;
	for (int64_t e = threadIdx.x; e < n2; e += blockDim.x) W[e] = (double)V32[e];
	__syncthreads();
	GemmArgs<double, double> g;
	g.d = nullptr; g.E = nullptr; g.ei = 0; g.ej = 0; g.beta = 0.0;
	// G = -W^T W / 2, then + 3I/2
	g.M = n; g.N = n; g.K = n; g.alpha = -0.5;
	g.P = W; g.pk = 1; g.pi = n;
	g.Q = W; g.qk = 1; g.qj = n;
	g.C = G; g.ci = 1; g.cj = n;
	block_gemm(g, ps, qs);
	for (int i = threadIdx.x; i < n; i += blockDim.x) G[(int64_t)i * n + i] += 1.5;
	__syncthreads();
	// V = W G
	g.alpha = 1.0;
	g.P = W; g.pk = n; g.pi = 1;
	g.Q = G; g.qk = 1; g.qj = n;
	g.C = V; g.ci = 1; g.cj = n;
	block_gemm(g, ps, qs);
	for (int64_t e = n2 + threadIdx.x; e < (int64_t)n * ncol; e += blockDim.x) V[e] = 0.0;
}

// Part 2, after the float64 cross-covariance: A := A V (through the float64 T scratch), so the
// rotations continue from the float32 solution and most pairs are already orthogonal.
__global__ void __launch_bounds__(256) k_warm_av(const SlWork *__restrict__ work, double *__restrict__ Ascr,
                                                 const double *__restrict__ Vscr, double *__restrict__ Tmp,
                                                 const SlStats *__restrict__ stats) {
	__shared__ double ps[16][65], qs[16][65];
	const SlWork w = work[blockIdx.x];
	if (!(stats[w.slot].flags & kFlagIllCond)) return;
	const int n = w.n;
	const int64_t n2 = (int64_t)n * n;
	double *A = Ascr + w.aofs;
	const double *V = Vscr + w.aofs;
	double *Tm = Tmp + w.tofs;
	GemmArgs<double, double> g;
	g.d = nullptr; g.E = nullptr; g.ei = 0; g.ej = 0; g.beta = 0.0; g.alpha = 1.0;
	g.M = n; g.N = n; g.K = n;
	g.P = A; g.pk = n; g.pi = 1;
	g.Q = V; g.qk = 1; g.qj = n;
	g.C = Tm; g.ci = 1; g.cj = n;
	block_gemm(g, ps, qs);
	for (int64_t e = threadIdx.x; e < n2; e += blockDim.x) A[e] = Tm[e];
}

// Blocked-mode T formation: T = U V^T with U, V in global scratch (one CTA per searchlight).
template <typename Real>
__global__ void __launch_bounds__(256) k_form_t_global(const SlWork *__restrict__ work, const Real *__restrict__ Ascr,
                                                       const Real *__restrict__ Vscr, float *__restrict__ Tscr,
                                                       const SlStats *__restrict__ stats, int t_rowmajor,
                                                       int only_flagged) {
	__shared__ Real ps[16][65], qs[16][65];
	const SlWork w = work[blockIdx.x];
	if (w.nblk == 2) return;
	if (only_flagged && !(stats[w.slot].flags & kFlagIllCond)) return;
	const int n = w.n;
	GemmArgs<Real, float> g;
	g.M = n; g.N = n; g.K = n;
	g.P = Ascr + w.aofs; g.pk = n; g.pi = 1;
	g.Q = Vscr + w.aofs; g.qk = n; g.qj = 1;
	g.d = nullptr; g.alpha = Real(1);
	g.E = nullptr; g.ei = 0; g.ej = 0; g.beta = 0;
	g.C = Tscr + w.tofs;
	g.ci = t_rowmajor ? n : 1;
	g.cj = t_rowmajor ? 1 : n;
	block_gemm(g, ps, qs);
}

// ---------------------------------------------------------------------------------------------
// Newton-Schulz orthogonality refinement  T <- T (3 I - T^T T) / 2   (float32)
// ---------------------------------------------------------------------------------------------
// T in the T scratch (row- or column-major), G = T^T T staged in Gs, result staged in Ws and
// copied back.  Searchlights solved in FP64 are skipped (already orthogonal to FP32 rounding).
__global__ void __launch_bounds__(256) k_ns_refine(const SlWork *__restrict__ work, float *__restrict__ Tscr,
                                                   float *__restrict__ Gscr, float *__restrict__ Wscr,
                                                   const SlStats *__restrict__ stats, int t_rowmajor) {
	__shared__ float ps[16][65], qs[16][65];
	const SlWork w = work[blockIdx.x];
	if (stats[w.slot].flags & kFlagFP64) return;
	const int n = w.n;
	float *T = Tscr + w.tofs;
	float *G = Gscr + w.aofs;
	float *W = Wscr + w.aofs;
	// element (i, j) of T at T[i*ti + j*tj]
	const int64_t ti = t_rowmajor ? n : 1, tj = t_rowmajor ? 1 : n;
	// G(a, b) = sum_i T(i, a) T(i, b) ; stored row-major
	GemmArgs<float> g;
	g.M = n; g.N = n; g.K = n;
	g.P = T; g.pk = ti; g.pi = tj;
	g.Q = T; g.qk = ti; g.qj = tj;
	g.d = nullptr; g.alpha = 1.0f;
	g.E = nullptr; g.ei = 0; g.ej = 0; g.beta = 0.0f;
	g.C = G; g.ci = n; g.cj = 1;
	block_gemm(g, ps, qs);
	// M = 1.5 I - 0.5 G  (in place)
	for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
		int a = (int)(e / n), b = (int)(e - (int64_t)a * n);
		G[e] = ((a == b) ? 1.5f : 0.0f) - 0.5f * G[e];
	}
	__syncthreads();
	// W(i, j) = sum_a T(i, a) M(a, j)
	g.P = T; g.pk = tj; g.pi = ti;
	g.Q = G; g.qk = n; g.qj = 1;
	g.C = W; g.ci = ti; g.cj = tj;
	block_gemm(g, ps, qs);
	for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) T[e] = W[e];
}

// ---------------------------------------------------------------------------------------------
// reflection fix (csrc/ha_searchlight.c:612-632): det(T) < 0 -> T -= 2 u_min v_min^T
// ---------------------------------------------------------------------------------------------
// sign(det T) from an LU factorisation with partial pivoting of a copy of T (T is orthogonal,
// so the factorisation is well conditioned).  Work copy in Wscr (float64, n*n per searchlight).
__global__ void __launch_bounds__(256) k_reflect_fix(const SlWork *__restrict__ work, float *__restrict__ Tscr,
                                                     double *__restrict__ Wscr, SlStats *__restrict__ stats,
                                                     const double *__restrict__ uvbuf, int t_rowmajor) {
	const SlWork w = work[blockIdx.x];
	const int n = w.n;
	float *T = Tscr + w.tofs;
	double *L = Wscr + w.aofs;  // column-major copy: L[c*n + r] = T(r, c)
	const int64_t ti = t_rowmajor ? n : 1, tj = t_rowmajor ? 1 : n;
	for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
		int c = (int)(e / n), r = (int)(e - (int64_t)c * n);
		L[e] = (double)T[r * ti + c * tj];
	}
	__syncthreads();
	__shared__ double pv[32];
	__shared__ int pr[32];
	__shared__ int piv_row;
	__shared__ double sign_acc;
	if (threadIdx.x == 0) sign_acc = 1.0;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	for (int k = 0; k < n; k++) {
		// pivot search in column k, rows k..n-1
		double best = -1.0;
		int bi = k;
		for (int r = k + threadIdx.x; r < n; r += blockDim.x) {
			double v = fabs(L[(int64_t)k * n + r]);
			if (v > best) { best = v; bi = r; }
		}
		for (int o = 16; o > 0; o >>= 1) {
			double ob = __shfl_xor_sync(0xffffffffu, best, o);
			int oi = __shfl_xor_sync(0xffffffffu, bi, o);
			if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
		}
		if (lane == 0) { pv[warp] = best; pr[warp] = bi; }
		__syncthreads();
		if (threadIdx.x == 0) {
			double b = -1.0;
			int i = k;
			for (int q = 0; q < nwarp; q++)
				if (pv[q] > b || (pv[q] == b && pr[q] < i)) { b = pv[q]; i = pr[q]; }
			piv_row = i;
			if (i != k) sign_acc = -sign_acc;
		}
		__syncthreads();
		int p = piv_row;
		if (p != k)
			for (int c = threadIdx.x; c < n; c += blockDim.x) {
				double a = L[(int64_t)c * n + k];
				L[(int64_t)c * n + k] = L[(int64_t)c * n + p];
				L[(int64_t)c * n + p] = a;
			}
		__syncthreads();
		double d = L[(int64_t)k * n + k];
		if (threadIdx.x == 0 && d < 0) sign_acc = -sign_acc;
		if (d != 0.0) {
			for (int r = k + 1 + threadIdx.x; r < n; r += blockDim.x) L[(int64_t)k * n + r] /= d;
			__syncthreads();
			for (int64_t e = threadIdx.x; e < (int64_t)(n - k - 1) * (n - k - 1); e += blockDim.x) {
				int cc = (int)(e / (n - k - 1)), rr = (int)(e - (int64_t)cc * (n - k - 1));
				int c = k + 1 + cc, r = k + 1 + rr;
				L[(int64_t)c * n + r] -= L[(int64_t)k * n + r] * L[(int64_t)c * n + k];
			}
		}
		__syncthreads();
	}
	if (sign_acc < 0) {
		const double *u = uvbuf + w.uvofs;
		const double *v = u + n;
		for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
			int i = (int)(e / n), j = (int)(e - (int64_t)i * n);
			T[i * ti + j * tj] = (float)((double)T[i * ti + j * tj] - 2.0 * u[i] * v[j]);
		}
		if (threadIdx.x == 0) {
			SlStats st = stats[w.slot];
			st.s_sum -= 2.0 * st.s_min;
			st.flags |= kFlagReflected;
			stats[w.slot] = st;
		}
	}
}

// ---------------------------------------------------------------------------------------------
// per-searchlight coefficient: scale = s_sum / (var_sum * nt) (csrc/ha_searchlight.c:635-656)
// ---------------------------------------------------------------------------------------------
__global__ void k_scale(const SlWork *__restrict__ work, int nwork, const int32_t *__restrict__ sl_idx,
                        const double *__restrict__ var_over_nt, const SlStats *__restrict__ stats, int nt,
                        int scaling, double *__restrict__ scale_out) {
	int q = blockIdx.x * blockDim.x + threadIdx.x;
	if (q >= nwork) return;
	const SlWork w = work[q];
	double sc = 1.0;
	if (scaling) {
		const int32_t *sl = sl_idx + w.sofs;
		double var_sum = 0.0;
		for (int j = 0; j < w.n; j++) var_sum = __dadd_rn(var_sum, var_over_nt[sl[j]]);
		sc = stats[w.slot].s_sum / (var_sum * nt);
	}
	scale_out[w.slot] = sc;
}

// ---------------------------------------------------------------------------------------------
// symmetric CSC / CSR pattern of the union of sl x sl blocks (csrc/ha_sparse.c:31-112)
// ---------------------------------------------------------------------------------------------
// Row (= column) v of the pattern is the set of vertices sharing a searchlight with v.
// One CTA per vertex marks them in a shared-memory bitmap of nv bits (restricted to the
// [lo, hi] window of vertices it can reach), then counts (pass 0) or writes them in
// ascending order (pass 1).  No pair enumeration, no sort.
__global__ void k_pattern(const int64_t *__restrict__ vl_ptr, const int2 *__restrict__ vl_ent,
                          const int32_t *__restrict__ sl_off, const int32_t *__restrict__ sl_idx,
                          const int32_t *__restrict__ sl_lo, const int32_t *__restrict__ sl_hi, int nv,
                          int pass, int64_t *__restrict__ row_len, const int64_t *__restrict__ row_ptr,
                          int32_t *__restrict__ cols) {
	extern __shared__ uint32_t bm[];
	__shared__ int s_lo, s_hi;
	__shared__ int64_t wsum[33];
	const int v = blockIdx.x;
	const int64_t e0 = vl_ptr[v], e1 = vl_ptr[v + 1];
	if (threadIdx.x == 0) { s_lo = nv; s_hi = -1; }
	__syncthreads();
	// window of reachable vertices
	for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
		int s = vl_ent[e].x;
		atomicMin(&s_lo, sl_lo[s]);
		atomicMax(&s_hi, sl_hi[s]);
	}
	__syncthreads();
	const int lo = s_lo & ~31, hi = s_hi;
	if (hi < lo) {
		if (pass == 0 && threadIdx.x == 0) row_len[v] = 0;
		return;
	}
	const int nwords = (hi - lo) / 32 + 1;
	for (int q = threadIdx.x; q < nwords; q += blockDim.x) bm[q] = 0u;
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	for (int64_t e = e0 + warp; e < e1; e += nwarp) {
		int s = vl_ent[e].x;
		int a0 = sl_off[s], a1 = sl_off[s + 1];
		for (int a = a0 + lane; a < a1; a += 32) {
			int u = sl_idx[a] - lo;
			atomicOr(&bm[u >> 5], 1u << (u & 31));
		}
	}
	__syncthreads();
	// per-thread contiguous word ranges -> prefix sum of popcounts
	const int per = (nwords + blockDim.x - 1) / blockDim.x;
	const int q0 = threadIdx.x * per, q1 = min(nwords, q0 + per);
	int64_t cnt = 0;
	for (int q = q0; q < q1; q++) cnt += __popc(bm[q]);
	// block exclusive scan of cnt
	int64_t incl = cnt;
	for (int o = 1; o < 32; o <<= 1) {
		int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o) incl += y;
	}
	if (lane == 31) wsum[warp] = incl;
	__syncthreads();
	if (threadIdx.x == 0) {
		int64_t run = 0;
		for (int q = 0; q < nwarp; q++) {
			int64_t t = wsum[q];
			wsum[q] = run;
			run += t;
		}
		wsum[32] = run;
	}
	__syncthreads();
	if (pass == 0) {
		if (threadIdx.x == 0) row_len[v] = wsum[32];
		return;
	}
	int64_t pos = row_ptr[v] + wsum[warp] + incl - cnt;
	for (int q = q0; q < q1; q++) {
		uint32_t b = bm[q];
		while (b) {
			int bit = __ffs(b) - 1;
			b &= b - 1;
			cols[pos++] = lo + q * 32 + bit;
		}
	}
}

// ---------------------------------------------------------------------------------------------
// deterministic segmented reduction into the pattern's values
// ---------------------------------------------------------------------------------------------
// One CTA per vertex v.  Its entries (s, a) (v is member a of searchlight s) are sorted by s;
// those of the current chunk [s_lo, s_hi) are visited in that order, and for each one the
// whole row a of the searchlight's M_s (M_s = T_s for CSR output, T_s^T for CSC output) is
// added at the slots of its columns, found by binary search in v's sorted pattern row.
// Within one searchlight the columns are distinct, so threads never collide; a barrier
// separates searchlights, so every sum runs in ascending searchlight order on every run.
//   CSR (row v = dense row v):   val(v, u_b) += w_s[a] * scale_s * T_s[a][b]
//   CSC (column v):              val(u_b, v) += w_s[b] * scale_s * T_s[b][a]
template <typename TT>
__global__ void __launch_bounds__(256) k_reduce(const int64_t *__restrict__ vl_ptr, const int2 *__restrict__ vl_ent,
                                                const int32_t *__restrict__ sl_off, const int32_t *__restrict__ sl_idx,
                                                const double *__restrict__ wts, const int64_t *__restrict__ pat_ptr,
                                                const int32_t *__restrict__ pat_col, const TT *__restrict__ Tscr,
                                                const int64_t *__restrict__ tofs_by_slot,
                                                const double *__restrict__ scale_by_slot, int s_lo, int s_hi,
                                                int csc, int smem_cap, double *__restrict__ values) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int v = blockIdx.x;
	const int64_t e0 = vl_ptr[v], e1 = vl_ptr[v + 1];
	// first entry with s >= s_lo (entries sorted by s)
	int64_t lo = e0, hi = e1;
	while (lo < hi) {
		int64_t mid = (lo + hi) >> 1;
		if (vl_ent[mid].x < s_lo) lo = mid + 1; else hi = mid;
	}
	const int64_t eb = lo;
	if (eb >= e1 || vl_ent[eb].x >= s_hi) return;
	const int64_t p0 = pat_ptr[v];
	const int L = (int)(pat_ptr[v + 1] - p0);
	const bool in_smem = L <= smem_cap;
	double *acc;
	const int32_t *cols;
	if (in_smem) {
		acc = reinterpret_cast<double *>(smem_raw);
		int32_t *cs = reinterpret_cast<int32_t *>(acc + L);
		for (int k = threadIdx.x; k < L; k += blockDim.x) {
			acc[k] = values[p0 + k];
			cs[k] = pat_col[p0 + k];
		}
		cols = cs;
		__syncthreads();
	} else {
		acc = values + p0;
		cols = pat_col + p0;
	}
	for (int64_t e = eb; e < e1; e++) {
		const int2 ent = vl_ent[e];
		const int s = ent.x;
		if (s >= s_hi) break;
		const int a = ent.y;
		const int o0 = sl_off[s];
		const int n = sl_off[s + 1] - o0;
		const int slot = s - s_lo;
		const TT *M = Tscr + tofs_by_slot[slot] + (int64_t)a * n;
		const double sc = scale_by_slot[slot];
		const double wa = wts ? wts[o0 + a] : 1.0;
		for (int b = threadIdx.x; b < n; b += blockDim.x) {
			const int u = sl_idx[o0 + b];
			int l = 0, h = L;
			while (l < h) {
				int mid = (l + h) >> 1;
				if (cols[mid] < u) l = mid + 1; else h = mid;
			}
			double wgt = csc ? (wts ? wts[o0 + b] : 1.0) : wa;
			acc[l] += (double)M[b] * (wgt * sc);
		}
		__syncthreads();
	}
	if (in_smem) {
		for (int k = threadIdx.x; k < L; k += blockDim.x) values[p0 + k] = acc[k];
	}
}

// ---------------------------------------------------------------------------------------------
// ridge  beta_s = (X_s^T X_s + alpha I)^-1 X_s^T Y_s   (csrc/ha_ridge.c:13-54, float64)
// ---------------------------------------------------------------------------------------------
// The reference computes V diag(s / (alpha + s^2)) U^T Y from the thin SVD X_s = U diag(s) V^T;
// for alpha > 0 that is exactly the solution of the regularised normal equations, solved here
// by a Cholesky factorisation of G + alpha I (G = X_s^T X_s in the A scratch, column-major) and
// two triangular solves with the n right-hand sides X_s^T Y_s (in the V scratch, column-major:
// column j holds right-hand side j).  One CTA per searchlight, float64 throughout, the factor
// overwriting G in place.  beta is written (float64) in the T layout: row-major for CSR output
// (row i = source vertex i), column-major for CSC output.  A non-positive pivot (alpha = 0 with a
// rank-deficient X_s) marks the searchlight kFlagUnconverged and writes zeros.
__global__ void __launch_bounds__(256) k_ridge_chol(const SlWork *__restrict__ work, double *__restrict__ Gscr,
                                                    double *__restrict__ Rscr, double *__restrict__ Bout, double alpha,
                                                    int t_rowmajor, SlStats *__restrict__ stats) {
	const SlWork w = work[blockIdx.x];
	const int n = w.n;
	double *G = Gscr + w.aofs;  // G[c * n + r] = G(r, c); lower triangle used
	double *R = Rscr + w.aofs;  // R[j * n + i] = rhs(i, j)
	__shared__ int bad;
	__shared__ double piv;
	if (threadIdx.x == 0) bad = 0;
	for (int k = threadIdx.x; k < n; k += blockDim.x) G[(int64_t)k * n + k] += alpha;
	__syncthreads();
	// right-looking Cholesky, column k at a time
	for (int k = 0; k < n; k++) {
		if (threadIdx.x == 0) {
			double d = G[(int64_t)k * n + k];
			if (!(d > 0.0)) {
				bad = 1;
				d = 1.0;
			}
			piv = sqrt(d);
			G[(int64_t)k * n + k] = piv;
		}
		__syncthreads();
		const double p = piv;
		for (int r = k + 1 + threadIdx.x; r < n; r += blockDim.x) G[(int64_t)k * n + r] /= p;
		__syncthreads();
		const int m = n - k - 1;
		for (int64_t e = threadIdx.x; e < (int64_t)m * m; e += blockDim.x) {
			const int c = k + 1 + (int)(e / m), r = k + 1 + (int)(e % m);
			if (r >= c) G[(int64_t)c * n + r] -= G[(int64_t)k * n + r] * G[(int64_t)k * n + c];
		}
		__syncthreads();
	}
	// forward solve L Z = rhs (all n right-hand sides), Z over R
	for (int k = 0; k < n; k++) {
		const double lkk = G[(int64_t)k * n + k];
		for (int j = threadIdx.x; j < n; j += blockDim.x) R[(int64_t)j * n + k] /= lkk;
		__syncthreads();
		const int m = n - k - 1;
		for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) {
			const int j = (int)(e / m), r = k + 1 + (int)(e % m);
			R[(int64_t)j * n + r] -= G[(int64_t)k * n + r] * R[(int64_t)j * n + k];
		}
		__syncthreads();
	}
	// backward solve L^T beta = Z
	for (int k = n - 1; k >= 0; k--) {
		const double lkk = G[(int64_t)k * n + k];
		for (int j = threadIdx.x; j < n; j += blockDim.x) R[(int64_t)j * n + k] /= lkk;
		__syncthreads();
		for (int64_t e = threadIdx.x; e < (int64_t)k * n; e += blockDim.x) {
			const int j = (int)(e / k), r = (int)(e % k);
			R[(int64_t)j * n + r] -= G[(int64_t)r * n + k] * R[(int64_t)j * n + k];
		}
		__syncthreads();
	}
	double *Bo = Bout + w.tofs;
	const int64_t ti = t_rowmajor ? n : 1, tj = t_rowmajor ? 1 : n;
	for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
		const int j = (int)(e / n), i = (int)(e % n);
		Bo[i * ti + j * tj] = bad ? 0.0 : R[e];
	}
	if (threadIdx.x == 0) {
		SlStats st = stats[w.slot];
		st.s_sum = 0.0;
		st.flags = bad ? (kFlagUnconverged | kFlagFP64) : kFlagFP64;
		stats[w.slot] = st;
	}
}

// ---------------------------------------------------------------------------------------------
// template loop helpers (csrc/ha_template.c:14-114 with searchlight solves)
// ---------------------------------------------------------------------------------------------

// out[:, c] = sum_k vals[ptr[c] + k] * X[:, col[ptr[c] + k]]  for every column c, i.e. X @ T with T
// given in CSC order over the symmetric pattern.  X, out: float64 vertex-major [nv][nt].  One
// CTA per output column, threads over time samples; the sum runs in pattern order.
__global__ void k_spmm_csc(const double *__restrict__ X, int nt, int nv, const int64_t *__restrict__ ptr,
                           const int32_t *__restrict__ col, const double *__restrict__ vals, double *__restrict__ out) {
	const int c = blockIdx.x;
	const int64_t k0 = ptr[c], k1 = ptr[c + 1];
	for (int t = threadIdx.x; t < nt; t += blockDim.x) {
		double acc = 0.0;
		for (int64_t k = k0; k < k1; k++) acc += vals[k] * X[(int64_t)col[k] * nt + t];
		out[(int64_t)c * nt + t] = acc;
	}
}

// Vertex-wise correlation of A with Y, the evaluation of benchmark_neuroboros.py:204-211 (mean
// over time of zscore(A)[:, c] * zscore(Y)[:, c] with population statistics), where A = X @ W for W
// in CSC form (ptr, row, vals) or A = X when vals is null. One warp per column c, lanes over time,
// two passes: the means, then the centred sums, r = sum(da dy) / sqrt(sum(da^2) sum(dy^2)). A column
// with zero variance gives 0 / 0 = NaN, as the z-score does. Pattern entries are checked before use:
// a column whose range lies outside [0, nnz] or decreases, or holds a row outside [0, nv), gets NaN
// and reads nothing. aligned (may be null) receives A; pass 2 reads it back instead of recomputing.
__global__ void k_aligned_corr(const double *__restrict__ X, const double *__restrict__ Y, int nt, int nv,
                               const int64_t *__restrict__ ptr, const int32_t *__restrict__ row,
                               const double *__restrict__ vals, int64_t nnz, double *__restrict__ r,
                               double *__restrict__ aligned) {
	const int lane = threadIdx.x & 31;
	const int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	if (c >= nv) return;  // whole warps leave together: c is the same for every lane of a warp
	const int64_t off = c * (int64_t)nt;
	int64_t k0 = 0, k1 = 0;
	if (vals) {
		k0 = ptr[c];
		k1 = ptr[c + 1];
		int ok = (k0 >= 0 && k1 >= k0 && k1 <= nnz) ? 1 : 0;
		if (ok)
			for (int64_t k = k0 + lane; k < k1; k += 32) ok &= (row[k] >= 0 && row[k] < nv) ? 1 : 0;
		if (!__all_sync(0xffffffffu, ok)) {
			const double nan = __longlong_as_double(0x7ff8000000000000LL);
			if (lane == 0) r[c] = nan;
			if (aligned)
				for (int t = lane; t < nt; t += 32) aligned[off + t] = nan;
			return;
		}
	}
	auto value = [&](int t) -> double {
		if (!vals) return X[off + t];
		double acc = 0.0;
		for (int64_t k = k0; k < k1; k++) acc = fma(vals[k], X[(int64_t)row[k] * nt + t], acc);
		return acc;
	};
	const double *y = Y + off;
	double sa = 0.0, sy = 0.0;
	for (int t = lane; t < nt; t += 32) {
		const double a = value(t);
		if (aligned) aligned[off + t] = a;
		sa += a;
		sy += y[t];
	}
	sa = warp_sum(sa);
	sy = warp_sum(sy);
	const double ma = sa / nt, my = sy / nt;
	double saa = 0.0, syy = 0.0, say = 0.0;
	for (int t = lane; t < nt; t += 32) {
		const double da = (aligned ? aligned[off + t] : value(t)) - ma;  // written by this lane in pass 1
		const double dy = y[t] - my;
		saa = fma(da, da, saa);
		syy = fma(dy, dy, syy);
		say = fma(da, dy, say);
	}
	saa = warp_sum(saa);
	syy = warp_sum(syy);
	say = warp_sum(say);
	if (lane == 0) r[c] = say / sqrt(saa * syy);
}

// One-pass column z-score of csrc/ha_linalg.c:263-291 (population variance from E[x^2] - m^2,
// var < 1e-30 -> the column becomes 0), float64, one thread per column summing in time order.
__global__ void k_zscore_cols(double *__restrict__ X, int nt, int nv) {
	const int v = blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= nv) return;
	double *x = X + (int64_t)v * nt;
	double s = 0.0, s2 = 0.0;
	for (int i = 0; i < nt; i++) {
		s = __dadd_rn(s, x[i]);
		s2 = __dadd_rn(s2, __dmul_rn(x[i], x[i]));
	}
	const double inv_m = 1.0 / nt;
	const double mean = __dmul_rn(s, inv_m);
	const double var = __dsub_rn(__dmul_rn(s2, inv_m), __dmul_rn(mean, mean));
	const double is = (var < 1e-30) ? 0.0 : 1.0 / sqrt(var);
	for (int i = 0; i < nt; i++) x[i] = __dmul_rn(__dsub_rn(x[i], mean), is);
}

// y = a * (x + b * z) elementwise over n entries (z may be null: y = a * x)
__global__ void k_axpbz(double *__restrict__ y, const double *__restrict__ x, const double *__restrict__ z, double a,
                        double b, int64_t n) {
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
		const double v = z ? __dadd_rn(x[e], __dmul_rn(b, z[e])) : x[e];
		y[e] = __dmul_rn(a, v);
	}
}

}  // namespace hab200
