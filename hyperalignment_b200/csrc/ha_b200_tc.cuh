// ha_b200_tc.cuh -- tensor-core (tcgen05) kernels: split-BF16 cross-covariance and the
// Newton-Schulz polar iteration of the searchlight Procrustes solve.
//
// The reference forms A = X_sl^T Y_sl with cblas_dgemm and T = U V^T from dgesdd
// (csrc/ha_searchlight.c:581-609).  Here T is the polar factor of A, computed by the scaled
// Newton-Schulz iteration
//     X_0 = A / u,   G_k = X_k^T X_k,   X_{k+1} = X_k (c1_k I + c3_k G_k),
// (u >= sigma_max(A); c1 = 3a/2, c3 = -a^3/2 with a from a capped scaling schedule, a = 1 in the
// final phase) on the 5th-generation tensor cores, with FP32 accumulation in tensor memory and
// every FP32 operand split exactly into 16-bit parts:
//   * the cross-covariance (inputs of any range): three BF16 parts x = hi + mid + lo and the six
//     products hi*hi + hi*mid + mid*hi + mid*mid + hi*lo + lo*hi (the dropped terms are below
//     2^-32 relative);
//   * the iteration, whose operands are bounded (the iterate's singular values stay <= 1, so
//     |X| <= 1, and |P| = |c1 I + c3 X^T X| <= |c1| + |c3| < 5): two FP16 parts of x * 2^12,
//     hi = fp16(x 2^12), mid = fp16(x 2^12 - hi), 22 significant bits (values below 2^-15 keep an
//     absolute error under 2^-37), and the three products hi*hi + hi*mid + mid*hi (the dropped
//     mid*mid is 2^-22 relative); the accumulator holds 2^24 times the product.
//
// One CTA computes one 128-row tile of one searchlight's product: 128 threads stage K-slices of
// 16 with cp.async into a ring of shared-memory stages (canonical no-swizzle core-matrix
// layout: 8 rows x 16 bytes per core matrix), thread 0 issues tcgen05.mma (M = 128, N = the
// searchlight's padded size, K = 16) into tensor memory and commits each stage to an mbarrier,
// and the four warps read the accumulator back with tcgen05.ld for the epilogue.
//
// Storage of a searchlight's iterate X and of P = c1 I + c3 G in HBM: two FP16 planes of
// np x np (np = n rounded up to 16), each in 8 x 8 core matrices, core (r, c) = rows 8r..8r+7,
// columns 8c..8c+7 at element offset (r * np/8 + c) * 64, row-major inside (16 bytes a row).
// The iterate alternates between two buffers (the update reads one and writes the other).
// The same bytes serve as a K-major operand (X in X P) and as an MN-major operand (X in X^T X,
// P in X P), so no transposed copy exists.  Padding rows and columns are zero and stay zero.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ha_b200_kernels.cuh"

namespace hab200 {

constexpr int kTcThreads = 128;
constexpr int kTcMaxStages = 8;
constexpr int kTcMaxNp = 512;                  // largest padded searchlight size (four 128-row tiles)
constexpr int kTcResSlots = 32;                // residual partials per searchlight: row tiles x column halves x warps
constexpr uint64_t kTcWaitNs = 2000000000ull;  // a pipeline wait longer than 2 s is declared failed

enum : int { kTcPhaseXcov = 0, kTcPhaseGram = 1, kTcPhaseUpdate = 2 };

constexpr float kTcOpScale = 4096.f;                 // iteration operands are stored as x * 2^12
constexpr float kTcAccUnscale = 1.f / 16777216.f;    // 2^-24: the iteration's accumulator -> product

// 16-bit planes per operand: three BF16 parts for the cross-covariance, two FP16 parts for the
// iteration's Gram and update products.
template <int PHASE>
struct TcFmt {
	static constexpr int planes = PHASE == kTcPhaseXcov ? 3 : 2;
};

// One searchlight of the tensor-core solve.
struct TcWork {
	int32_t s;     // searchlight index
	int32_t slot;  // index within the chunk (stats, state, residual slots)
	int32_t n;     // size
	int32_t np;    // n rounded up to 16
	int32_t sofs;  // flat offset of the searchlight in sl_indices
	int32_t pad_;
	int64_t xofs;  // 16-bit element offset of the iterate's two planes (2 np^2)
	int64_t pofs;  // 16-bit element offset of P's two planes
	int64_t aofs;  // float element offset of A (np x np, row-major, leading dimension np)
	int64_t tofs;  // float element offset of T in the T scratch (n x n)
};

// One CTA's output tile: 128 rows x nn columns starting at column n0 (nn <= 256; searchlights with
// np > 256 have two column halves, so every tile fits two CTAs per SM).
struct TcTile {
	int32_t w;   // work index
	int32_t t;   // 128-row tile
	int32_t n0;  // first column
	int32_t nn;  // columns (a multiple of 16)
};

// Per-searchlight iteration state; one copy is read and the other written by each update launch.
struct TcState {
	int32_t plain;  // the last update used the plain coefficients (a = 1)
	int32_t done;   // T written; no further work
	int32_t iters;  // iterations taken
	int32_t conv;   // residual fell below the stop threshold
	float res;        // ||G - I||_F / sqrt(n) of the last Gram product
	float u;          // the upper bound of sigma_max(A) that X_0 was scaled by
	int32_t stalled;  // plain steps stopped changing the residual: some singular values stay zero
	float pad_;
};

struct TcArgs {
	const TcWork *work;
	const TcTile *tiles;
	// cross-covariance: vertex-major bf16 planes [plane][nv][ntp], ntp = nt rounded up to 16
	const __nv_bfloat16 *Xb;
	const __nv_bfloat16 *Yb;
	int64_t vplane;  // elements per vertex-major plane (nv * ntp)
	int ntp;
	const int32_t *sl_idx;
	// Newton-Schulz
	__nv_bfloat16 *Xp;  // iterate planes (offsets from TcWork::xofs), read
	__nv_bfloat16 *Xw;  // where the update writes the next iterate: the other of two buffers, since the
	                    // two column halves of a row tile both read the whole row tile of X
	__nv_bfloat16 *Pp;  // P planes (TcWork::pofs)
	float *A32;         // cross-covariance (TcWork::aofs)
	float *T;           // T scratch (TcWork::tofs)
	int t_rowmajor;
	const TcState *st_in;
	TcState *st_out;
	float *res_part;  // [slot][kTcResSlots]
	float c1, c3;     // schedule coefficients of this iteration
	int plain;        // c1 = 3/2, c3 = -1/2 exactly (convergence is only accepted on such an iteration)
	int last;         // the iteration limit: this update is final for every searchlight
	float tol_stop;   // stop once ||G - I||_F / sqrt(n) is below this (after one more update)
	int smem_bytes;   // dynamic shared memory of the launch
	int *err;         // set when a wait times out
};

// ---------------------------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
	uint32_t ok;
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	    "selp.u32 %0, 1, 0, p;\n\t}"
	    : "=r"(ok)
	    : "r"(smem_u32(bar)), "r"(parity)
	    : "memory");
	return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Bounded wait for phase `parity` of an mbarrier: false once kTcWaitNs have passed.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
	if (mbar_try_wait(bar, parity)) return true;
	const uint64_t t0 = global_ns();
	while (!mbar_try_wait(bar, parity))
		if (global_ns() - t0 > kTcWaitNs) return false;
	return true;
}

// One arrival on `bar` that also expects `bytes` of bulk copies to land before its phase ends.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
	             : "memory");
}

// `bytes` more bulk-copy bytes for the current phase of `bar`, without an arrival.
__device__ __forceinline__ void mbar_add_tx(uint64_t *bar, uint32_t bytes) {
	asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// An arrival on `bar` once every cp.async this thread has issued so far has completed (the
// barrier's expected count includes it).
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
	asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One plain arrival on `bar`.
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global memory into
// this CTA's shared memory; its completion counts against the transaction bytes of `bar`.  A plain
// copy into the CTA's own shared memory: no multicast.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint64_t *bar) {
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
	             "l"(src), "r"(bytes), "r"(smem_u32(bar))
	             : "memory");
}

// The same bounded wait for threads with nothing else to do meanwhile: a short sleep between
// polls leaves the issue slots to the warps that produce and consume the stages.
__device__ __forceinline__ bool mbar_wait_idle(uint64_t *bar, uint32_t parity) {
	if (mbar_try_wait(bar, parity)) return true;
	const uint64_t t0 = global_ns();
	while (!mbar_try_wait(bar, parity)) {
		__nanosleep(64);
		if (global_ns() - t0 > kTcWaitNs) return false;
	}
	return true;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes) {
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_keep(int keep) {
	// wait until at most `keep` groups are pending (immediate operand, so one branch per value)
	if (keep <= 0)
		asm volatile("cp.async.wait_group 0;" ::: "memory");
	else if (keep == 1)
		asm volatile("cp.async.wait_group 1;" ::: "memory");
	else if (keep == 2)
		asm volatile("cp.async.wait_group 2;" ::: "memory");
	else if (keep == 3)
		asm volatile("cp.async.wait_group 3;" ::: "memory");
	else if (keep == 4)
		asm volatile("cp.async.wait_group 4;" ::: "memory");
	else if (keep == 5)
		asm volatile("cp.async.wait_group 5;" ::: "memory");
	else
		asm volatile("cp.async.wait_group 6;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Warp-wide: allocate `ncols` (power of two >= 32) tensor-memory columns; the base address is
// written to shared memory at `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
	             : "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor, no swizzle: start address, leading byte offset (between
// core matrices adjacent in K), stride byte offset (between core matrices adjacent in M/N),
// descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
	uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
	d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
	d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
	d |= (uint64_t)1 << 46;
	return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B and an FP32 accumulator.
// f16: A and B are FP16 (type field 0) instead of BF16 (type field 1); both operands always share
// one type.
__host__ __device__ __forceinline__ uint32_t mma_idesc(int M, int N, int a_mn, int b_mn, bool f16 = false) {
	return (1u << 4) | (f16 ? 0u : ((1u << 7) | (1u << 10))) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
	       ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
	    "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
	    : "memory");
}

// Arrive on `bar` once every tcgen05.mma issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
	             : "memory");
}

// Warp-wide: 16 consecutive FP32 columns of this warp's 32 tensor-memory lanes (lane i of the
// warp gets row 32 * (warp % 4) + i).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
	uint32_t r[16];
	asm volatile(
	    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
	    "%15}, [%16];"
	    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	    : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Warp-wide: 64 consecutive FP32 columns of this warp's 32 tensor-memory lanes, one load and one
// wait (the wait is inside the same statement, so no use of the registers can precede it).
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
	uint32_t r[64];
	asm volatile(
	    "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n\t"
	    "tcgen05.wait::ld.sync.aligned;"
	    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
	      "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
	      "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
	      "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
	      "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
	      "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
	      "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
	    : "r"(taddr)
	    : "memory");
#pragma unroll
	for (int i = 0; i < 64; i++) v[i] = __uint_as_float(r[i]);
}

// Exact three-way split of an FP32 value into BF16 parts: v = hi + mid + lo.
__device__ __forceinline__ void split3(float v, __nv_bfloat16 &hi, __nv_bfloat16 &mid, __nv_bfloat16 &lo) {
	hi = __float2bfloat16_rn(v);
	const float r1 = v - __bfloat162float(hi);
	mid = __float2bfloat16_rn(r1);
	lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
}

// Eight consecutive FP32 values of one core-matrix row of an iteration operand -> 16 bytes in each
// of the two FP16 planes: hi = fp16(x 2^12), mid = fp16(x 2^12 - hi) (the difference is exact in
// FP32).
__device__ __forceinline__ void store_split8h(const float *v, __nv_bfloat16 *p0, __nv_bfloat16 *p1) {
	__half2 h[4], m[4];
#pragma unroll
	for (int i = 0; i < 4; i++) {
		const float a = v[2 * i] * kTcOpScale, b = v[2 * i + 1] * kTcOpScale;
		h[i] = __floats2half2_rn(a, b);
		m[i] = __floats2half2_rn(a - __low2float(h[i]), b - __high2float(h[i]));
	}
	*reinterpret_cast<uint4 *>(p0) = *reinterpret_cast<const uint4 *>(h);
	*reinterpret_cast<uint4 *>(p1) = *reinterpret_cast<const uint4 *>(m);
}

// Bytes of one pipeline stage for an N-column product: A (128 x 16) and B (N x 16), `planes` each.
__host__ __device__ __forceinline__ int tc_stage_bytes(int N, int planes) {
	return planes * (128 * 16 * 2) + planes * (N * 16 * 2);
}

// tensor-memory columns for an N-column FP32 accumulator
__device__ __forceinline__ uint32_t tc_tmem_cols(int N) {
	uint32_t c = 32;
	while ((int)c < N) c <<= 1;
	return c;
}

// ---------------------------------------------------------------------------------------------
// stage loads
// ---------------------------------------------------------------------------------------------
// Stage layout (bytes), NPL planes per operand: A plane p at p * 4096, B plane p at NPL * 4096 +
// p * 32 N.  Inside a plane,
// core matrix (g, k) (g: 8-row group along M or N, k: which 8-element half of the K-slice) sits at
// (g * 2 + k) * 128, so LBO = 128 and SBO = 256 for both operand majors.

// Per-thread load plan of one tile: the thread's chunks (16 bytes each) of one plane's A and B
// stages, with their shared-memory offsets and their source element offsets at K-slice 0.  Every
// source offset grows linearly with the K-slice (by strideA / strideB elements), so a K-slice's
// loads are one add and one cp.async per chunk and plane.  Chunk c of A (256 per plane) is row
// r = c & 7 of core matrix c >> 3 = (g, k) = (8-row group, K half); B has 2N chunks per plane.
constexpr int kTcMaxBChunks = 8;  // 2N / 128 for N <= 512
struct TcLoadPlan {
	uint32_t dA[2], dB[kTcMaxBChunks];
	int32_t sA[2], sB[kTcMaxBChunks];  // -1: zero fill
	int nB;
	int32_t strideA, strideB;
};

// PHASE kTcPhaseXcov: sources are vertex rows of the vertex-major planes (s_sl: the searchlight's
// vertices); Gram / update: core-tiled planes of the searchlight (npg = np / 8 core groups).
template <int PHASE>
__device__ __forceinline__ void tc_plan_tile(TcLoadPlan &lp, const int32_t *s_sl, int n, int np, int ntp, int t,
                                             int n0, int N) {
	const int npg = np >> 3, g0 = n0 >> 3, tid = threadIdx.x;
#pragma unroll
	for (int i = 0; i < 2; i++) {
		const int c = tid + 128 * i, core = c >> 3, r = c & 7, g = core >> 1, k = core & 1;
		lp.dA[i] = (uint32_t)(core * 128 + r * 16);
		if (PHASE == kTcPhaseXcov) {
			const int row = 128 * t + 8 * g + r;
			lp.sA[i] = row < n ? s_sl[row] * ntp + 8 * k : -1;
		} else if (PHASE == kTcPhaseGram) {
			lp.sA[i] = (16 * t + g < npg) ? (k * npg + 16 * t + g) * 64 + 8 * r : -1;
		} else {
			lp.sA[i] = (16 * t + g < npg) ? ((16 * t + g) * npg + k) * 64 + 8 * r : -1;
		}
	}
	lp.nB = (2 * N + 127) >> 7;
#pragma unroll
	for (int j = 0; j < kTcMaxBChunks; j++) {
		const int c = tid + 128 * j, core = c >> 3, r = c & 7, g = core >> 1, k = core & 1;
		lp.dB[j] = (uint32_t)(core * 128 + r * 16);
		if (c >= 2 * N) lp.sB[j] = -2;  // not a chunk of this tile
		else if (PHASE == kTcPhaseXcov) lp.sB[j] = (n0 + 8 * g + r) < n ? s_sl[n0 + 8 * g + r] * ntp + 8 * k : -1;
		else lp.sB[j] = (k * npg + g0 + g) * 64 + 8 * r;
	}
	lp.strideA = (PHASE == kTcPhaseXcov) ? 16 : (PHASE == kTcPhaseGram) ? 128 * npg : 128;
	lp.strideB = (PHASE == kTcPhaseXcov) ? 16 : 128 * npg;
}

// Issue the cp.async copies of K-slice ks into the stage at shared address `stage`.  A planes at
// A + p * pstrideA, B planes at B + p * pstrideB (elements).
template <int NPL>
__device__ __forceinline__ void tc_load_slice(const TcLoadPlan &lp, const __nv_bfloat16 *A, int64_t pstrideA,
                                              const __nv_bfloat16 *B, int64_t pstrideB, int N, int ks,
                                              uint32_t stage) {
	const int32_t oa = ks * lp.strideA, ob = ks * lp.strideB;
#pragma unroll
	for (int p = 0; p < NPL; p++) {
		const __nv_bfloat16 *Ap = A + p * pstrideA;
		const __nv_bfloat16 *Bp = B + p * pstrideB;
		const uint32_t sa = stage + p * 4096, sb = stage + NPL * 4096 + p * 32 * N;
#pragma unroll
		for (int i = 0; i < 2; i++) {
			const bool ok = lp.sA[i] >= 0;
			cp_async16(sa + lp.dA[i], ok ? Ap + lp.sA[i] + oa : Ap, ok ? 16u : 0u);
		}
#pragma unroll
		for (int j = 0; j < kTcMaxBChunks; j++) {
			if (j >= lp.nB || lp.sB[j] == -2) break;
			const bool ok = lp.sB[j] >= 0;
			cp_async16(sb + lp.dB[j], ok ? Bp + lp.sB[j] + ob : Bp, ok ? 16u : 0u);
		}
	}
}

// The products of one K-slice staged at shared address `st` into the accumulator at `tmem`
// (columns 0..255 and, for N > 256, 256..N-1), smallest first.  Issued by one thread.
// Stage layouts: the per-thread loads put core matrix (g, k) (g along M or N, k the K half) at
// (2 g + k) * 128 in every operand (LBO 128 between the K halves, SBO 256 between 8-row groups).
// The bulk-copy pipeline (BULK) keeps that layout for the update's K-major A, whose K halves are
// adjacent in memory, and puts the MN-major operands (the Gram's A, every B) K half by K half:
// core (g, k) at (k G + g) * 128 with G the operand's 8-row groups (16 for A, N / 8 for B), so each
// K half of a plane is one contiguous copy (LBO G * 128, SBO 128).
// A_KH / B_KH: the operand is staged K half by K half (else interleaved); by default the bulk form's
// choice.  The persistent iteration kernel stages A interleaved (per-lane copies) and B by K halves.
template <int PHASE, bool BULK = false, bool A_KH = BULK && PHASE == kTcPhaseGram, bool B_KH = BULK>
__device__ __forceinline__ void tc_issue_products(uint32_t tmem, uint32_t st, int N, uint32_t id0, uint32_t id1,
                                                  bool first) {
	constexpr int NPL = TcFmt<PHASE>::planes;
	constexpr int NQ = NPL == 3 ? 6 : 3;
	const uint32_t a_lbo = A_KH ? 2048u : 128u;
	const uint32_t a_sbo = A_KH ? 128u : 256u;
	const uint32_t b_lbo = B_KH ? 16u * N : 128u, b_sbo = B_KH ? 128u : 256u;
	const uint32_t b_half = B_KH ? 32u * 128u : 32u * 256u;  // 32 8-row groups: the second MMA's B
#pragma unroll
	for (int q = 0; q < NQ; q++) {
		// three planes: lo*hi, hi*lo, mid*mid, mid*hi, hi*mid, hi*hi; two: mid*hi, hi*mid, hi*hi
		const int pa = NPL == 3 ? ((q == 0) ? 2 : (q == 2 || q == 3) ? 1 : 0) : (q == 0 ? 1 : 0);
		const int pb = NPL == 3 ? ((q == 1) ? 2 : (q == 2 || q == 4) ? 1 : 0) : (q == 1 ? 1 : 0);
		const uint32_t acc = (!first || q > 0) ? 1u : 0u;
		const uint64_t ad = smem_desc(st + pa * 4096, a_lbo, a_sbo);
		const uint32_t baddr = st + NPL * 4096 + pb * 32 * N;
		mma_bf16(tmem, ad, smem_desc(baddr, b_lbo, b_sbo), id0, acc);
		if (N > 256) mma_bf16(tmem + 256, ad, smem_desc(baddr + b_half, b_lbo, b_sbo), id1, acc);
	}
}

// ---------------------------------------------------------------------------------------------
// the tile-product kernel
// ---------------------------------------------------------------------------------------------
// PHASE kTcPhaseXcov:   A32 = X_sl^T Y_sl                       (K = time, padded to 16)
// PHASE kTcPhaseGram:   P = c1 I + c3 X^T X, residual partials   (skips searchlights already done)
// PHASE kTcPhaseUpdate: X <- X P, or T = X P for the final update (decided from the residual)
// BULK (Gram and update only): warp-specialised stages filled by bulk copies instead of the
// per-thread loads (see the main loop).
template <int PHASE, bool BULK = false>
__global__ void __launch_bounds__(kTcThreads) k_tc_gemm(const TcArgs a) {
	static_assert(!(BULK && PHASE == kTcPhaseXcov), "the gathered cross-covariance has no bulk form");
	extern __shared__ __align__(128) unsigned char tc_smem[];
	__shared__ uint64_t s_bar[kTcMaxStages];   // stage consumed: the stage's products completed
	__shared__ uint64_t s_full[kTcMaxStages];  // stage filled (bulk form): its copies landed
	__shared__ uint64_t s_acc;
	__shared__ uint32_t s_tmem;
	__shared__ int s_fail;
	__shared__ int32_t s_sl[PHASE == kTcPhaseXcov ? kTcMaxNp : 1];

	const TcTile tl = a.tiles[blockIdx.x];
	const TcWork w = a.work[tl.w];
	const int n = w.n, np = w.np, t = tl.t;
	const int n0 = tl.n0, N = tl.nn;
	if (PHASE == kTcPhaseUpdate && a.Xw == nullptr) {  // no target for the next iterate: refuse
		if (threadIdx.x == 0) atomicOr(a.err, 1);
		return;
	}
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

	const float c1 = a.c1, c3 = a.c3;
	bool final_update = false;
	if (PHASE != kTcPhaseXcov) {
		const TcState st = a.st_in[w.slot];
		if (st.done) {
			if (PHASE == kTcPhaseUpdate && t == 0 && tid == 0) a.st_out[w.slot] = st;
			return;
		}
		if (PHASE == kTcPhaseUpdate) {
			// residual of this iteration's Gram product: fixed-order sum, identical in every tile CTA
			double ss = 0.0;
			for (int i = 0; i < kTcResSlots; i++) ss += (double)a.res_part[(int64_t)w.slot * kTcResSlots + i];
			const double resd = sqrt(ss / (double)n);
			const float res = (float)resd;
			const bool conv = a.plain && res < a.tol_stop;
			// A plain step multiplies every singular value sigma < 1 by about 3/2, which changes the
			// residual by about 2.5 sigma^2 / (n res^2) relative; a residual that a plain step leaves
			// unchanged to 5e-7 relative belongs to singular values below ~1e-3 after the schedule's
			// growth, i.e. below the FP32 resolution of A (exact zeros for duplicated or zero vertex
			// columns): stop here and let the completion kernel fill them.
			const bool stalled = !conv && a.plain && st.plain && fabs(resd - (double)st.res) <= 5e-7 * resd;
			final_update = conv || stalled || a.last;
			if (t == 0 && tid == 0) {
				TcState o = st;
				o.iters = st.iters + 1;
				o.res = res;
				o.conv = conv ? 1 : 0;
				o.stalled = stalled ? 1 : 0;
				o.done = final_update ? 1 : 0;
				o.plain = a.plain;
				a.st_out[w.slot] = o;
			}
		}
	}

	constexpr int NPL = TcFmt<PHASE>::planes;
	const int stage_bytes = tc_stage_bytes(N, NPL);
	int S = a.smem_bytes / stage_bytes;
	if (S > kTcMaxStages) S = kTcMaxStages;
	const int nk = (PHASE == kTcPhaseXcov) ? (a.ntp >> 4) : (np >> 4);
	const uint32_t ncols = tc_tmem_cols(N);
	const uint32_t smem0 = smem_u32(tc_smem);

	// bulk form: 8-row groups of the A tile inside the searchlight (the rest of A stays zero)
	const int gA = min(16, (np >> 3) - 16 * t);
	if (tid == 0) {
		for (int i = 0; i < kTcMaxStages; i++) {
			mbar_init(&s_bar[i], 1);
			mbar_init(&s_full[i], 1);
		}
		mbar_init(&s_acc, 1);
		s_fail = (S < 2) ? 1 : 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (PHASE == kTcPhaseXcov)
		for (int i = tid; i < n; i += kTcThreads) s_sl[i] = a.sl_idx[w.sofs + i];
	if (BULK && gA < 16 && S <= kTcMaxStages) {
		// the copies fill only the A rows inside the searchlight: zero every stage's A planes once
		for (int st = 0; st < S; st++)
			for (int e = tid; e < NPL * 4096 / 16; e += kTcThreads)
				reinterpret_cast<uint4 *>(tc_smem + st * stage_bytes)[e] = make_uint4(0u, 0u, 0u, 0u);
		fence_proxy_async_smem();
	}
	if (warp == 0) tmem_alloc(&s_tmem, ncols);
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = s_tmem;
	bool failed = s_fail != 0;

	const __nv_bfloat16 *Xs = a.Xp + w.xofs;
	const __nv_bfloat16 *Bs = (PHASE == kTcPhaseGram) ? Xs : (const __nv_bfloat16 *)(a.Pp + w.pofs);
	TcLoadPlan lp;
	tc_plan_tile<PHASE>(lp, s_sl, n, np, a.ntp, t, n0, N);
	const __nv_bfloat16 *srcA = (PHASE == kTcPhaseXcov) ? a.Xb : Xs;
	const __nv_bfloat16 *srcB = (PHASE == kTcPhaseXcov) ? a.Yb : Bs;
	const int64_t pstride = (PHASE == kTcPhaseXcov) ? a.vplane : (int64_t)np * np;
	auto load = [&](int ks, int s) {
		tc_load_slice<NPL>(lp, srcA, pstride, srcB, pstride, N, ks, smem0 + s * stage_bytes);
	};

	// operand majors: cross-covariance K/K, Gram MN/MN, update K/MN
	const int a_mn = (PHASE == kTcPhaseGram) ? 1 : 0;
	const int b_mn = (PHASE == kTcPhaseXcov) ? 0 : 1;
	const int N0 = N > 256 ? 256 : N;
	const bool f16 = PHASE != kTcPhaseXcov;
	const uint32_t id0 = mma_idesc(128, N0, a_mn, b_mn, f16);
	const uint32_t id1 = N > 256 ? mma_idesc(128, N - 256, a_mn, b_mn, f16) : 0u;

	if (BULK && !failed) {
		// Warp 0 fills stage ks % S with bulk copies (their bytes complete the stage's full barrier)
		// once the products of slice ks - S have released it; thread 32 issues each slice's products
		// as soon as its stage is full and commits them to the stage's consumed barrier.  Per slice
		// and plane: the Gram's A as two K halves of gA cores (contiguous along M), the update's A as
		// gA pairs of K-adjacent cores, B as two K halves of N / 8 cores.
		volatile int *vfail = &s_fail;
		const int64_t pe = (int64_t)np * np;
		const int npg = np >> 3, g0 = n0 >> 3;
		const uint32_t tx = 2u * (256u * (uint32_t)gA + 32u * (uint32_t)N);
		if (warp == 0) {
			// the producer warp: lane 0 waits for the stage and sets the expected bytes, then every
			// lane issues its share of the copies (one A part each; lanes 0-3 also the B parts)
			int issued = 0;
			for (int ks = 0; ks < nk; ks++) {
				const int s = ks % S;
				int ok = 1;
				if (lane == 0) {
					ok = !*vfail;
					if (ok && ks >= S && !mbar_wait(&s_bar[s], (uint32_t)((ks / S - 1) & 1))) {
						*vfail = 1;
						ok = 0;
					}
					if (ok) mbar_expect_tx(&s_full[s], tx);
				}
				if (!__shfl_sync(0xffffffffu, ok, 0)) break;
				const uint32_t st = smem0 + s * stage_bytes;
				const int p = lane >> 4, q = lane & 15;  // A part: plane p, core group q (update) or K half q (Gram)
				const __nv_bfloat16 *Ap = srcA + p * pe;
				const uint32_t sa = st + p * 4096;
				if (PHASE == kTcPhaseGram) {
					if (q < 2)
						bulk_g2s(sa + q * 2048, Ap + ((int64_t)(2 * ks + q) * npg + 16 * t) * 64, 128u * gA, &s_full[s]);
				} else if (q < gA) {
					bulk_g2s(sa + q * 256, Ap + ((int64_t)(16 * t + q) * npg + 2 * ks) * 64, 256u, &s_full[s]);
				}
				if (lane < 4) {  // B part: plane lane >> 1, K half lane & 1
					const int pb = lane >> 1, k = lane & 1;
					bulk_g2s(st + 2 * 4096 + pb * 32 * N + k * 16 * N,
					         srcB + pb * pe + ((int64_t)(2 * ks + k) * npg + g0) * 64, 16u * N, &s_full[s]);
				}
				issued = ks + 1;
			}
			// the copies still in flight must land before the CTA may leave
			if (lane == 0)
				for (int ks = issued > S ? issued - S : 0; ks < issued; ks++)
					if (!mbar_wait(&s_full[ks % S], (uint32_t)((ks / S) & 1))) *vfail = 1;
			__syncwarp();
		} else if (warp == 1) {
			// lane 0 issues; the other lanes wait at the warp barrier instead of polling beside it
			for (int ks = 0; ks < nk; ks++) {
				int ok = 1;
				if (lane == 0) {
					const int s = ks % S;
					if (mbar_wait(&s_full[s], (uint32_t)((ks / S) & 1))) {
						tc_fence_after();
						tc_issue_products<PHASE, true>(tmem, smem0 + s * stage_bytes, N, id0, id1, ks == 0);
						mma_commit(&s_bar[s]);
					} else {
						*vfail = 1;
						ok = 0;
					}
				}
				if (!__shfl_sync(0xffffffffu, ok, 0)) break;
			}
			if (lane == 0) mma_commit(&s_acc);  // tracks every product issued, also after a failed wait
			__syncwarp();
		}
	}
	if (!BULK && !failed) {
		for (int j = 0; j < S - 1; j++) {
			if (j < nk) load(j, j);
			cp_async_commit();
		}
		// K-slice ks: wait for its stage, issue its products, then refill the stage the products of
		// slice ks - 1 read (so slice ks stays queued on the tensor pipe while the refill waits)
		for (int ks = 0; ks < nk; ks++) {
			const int s = ks % S;
			cp_async_wait_keep(S - 2);
			fence_proxy_async_smem();
			__syncthreads();
			if (s_fail) { failed = true; break; }
			if (tid == 0) {
				tc_fence_after();
				tc_issue_products<PHASE>(tmem, smem0 + s * stage_bytes, N, id0, id1, ks == 0);
				mma_commit(&s_bar[s]);
			}
			const int kn = ks + S - 1;
			if (kn < nk) {
				// stage kn % S was last read by the products of K-slice ks - 1
				if (ks >= 1 && !mbar_wait(&s_bar[(ks - 1) % S], (uint32_t)(((ks - 1) / S) & 1))) s_fail = 1;
				load(kn, kn % S);
			}
			cp_async_commit();
		}
	}
	cp_async_wait_all();
	if (!failed) {
		if (!BULK && tid == 0) mma_commit(&s_acc);
		if (!(BULK ? mbar_wait_idle(&s_acc, 0) : mbar_wait(&s_acc, 0))) s_fail = 1;
	}
	__syncthreads();
	failed = failed || s_fail;
	tc_fence_after();

	if (!failed) {
		// epilogue: row m of the tile = tensor-memory lane m; warp w owns lanes 32w..32w+31
		const int m = 32 * warp + lane;
		const int row = 128 * t + m;
		const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
		const int npg = np >> 3;
		float res = 0.f;
		for (int c0 = 0; c0 < N; c0 += 16) {
			float v[16];
			tmem_ld16(trow + (uint32_t)c0, v);
			if (row >= np) continue;
			if (PHASE != kTcPhaseXcov) {
#pragma unroll
				for (int q = 0; q < 16; q++) v[q] *= kTcAccUnscale;
			}
			if (PHASE == kTcPhaseXcov) {
				if (row < n) {
					float4 *dst = reinterpret_cast<float4 *>(a.A32 + w.aofs + (int64_t)row * np + n0 + c0);
#pragma unroll
					for (int q = 0; q < 4; q++) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
				}
			} else if (PHASE == kTcPhaseGram) {
#pragma unroll
				for (int q = 0; q < 16; q++) {
					const int col = n0 + c0 + q;
					const float g = v[q];
					if (row < n && col < n) {
						const float d = g - (col == row ? 1.f : 0.f);
						res += d * d;
					}
					v[q] = c3 * g + (col == row ? c1 : 0.f);
				}
				__nv_bfloat16 *P0 = a.Pp + w.pofs;
				const int64_t pe = (int64_t)np * np;
#pragma unroll
				for (int h = 0; h < 2; h++) {
					const int64_t o = ((int64_t)(row >> 3) * npg + ((n0 + c0) >> 3) + h) * 64 + (row & 7) * 8;
					store_split8h(v + 8 * h, P0 + o, P0 + pe + o);
				}
			} else {
				if (final_update) {
					if (row < n) {
						float *T = a.T + w.tofs;
						for (int q = 0; q < 16; q++) {
							const int col = n0 + c0 + q;
							if (col < n) T[a.t_rowmajor ? (int64_t)row * n + col : (int64_t)col * n + row] = v[q];
						}
					}
				} else {
					__nv_bfloat16 *X0 = a.Xw + w.xofs;
					const int64_t pe = (int64_t)np * np;
#pragma unroll
					for (int h = 0; h < 2; h++) {
						const int64_t o = ((int64_t)(row >> 3) * npg + ((n0 + c0) >> 3) + h) * 64 + (row & 7) * 8;
						store_split8h(v + 8 * h, X0 + o, X0 + pe + o);
					}
				}
			}
		}
		if (PHASE == kTcPhaseGram) {
			res = warp_sum(res);
			if (lane == 0) a.res_part[(int64_t)w.slot * kTcResSlots + (2 * t + (n0 > 0 ? 1 : 0)) * 4 + warp] = res;
		}
	} else if (tid == 0) {
		atomicOr(a.err, 1);
	}
	tc_fence_before();
	__syncthreads();
	if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------------------------
// persistent iteration kernel: one CTA per SM walks the tiles of a phase
// ---------------------------------------------------------------------------------------------
// Epilogue of one iteration tile read from the accumulator at tensor-memory column `col0`: warp
// quarter q (warp % 4) owns rows 32 q .. 32 q + 31 of the tile.  Gram: P = c1 I + c3 G into the P
// planes and the tile's residual partials; update: the next iterate into the other iterate buffer,
// or T for the final update.  The accumulator holds 2^24 times the product.
template <int PHASE>
__device__ __forceinline__ void tc_iter_epilogue(const TcArgs &a, const TcWork &w, int t, int n0, int N,
                                                 uint32_t tmem, uint32_t col0, int q, int lane, bool final_update,
                                                 float c1, float c3) {
	const int n = w.n, np = w.np, npg = np >> 3;
	const int row = 128 * t + 32 * q + lane;
	const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16) + col0;
	const int64_t pe = (int64_t)np * np;
	float res = 0.f;
	for (int cb = 0; cb < N; cb += 64) {
		// 64 columns per tensor-memory load (inside the 256-column accumulator; columns past N unused)
		float vv[64];
		tmem_ld64(trow + (uint32_t)cb, vv);
		if (row >= np) continue;
#pragma unroll
		for (int sb = 0; sb < 4; sb++) {
			const int c0 = cb + 16 * sb;
			if (c0 >= N) break;
			float *v = vv + 16 * sb;
#pragma unroll
			for (int k = 0; k < 16; k++) v[k] *= kTcAccUnscale;
			if (PHASE == kTcPhaseGram) {
#pragma unroll
				for (int k = 0; k < 16; k++) {
					const int col = n0 + c0 + k;
					const float g = v[k];
					if (row < n && col < n) {
						const float d = g - (col == row ? 1.f : 0.f);
						res += d * d;
					}
					v[k] = c3 * g + (col == row ? c1 : 0.f);
				}
				__nv_bfloat16 *P0 = a.Pp + w.pofs;
#pragma unroll
				for (int h = 0; h < 2; h++) {
					const int64_t o = ((int64_t)(row >> 3) * npg + ((n0 + c0) >> 3) + h) * 64 + (row & 7) * 8;
					store_split8h(v + 8 * h, P0 + o, P0 + pe + o);
				}
			} else if (final_update) {
				if (row < n) {
					float *T = a.T + w.tofs;
#pragma unroll
					for (int k = 0; k < 16; k++) {
						const int col = n0 + c0 + k;
						if (col < n) T[a.t_rowmajor ? (int64_t)row * n + col : (int64_t)col * n + row] = v[k];
					}
				}
			} else {
				__nv_bfloat16 *X0 = a.Xw + w.xofs;
#pragma unroll
				for (int h = 0; h < 2; h++) {
					const int64_t o = ((int64_t)(row >> 3) * npg + ((n0 + c0) >> 3) + h) * 64 + (row & 7) * 8;
					store_split8h(v + 8 * h, X0 + o, X0 + pe + o);
				}
			}
		}
	}
	if (PHASE == kTcPhaseGram) {
		res = warp_sum(res);
		if (lane == 0) a.res_part[(int64_t)w.slot * kTcResSlots + (2 * t + (n0 > 0 ? 1 : 0)) * 4 + q] = res;
	}
}

// The update's decision for one searchlight from the residual partials of this iteration's Gram
// (fixed-order sum, the same in every thread) and the state it read: final update or not; the
// state for the next iteration goes to *out.
__device__ __forceinline__ bool tc_update_decision(const TcArgs &a, const TcWork &w, const TcState &st, TcState *out) {
	double ss = 0.0;
	for (int i = 0; i < kTcResSlots; i++) ss += (double)a.res_part[(int64_t)w.slot * kTcResSlots + i];
	const double resd = sqrt(ss / (double)w.n);
	const float res = (float)resd;
	const bool conv = a.plain && res < a.tol_stop;
	// a residual that a plain step leaves unchanged to 5e-7 relative: singular values below the FP32
	// resolution of A (see k_tc_gemm)
	const bool stalled = !conv && a.plain && st.plain && fabs(resd - (double)st.res) <= 5e-7 * resd;
	const bool fin = conv || stalled || a.last;
	TcState o = st;
	o.iters = st.iters + 1;
	o.res = res;
	o.conv = conv ? 1 : 0;
	o.stalled = stalled ? 1 : 0;
	o.done = fin ? 1 : 0;
	o.plain = a.plain;
	*out = o;
	return fin;
}

constexpr int kTcIterThreads = 192;    // warp 0 producer, warp 1 MMA, warps 2-5 epilogue
constexpr uint32_t kTcIterCols = 512;  // two accumulators of up to 256 columns
constexpr int kTcIterMaxTiles = 256;   // tiles per CTA (the grid grows to keep within it)

// One tile of a persistent launch as the roles need it, gathered once at the kernel's start.
struct TcIterTile {
	int32_t slot, n, np, t, n0, nn;
	int32_t skip;  // the searchlight is done
	int32_t fin;   // update: this update is the searchlight's last (it writes T)
	int64_t xofs, pofs, tofs;
};

// The Gram (PHASE 1) or update (PHASE 2) products of every tile of a launch, one CTA per SM walking
// tiles blockIdx.x, blockIdx.x + gridDim.x, ...  Stages are filled continuously across tile
// boundaries: warp 0 copies the A tile with per-lane cp.async (the hardware arrives on the stage's
// full barrier for each lane once that lane's copies have landed; the MMA thread fences the proxy
// after its wait) and the B operand with bulk copies (K half by K half, their bytes counted by the same
// barrier); lane 0 of warp 1 issues each stage's three products into one of two tensor-memory
// accumulators (tiles alternate) and commits the stage to its consumed barrier and the finished
// tile to the accumulator's full barrier; warps 2-5 read the finished accumulator, write the
// epilogue and release it, while the next tile's products run in the other accumulator.
// Searchlights already done are skipped by every role alike.  nmax: the widest tile of the launch
// (128 or 256), which sizes the B planes of a stage.  Every wait is bounded; a timeout sets the
// error flag and every role ends.
template <int PHASE>
__global__ void __launch_bounds__(kTcIterThreads, 1) k_tc_iter(const TcArgs a, int ntiles, int nmax) {
	static_assert(PHASE != kTcPhaseXcov, "the cross-covariance keeps the per-tile kernel");
	extern __shared__ __align__(128) unsigned char tc_smem[];
	__shared__ uint64_t s_full[kTcMaxStages], s_empty[kTcMaxStages], s_accf[2], s_acce[2], s_fin;
	__shared__ uint32_t s_tmem;
	__shared__ int s_fail;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	if (PHASE == kTcPhaseUpdate && a.Xw == nullptr) {
		if (tid == 0) atomicOr(a.err, 1);
		return;
	}
	const int stage_bytes = 2 * 4096 + 2 * 32 * nmax;
	// the tile list sits after the stages
	// tiles dealt in snake order (round e: CTA b takes e G + b, or e G + G - 1 - b in odd rounds), which
	// balances a largest-first tile list better than plain round-robin
	const int G = (int)gridDim.x, B = (int)blockIdx.x;
	auto tile_of = [&](int e) { return e * G + ((e & 1) ? G - 1 - B : B); };
	int mine = ntiles / G;
	if (mine * G < ntiles && tile_of(mine) < ntiles) mine++;
	int S = (a.smem_bytes - kTcIterMaxTiles * (int)sizeof(TcIterTile)) / stage_bytes;
	if (S > kTcMaxStages) S = kTcMaxStages;
	TcIterTile *tlist = reinterpret_cast<TcIterTile *>(tc_smem + S * stage_bytes);
	const uint32_t smem0 = smem_u32(tc_smem);
	if (tid == 0) {
		for (int i = 0; i < kTcMaxStages; i++) {
			mbar_init(&s_full[i], 32);
			mbar_init(&s_empty[i], 1);
		}
		for (int b = 0; b < 2; b++) {
			mbar_init(&s_accf[b], 1);
			mbar_init(&s_acce[b], 4);
		}
		mbar_init(&s_fin, 1);
		s_fail = (S < 2 || nmax > 256 || mine > kTcIterMaxTiles) ? 1 : 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == 0) tmem_alloc(&s_tmem, kTcIterCols);
	// every thread gathers some of this CTA's tiles: one round of independent loads instead of a
	// chain of dependent ones per tile in every role; the update's decisions and next states too
	if (mine <= kTcIterMaxTiles)
		for (int e = tid; e < mine; e += kTcIterThreads) {
			const TcTile tl = a.tiles[tile_of(e)];
			const TcWork w = a.work[tl.w];
			const TcState st = a.st_in[w.slot];
			TcIterTile d;
			d.slot = w.slot; d.n = w.n; d.np = w.np; d.t = tl.t; d.n0 = tl.n0; d.nn = tl.nn;
			d.skip = st.done ? 1 : 0;
			d.fin = 0;
			d.xofs = w.xofs; d.pofs = w.pofs; d.tofs = w.tofs;
			if (PHASE == kTcPhaseUpdate) {
				TcState o = st;
				if (!st.done) d.fin = tc_update_decision(a, w, st, &o) ? 1 : 0;
				if (tl.t == 0 && tl.n0 == 0) a.st_out[w.slot] = o;
			}
			tlist[e] = d;
		}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = s_tmem;
	volatile int *vfail = &s_fail;
	const bool failed0 = *vfail != 0;

	if (warp == 0 && !failed0) {
		uint32_t g = 0;  // slices issued by this CTA
		bool ok = true;
		for (int e = 0; e < mine && ok; e++) {
			const TcIterTile d = tlist[e];
			if (d.skip) continue;
			const int np = d.np, npg = np >> 3, t = d.t, N = d.nn, g0 = d.n0 >> 3, nk = np >> 4;
			const int64_t pe = (int64_t)np * np;
			const __nv_bfloat16 *As = a.Xp + d.xofs;
			const __nv_bfloat16 *Bs = (PHASE == kTcPhaseGram) ? As : (const __nv_bfloat16 *)(a.Pp + d.pofs);
			for (int ks = 0; ks < nk; ks++, g++) {
				const int s = (int)(g % (uint32_t)S);
				int go = 1;
				if (lane == 0) {
					if (g >= (uint32_t)S && !mbar_wait(&s_empty[s], (g / S - 1) & 1u)) {
						*vfail = 1;
						go = 0;
					}
					if (go) mbar_add_tx(&s_full[s], 64u * (uint32_t)N);  // B: two planes x two K halves x 16 N
				}
				if (!__shfl_sync(0xffffffffu, go, 0)) {
					ok = false;
					break;
				}
				const uint32_t st = smem0 + s * stage_bytes;
				if (lane < 4) {  // B: plane lane >> 1, K half lane & 1
					const int pb = lane >> 1, k = lane & 1;
					bulk_g2s(st + 8192 + pb * 32 * nmax + k * 16 * N, Bs + pb * pe + ((int64_t)(2 * ks + k) * npg + g0) * 64,
					         16u * N, &s_full[s]);
				}
				// A: 256 chunks of 16 bytes per plane, chunk c = lane + 32 j: core (g, k) = (c >> 4, (c >> 3) & 1)
#pragma unroll
				for (int p = 0; p < 2; p++)
#pragma unroll
					for (int j = 0; j < 8; j++) {
						const int c = lane + 32 * j, core = c >> 3, r = c & 7, gg = core >> 1, k = core & 1;
						const bool valid = 16 * t + gg < npg;
						const int64_t src = (PHASE == kTcPhaseGram) ? ((int64_t)(2 * ks + k) * npg + 16 * t + gg) * 64 + 8 * r
						                                            : ((int64_t)(16 * t + gg) * npg + 2 * ks + k) * 64 + 8 * r;
						cp_async16(st + p * 4096 + core * 128 + r * 16, valid ? As + p * pe + src : As, valid ? 16u : 0u);
					}
				cp_async_arrive_noinc(&s_full[s]);  // when this lane's copies of the stage have landed
			}
		}
		cp_async_wait_all();
		// every copy issued has landed before the CTA may leave
		if (lane == 0)
			for (uint32_t h = g > (uint32_t)S ? g - S : 0u; h < g; h++)
				if (!mbar_wait(&s_full[h % S], (h / S) & 1u)) *vfail = 1;
		__syncwarp();
	}
	if (warp == 1 && !failed0) {
		// lane 0 issues; the other lanes wait at the warp barrier
		uint32_t g = 0, j = 0;  // slices consumed, tiles computed
		const int a_mn = (PHASE == kTcPhaseGram) ? 1 : 0;
		for (int e = 0; e < mine; e++) {
			const TcIterTile d = tlist[e];
			if (d.skip) continue;
			const int nk = d.np >> 4, N = d.nn, b = (int)(j & 1u);
			int ok = 1;
			if (lane == 0) {
				// the accumulator's previous tile (j - 2) must have been read out
				if (j >= 2 && !mbar_wait(&s_acce[b], ((j >> 1) - 1) & 1u)) ok = 0;
				const uint32_t id = mma_idesc(128, N, a_mn, 1, true);
				const uint32_t acc_t = tmem + (uint32_t)(256 * b);
				tc_fence_after();
				for (int ks = 0; ks < nk && ok; ks++, g++) {
					const int s = (int)(g % (uint32_t)S);
					if (!mbar_wait(&s_full[s], (g / S) & 1u)) {
						ok = 0;
						break;
					}
					fence_proxy_async_smem();  // the lanes' cp.async writes, seen through the barrier, to the MMA
					tc_fence_after();
					const uint32_t st = smem0 + s * stage_bytes;
#pragma unroll
					for (int q = 0; q < 3; q++) {  // mid*hi, hi*mid, hi*hi
						const int pa = q == 0 ? 1 : 0, pb = q == 1 ? 1 : 0;
						mma_bf16(acc_t, smem_desc(st + pa * 4096, 128, 256),
						         smem_desc(st + 8192 + pb * 32 * nmax, 16u * N, 128), id, (ks > 0 || q > 0) ? 1u : 0u);
					}
					mma_commit(&s_empty[s]);
				}
				if (ok) mma_commit(&s_accf[b]);
				else *vfail = 1;
			}
			if (!__shfl_sync(0xffffffffu, ok, 0)) break;
			j++;
		}
		if (lane == 0) mma_commit(&s_fin);  // completes once every product issued has
		__syncwarp();
	}
	if (warp >= 2 && !failed0) {
		uint32_t j = 0;
		for (int e = 0; e < mine; e++) {
			const TcIterTile d = tlist[e];
			if (d.skip) continue;
			TcWork w = {};
			w.slot = d.slot; w.n = d.n; w.np = d.np; w.xofs = d.xofs; w.pofs = d.pofs; w.tofs = d.tofs;
			const bool fin = d.fin != 0;
			const int b = (int)(j & 1u);
			if (!mbar_wait_idle(&s_accf[b], (j >> 1) & 1u)) {
				*vfail = 1;
				break;
			}
			tc_fence_after();
			tc_iter_epilogue<PHASE>(a, w, d.t, d.n0, d.nn, tmem, (uint32_t)(256 * b), warp & 3, lane, fin, a.c1, a.c3);
			tc_fence_before();
			__syncwarp();
			if (lane == 0) mbar_arrive(&s_acce[b]);
			j++;
		}
	}
	__syncthreads();
	if (tid == 0) {
		if (!failed0 && !mbar_wait(&s_fin, 0)) *vfail = 1;
		if (*vfail) atomicOr(a.err, 1);
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (warp == 0) tmem_dealloc(tmem, kTcIterCols);
}

// ---------------------------------------------------------------------------------------------
// persistent solve: one CTA runs whole searchlights
// ---------------------------------------------------------------------------------------------
// Each CTA takes searchlights from a queue (largest first) and runs the whole solve of one
// searchlight before the next: the cross-covariance tiles, X_0 = A / u, every Gram and update
// phase (the residual is summed in shared memory), the trace for the scaling.  The searchlight's
// planes (~12 np^2 bytes) stay in L2 across its iterations instead of streaming through DRAM
// once per phase, and the whole step is one launch per size class.  The products are the same
// as k_tc_gemm's; mbarrier phases are tracked per stage across tiles and searchlights.

struct TcSolveArgs {
	const TcWork *work;
	const int32_t *order;  // work indices of this launch's size class, largest first
	int count;
	int32_t *queue;        // next position in `order` (zero before the launch)
	const __nv_bfloat16 *Xb;
	const __nv_bfloat16 *Yb;
	int64_t vplane;
	int ntp;
	const int32_t *sl_idx;
	__nv_bfloat16 *Xp;
	__nv_bfloat16 *Pp;
	float *A32;
	float *T;
	int t_rowmajor;
	const float *c1;  // schedule, maxit entries
	const float *c3;
	const int32_t *plain;
	int maxit;
	float tol_stop;
	SlStats *stats;
	int smem_bytes;
	int *err;
};

struct TcPipe {
	uint32_t uses[kTcMaxStages];  // completed commits per stage barrier (identical in every thread)
	uint32_t acc;                 // completed commits of the accumulator barrier
};

__device__ __forceinline__ float block_sum128(float v, float *red) {
	v = warp_sum(v);
	__syncthreads();
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
	__syncthreads();
	return red[0] + red[1] + red[2] + red[3];
}

// One 128-row tile of one phase, inside the persistent CTA.  Returns false (in every thread) when
// a wait timed out.  On return all products are complete and the epilogue's stores are issued.
template <int PHASE>
__device__ bool tc_tile(const TcSolveArgs &a, const TcWork &w, int t, const int32_t *s_sl, float c1, float c3,
                        bool final_update, TcPipe &pp, uint64_t *s_bar, uint64_t *s_acc, uint32_t tmem,
                        uint32_t smem0, int S, int stage_bytes, int *s_fail, float *s_res) {
	const int n = w.n, np = w.np, N = np;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int nk = (PHASE == kTcPhaseXcov) ? (a.ntp >> 4) : (np >> 4);
	const __nv_bfloat16 *Xs = a.Xp + w.xofs;
	const __nv_bfloat16 *Bs = (PHASE == kTcPhaseGram) ? Xs : (const __nv_bfloat16 *)(a.Pp + w.pofs);
	TcLoadPlan lp;
	tc_plan_tile<PHASE>(lp, s_sl, n, np, a.ntp, t, 0, N);
	const __nv_bfloat16 *srcA = (PHASE == kTcPhaseXcov) ? a.Xb : Xs;
	const __nv_bfloat16 *srcB = (PHASE == kTcPhaseXcov) ? a.Yb : Bs;
	const int64_t pstride = (PHASE == kTcPhaseXcov) ? a.vplane : (int64_t)np * np;
	constexpr int NPL = TcFmt<PHASE>::planes;
	auto load = [&](int ks, int s) {
		tc_load_slice<NPL>(lp, srcA, pstride, srcB, pstride, N, ks, smem0 + s * stage_bytes);
	};
	const int a_mn = (PHASE == kTcPhaseGram) ? 1 : 0;
	const int b_mn = (PHASE == kTcPhaseXcov) ? 0 : 1;
	const int N0 = N > 256 ? 256 : N;
	const bool f16 = PHASE != kTcPhaseXcov;
	const uint32_t id0 = mma_idesc(128, N0, a_mn, b_mn, f16);
	const uint32_t id1 = N > 256 ? mma_idesc(128, N - 256, a_mn, b_mn, f16) : 0u;

	// every stage is free here: the previous tile's products all completed
	for (int j = 0; j < S - 1; j++) {
		if (j < nk) load(j, j);
		cp_async_commit();
	}
	bool failed = false;
	for (int ks = 0; ks < nk; ks++) {
		const int s = ks % S;
		cp_async_wait_keep(S - 2);
		fence_proxy_async_smem();
		__syncthreads();
		if (*s_fail) { failed = true; break; }
		if (tid == 0) {
			tc_fence_after();
			tc_issue_products<PHASE>(tmem, smem0 + s * stage_bytes, N, id0, id1, ks == 0);
			mma_commit(&s_bar[s]);
		}
		pp.uses[s]++;
		// refill the stage the products of K-slice ks - 1 read, while slice ks stays queued
		const int kn = ks + S - 1;
		if (kn < nk) {
			const int sp = kn % S;
			if (ks >= 1 && !mbar_wait(&s_bar[sp], (pp.uses[sp] - 1u) & 1u)) *s_fail = 1;
			load(kn, sp);
		}
		cp_async_commit();
	}
	cp_async_wait_all();
	if (!failed) {
		if (tid == 0) mma_commit(s_acc);
		pp.acc++;
		if (!mbar_wait(s_acc, (pp.acc - 1u) & 1u)) *s_fail = 1;
	}
	__syncthreads();
	if (*s_fail) return false;
	tc_fence_after();

	const int m = 32 * warp + lane;
	const int row = 128 * t + m;
	const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
	const int npg = np >> 3;
	float res = 0.f;
	for (int c0 = 0; c0 < N; c0 += 16) {
		float v[16];
		tmem_ld16(trow + (uint32_t)c0, v);
		if (row >= np) continue;
		if (PHASE != kTcPhaseXcov) {
#pragma unroll
			for (int q = 0; q < 16; q++) v[q] *= kTcAccUnscale;
		}
		if (PHASE == kTcPhaseXcov) {
			if (row < n) {
				float4 *dst = reinterpret_cast<float4 *>(a.A32 + w.aofs + (int64_t)row * np + c0);
#pragma unroll
				for (int q = 0; q < 4; q++) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
			}
		} else if (PHASE == kTcPhaseGram) {
#pragma unroll
			for (int q = 0; q < 16; q++) {
				const int col = c0 + q;
				const float g = v[q];
				if (row < n && col < n) {
					const float d = g - (col == row ? 1.f : 0.f);
					res += d * d;
				}
				v[q] = c3 * g + (col == row ? c1 : 0.f);
			}
			__nv_bfloat16 *P0 = a.Pp + w.pofs;
			const int64_t pe = (int64_t)np * np;
#pragma unroll
			for (int h = 0; h < 2; h++) {
				const int64_t o = ((int64_t)(row >> 3) * npg + (c0 >> 3) + h) * 64 + (row & 7) * 8;
				store_split8h(v + 8 * h, P0 + o, P0 + pe + o);
			}
		} else if (final_update) {
			if (row < n) {
				float *T = a.T + w.tofs;
				for (int q = 0; q < 16; q++) {
					const int col = c0 + q;
					if (col < n) T[a.t_rowmajor ? (int64_t)row * n + col : (int64_t)col * n + row] = v[q];
				}
			}
		} else {
			__nv_bfloat16 *X0 = a.Xp + w.xofs;
			const int64_t pe = (int64_t)np * np;
#pragma unroll
			for (int h = 0; h < 2; h++) {
				const int64_t o = ((int64_t)(row >> 3) * npg + (c0 >> 3) + h) * 64 + (row & 7) * 8;
				store_split8h(v + 8 * h, X0 + o, X0 + pe + o);
			}
		}
	}
	if (PHASE == kTcPhaseGram) {
		res = warp_sum(res);
		if (lane == 0) s_res[2 * t * 4 + warp] = res;
	}
	// the next tile's products overwrite tensor memory: order this tile's reads before them, and
	// make the global stores visible to the next phase's cp.async reads (through L2)
	tc_fence_before();
	__threadfence();
	__syncthreads();
	return true;
}

__global__ void __launch_bounds__(kTcThreads) k_tc_solve(const TcSolveArgs a) {
	extern __shared__ __align__(128) unsigned char tc_smem[];
	__shared__ uint64_t s_bar[kTcMaxStages];
	__shared__ uint64_t s_acc;
	__shared__ uint32_t s_tmem;
	__shared__ int s_fail, s_item;
	__shared__ int32_t s_sl[kTcMaxNp];
	__shared__ float s_res[kTcResSlots];
	__shared__ float s_red[4];
	__shared__ float s_u;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const uint32_t smem0 = smem_u32(tc_smem);
	// tensor memory for the largest accumulator this launch can meet
	const uint32_t ncols = a.smem_bytes > 120 * 1024 ? 512u : 256u;
	if (tid == 0) {
		for (int i = 0; i < kTcMaxStages; i++) mbar_init(&s_bar[i], 1);
		mbar_init(&s_acc, 1);
		s_fail = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == 0) tmem_alloc(&s_tmem, ncols);
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = s_tmem;
	TcPipe pp = {};
	bool failed = false;
	for (;;) {
		if (tid == 0) s_item = atomicAdd(a.queue, 1);
		__syncthreads();
		const int item = s_item;
		if (item >= a.count) break;
		const TcWork w = a.work[a.order[item]];
		const int n = w.n, np = w.np, ntiles = (np + 127) >> 7;
		const int stage_bytes = tc_stage_bytes(np, 3);  // the largest format; the iteration's fit too
		int S = a.smem_bytes / stage_bytes;
		if (S > kTcMaxStages) S = kTcMaxStages;
		if (S < 2 || (uint32_t)np > ncols) { s_fail = 1; failed = true; break; }
		for (int i = tid; i < n; i += kTcThreads) s_sl[i] = a.sl_idx[w.sofs + i];
		__syncthreads();
		// cross-covariance A = X_sl^T Y_sl
		for (int t = 0; t < ntiles && !failed; t++)
			failed = !tc_tile<kTcPhaseXcov>(a, w, t, s_sl, 0.f, 0.f, false, pp, s_bar, &s_acc, tmem, smem0, S,
			                                 stage_bytes, &s_fail, s_res);
		if (failed) break;
		// X_0 = A / u, u = min(||A||_F, sqrt(||A||_1 ||A||_inf)) >= sigma_max
		const float *A = a.A32 + w.aofs;
		{
			float *colsum = reinterpret_cast<float *>(tc_smem);  // the stages are free here
			float fro = 0.f, rowmax = 0.f;
			for (int r = warp; r < n; r += 4) {
				float rs = 0.f;
				for (int c = lane; c < n; c += 32) {
					const float x = A[(int64_t)r * np + c];
					fro += x * x;
					rs += fabsf(x);
				}
				rowmax = fmaxf(rowmax, warp_sum(rs));
			}
			for (int c = tid; c < n; c += kTcThreads) {
				float cs = 0.f;
				for (int r = 0; r < n; r++) cs += fabsf(A[(int64_t)r * np + c]);
				colsum[c] = cs;
			}
			const float f = block_sum128(fro, s_red);
			float cm = 0.f;
			for (int c = tid; c < n; c += kTcThreads) cm = fmaxf(cm, colsum[c]);
			for (int o = 16; o > 0; o >>= 1) {
				cm = fmaxf(cm, __shfl_xor_sync(0xffffffffu, cm, o));
				rowmax = fmaxf(rowmax, __shfl_xor_sync(0xffffffffu, rowmax, o));
			}
			__syncthreads();
			if (lane == 0) { s_red[warp] = cm; colsum[kTcMaxNp + warp] = rowmax; }
			__syncthreads();
			if (tid == 0) {
				float cmax = 0.f, rmax = 0.f;
				for (int i = 0; i < 4; i++) { cmax = fmaxf(cmax, s_red[i]); rmax = fmaxf(rmax, colsum[kTcMaxNp + i]); }
				double u = fmin(sqrt((double)f), sqrt((double)rmax * (double)cmax));
				if (!(u > 0.0)) u = 1.0;
				s_u = (float)(u * (1.0 + 1e-6));
			}
			__syncthreads();
			const float inv = 1.f / s_u;
			const int npg = np >> 3;
			const int64_t pe = (int64_t)np * np;
			__nv_bfloat16 *X0 = a.Xp + w.xofs;
			for (int64_t e = tid; e < (int64_t)np * npg; e += kTcThreads) {
				const int row = (int)(e / npg), cg = (int)(e - (int64_t)row * npg);
				float v[8];
#pragma unroll
				for (int q = 0; q < 8; q++) {
					const int col = 8 * cg + q;
					v[q] = (row < n && col < n) ? A[(int64_t)row * np + col] * inv : 0.f;
				}
				const int64_t o = ((int64_t)(row >> 3) * npg + cg) * 64 + (row & 7) * 8;
				store_split8h(v, X0 + o, X0 + pe + o);
			}
			__threadfence();
			__syncthreads();
		}
		// the iteration
		bool conv = false, stalled = false, prev_plain = false;
		double prev_res = 0.0;
		int k = 0;
		for (; k < a.maxit; k++) {
			if (tid < kTcResSlots) s_res[tid] = 0.f;
			__syncthreads();
			const float c1 = a.c1[k], c3 = a.c3[k];
			const bool plain = a.plain[k] != 0;
			for (int t = 0; t < ntiles && !failed; t++)
				failed = !tc_tile<kTcPhaseGram>(a, w, t, s_sl, c1, c3, false, pp, s_bar, &s_acc, tmem, smem0, S,
				                                 stage_bytes, &s_fail, s_res);
			if (failed) break;
			double ss = 0.0;
			for (int i = 0; i < kTcResSlots; i++) ss += (double)s_res[i];
			const double resd = sqrt(ss / (double)n);
			conv = plain && (float)resd < a.tol_stop;
			stalled = !conv && plain && prev_plain && fabs(resd - prev_res) <= 5e-7 * resd;
			const bool final_update = conv || stalled || k == a.maxit - 1;
			for (int t = 0; t < ntiles && !failed; t++)
				failed = !tc_tile<kTcPhaseUpdate>(a, w, t, s_sl, 0.f, 0.f, final_update, pp, s_bar, &s_acc, tmem,
				                                   smem0, S, stage_bytes, &s_fail, s_res);
			if (failed) break;
			prev_plain = plain;
			prev_res = (double)(float)resd;
			if (final_update) { k++; break; }
		}
		if (failed) break;
		// sum of singular values = trace(T^T A) (the scaling numerator), flags
		{
			const float *T = a.T + w.tofs;
			double s = 0.0;
			for (int64_t e = tid; e < (int64_t)n * n; e += kTcThreads) {
				const int r = (int)(e / n), c = (int)(e - (int64_t)r * n);
				const float tv = a.t_rowmajor ? T[(int64_t)r * n + c] : T[(int64_t)c * n + r];
				s += (double)tv * (double)A[(int64_t)r * np + c];
			}
			s = warp_sum(s);
			__syncthreads();
			double *red = reinterpret_cast<double *>(tc_smem);
			if (lane == 0) red[warp] = s;
			__syncthreads();
			if (tid == 0) {
				SlStats o = {};
				o.s_sum = red[0] + red[1] + red[2] + red[3];
				o.s_max = (double)s_u;
				o.sweeps = k;
				o.flags = conv ? 0 : kFlagIllCond;
				a.stats[w.slot] = o;
			}
			__syncthreads();
		}
	}
	if (failed && tid == 0) atomicOr(a.err, 1);
	cp_async_wait_all();
	tc_fence_before();
	__syncthreads();
	if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------------------------
// SIMT helpers of the tensor-core solve
// ---------------------------------------------------------------------------------------------

// float64 column-major [v][nt] -> three bf16 planes [plane][v][ntp] (exact split of the value rounded
// to FP32; samples past nt are zero).
__global__ void k_split3_vertex_major(const double *__restrict__ X, int nt, int nv, int ntp,
                                      __nv_bfloat16 *__restrict__ out) {
	const int64_t total = (int64_t)nv * ntp;
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
		const int64_t v = e / ntp;
		const int t = (int)(e - v * ntp);
		const float x = (t < nt) ? (float)X[v * nt + t] : 0.f;
		__nv_bfloat16 h, m, l;
		split3(x, h, m, l);
		out[e] = h;
		out[total + e] = m;
		out[2 * total + e] = l;
	}
}

// X_0 = A / u with u = min(||A||_F, sqrt(||A||_1 ||A||_inf)) >= sigma_max(A), written as the two
// core-tiled FP16 planes of the iteration (np x np, padding zero); iteration state and residual
// slots cleared.
__global__ void __launch_bounds__(256) k_tc_ns_init(const TcWork *__restrict__ work, const float *__restrict__ A32,
                                                    __nv_bfloat16 *__restrict__ Xp, TcState *__restrict__ st,
                                                    float *__restrict__ res_part) {
	const TcWork w = work[blockIdx.x];
	const int n = w.n, np = w.np, npg = np >> 3;
	const float *A = A32 + w.aofs;
	__shared__ double s_red[2][8];
	__shared__ float s_colsum[kTcMaxNp];
	__shared__ float s_u;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	double fro = 0.0, rowmax = 0.0;
	for (int r = warp; r < n; r += 8) {
		double rs = 0.0;
		for (int c = lane; c < n; c += 32) {
			const double x = A[(int64_t)r * np + c];
			fro += x * x;
			rs += fabs(x);
		}
		rs = warp_sum(rs);
		rowmax = fmax(rowmax, rs);
	}
	for (int c = threadIdx.x; c < n; c += blockDim.x) {
		float cs = 0.f;
		for (int r = 0; r < n; r++) cs += fabsf(A[(int64_t)r * np + c]);
		s_colsum[c] = cs;
	}
	fro = warp_sum(fro);
	if (lane == 0) { s_red[0][warp] = fro; s_red[1][warp] = rowmax; }
	__syncthreads();
	if (threadIdx.x == 0) {
		double f = 0.0, rm = 0.0, cm = 0.0;
		for (int i = 0; i < 8; i++) { f += s_red[0][i]; rm = fmax(rm, s_red[1][i]); }
		for (int c = 0; c < n; c++) cm = fmax(cm, (double)s_colsum[c]);
		double u = fmin(sqrt(f), sqrt(rm * cm));
		if (!(u > 0.0)) u = 1.0;  // zero matrix: the iterate stays zero and the solve is flagged
		s_u = (float)(u * (1.0 + 1e-6));
		TcState z = {};
		z.u = s_u;
		st[w.slot] = z;
	}
	for (int i = threadIdx.x; i < kTcResSlots; i += blockDim.x) res_part[(int64_t)w.slot * kTcResSlots + i] = 0.f;
	__syncthreads();
	const float inv = 1.f / s_u;
	const int64_t pe = (int64_t)np * np;
	__nv_bfloat16 *X0 = Xp + w.xofs;
	// one thread per core-matrix row (8 elements)
	const int64_t chunks = (int64_t)np * npg;
	for (int64_t e = threadIdx.x; e < chunks; e += blockDim.x) {
		const int row = (int)(e / npg), cg = (int)(e - (int64_t)row * npg);
		float v[8];
#pragma unroll
		for (int q = 0; q < 8; q++) {
			const int col = 8 * cg + q;
			v[q] = (row < n && col < n) ? A[(int64_t)row * np + col] * inv : 0.f;
		}
		const int64_t o = ((int64_t)(row >> 3) * npg + cg) * 64 + (row & 7) * 8;
		store_split8h(v, X0 + o, X0 + pe + o);
	}
}

// After the iteration: sum of singular values = trace(T^T A) (the scaling numerator,
// csrc/ha_searchlight.c:635-656), iteration count, and the flag that hands unconverged
// searchlights (exactly singular ones keep a zero singular value that the iteration cannot
// complete) to the float64 Jacobi re-solve.
__global__ void __launch_bounds__(256) k_tc_ns_finish(const TcWork *__restrict__ work, const float *__restrict__ A32,
                                                      const float *__restrict__ Tscr, const TcState *__restrict__ st,
                                                      SlStats *__restrict__ stats, int t_rowmajor) {
	const TcWork w = work[blockIdx.x];
	const int n = w.n, np = w.np;
	const float *A = A32 + w.aofs;
	const float *T = Tscr + w.tofs;
	double s = 0.0;
	for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
		const int r = (int)(e / n), c = (int)(e - (int64_t)r * n);
		const float tv = t_rowmajor ? T[(int64_t)r * n + c] : T[(int64_t)c * n + r];
		s += (double)tv * (double)A[(int64_t)r * np + c];
	}
	s = warp_sum(s);
	__shared__ double red[8];
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x == 0) {
		double tot = 0.0;
		for (int i = 0; i < (int)(blockDim.x >> 5); i++) tot += red[i];
		const TcState z = st[w.slot];
		SlStats o = {};
		o.s_sum = tot;
		o.s_max = (double)z.u;
		o.s_min = 0.0;
		o.k_min = 0;
		o.sweeps = z.iters;
		o.flags = z.conv ? 0 : kFlagIllCond;
		stats[w.slot] = o;
	}
}

// ---------------------------------------------------------------------------------------------
// completion of exactly singular searchlights
// ---------------------------------------------------------------------------------------------
// A searchlight whose iteration stalled ends with T = U_r V_r^T (its converged directions) and
// d singular values that stay exactly zero (A singular: duplicated or zero vertex columns).  The
// reference's SVD completes such a T with an arbitrary orthonormal pairing of the null spaces
// (only T on the row space of A, and X T, are unique); here: E = I - T^T T and F = I - T T^T are
// the projectors onto the right and left null spaces, pivoted Cholesky (stopping at pivots below
// 1e-4, the level of the converged directions' residue) gives their bases L_E, L_F, which must be
// orthonormal already (L^T L = I to 1e-3: the extracted directions are fully null, not partly
// converged), Gram-Schmidt cleans them, and T <- (I - U_0 U_0^T) T + U_0 V_0^T.  Searchlights that
// fail a check keep kFlagIllCond and go to the float64 re-solve.  E and F are never formed: the
// factorisation is left-looking and reads only the diagonal (1 - the squared column norms of T or
// T^T) and the at most kTcNullMax + 1 pivot columns (e_p - S^T S(:, p)), O(d n^2) work instead of
// 2 n^3.  The projection coefficients U_0^T T go to the searchlight's P planes (free after the
// iteration) as FP32 scratch.
constexpr int kTcNullMax = 8;

__device__ __forceinline__ float block_sum256(float v, float *red) {
	v = warp_sum(v);
	__syncthreads();
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
	__syncthreads();
	float t = 0.f;
	for (int i = 0; i < 8; i++) t += red[i];
	return t;
}

// r[i] = sum_k S(k, i) u(k) for i < n, S(k, i) = S0[k sk + i si], u = the shared vector v, or S(:, i)
// itself when v is null.  One thread per i when i runs contiguously in memory (si == 1), else one
// warp per i with k across the lanes (sk == 1): both read memory in order across a warp.
__device__ __forceinline__ void tc_cols_dot(const float *__restrict__ S0, int64_t sk, int64_t si, int n,
                                            const float *v, float *r) {
	if (si == 1) {
		for (int i = threadIdx.x; i < n; i += blockDim.x) {
			float acc = 0.f;
			for (int k = 0; k < n; k++) {
				const float x = S0[k * sk + i];
				acc = fmaf(x, v ? v[k] : x, acc);
			}
			r[i] = acc;
		}
	} else {
		const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
		for (int i = threadIdx.x >> 5; i < n; i += nw) {
			float acc = 0.f;
			for (int k = lane; k < n; k += 32) {
				const float x = S0[k * sk + i * si];
				acc = fmaf(x, v ? v[k] : x, acc);
			}
			acc = warp_sum(acc);
			if (lane == 0) r[i] = acc;
		}
	}
}

__global__ void __launch_bounds__(256) k_tc_complete(const TcWork *__restrict__ work, float *__restrict__ Tscr,
                                                     __nv_bfloat16 *__restrict__ Xp, __nv_bfloat16 *__restrict__ Pp,
                                                     SlStats *__restrict__ stats, int t_rowmajor) {
	(void)Xp;
	const TcWork w = work[blockIdx.x];
	if (!(stats[w.slot].flags & kFlagIllCond)) return;
	const int n = w.n;
	float *T = Tscr + w.tofs;
	float *Cs = reinterpret_cast<float *>(Pp + w.pofs);  // d x n projection coefficients
	const int64_t ti = t_rowmajor ? n : 1, tj = t_rowmajor ? 1 : n;  // T(i, j) = T[i ti + j tj]
	__shared__ float Lv[2][kTcNullMax][kTcMaxNp];
	__shared__ float dg[kTcMaxNp], vp[kTcMaxNp], col[kTcMaxNp];
	__shared__ float red[8];
	__shared__ int redi[8];
	__shared__ float s_best;
	__shared__ int s_piv, s_d[2], s_bad;
	if (threadIdx.x == 0) s_bad = 0;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int m = 0; m < 2; m++) {
		// M = I - S^T S with S(k, i) = T(k, i) (m = 0: E, the right null space) or T(i, k) (m = 1: F,
		// the left null space)
		const int64_t sk = m ? tj : ti, si = m ? ti : tj;
		tc_cols_dot(T, sk, si, n, nullptr, col);
		__syncthreads();
		for (int i = threadIdx.x; i < n; i += blockDim.x) dg[i] = 1.f - col[i];
		int d = 0;
		for (;;) {
			__syncthreads();
			// largest remaining diagonal entry (first index on ties)
			float best = -1.f;
			int bi = 0;
			for (int i = threadIdx.x; i < n; i += blockDim.x) {
				const float v = dg[i];
				if (v > best) { best = v; bi = i; }
			}
			for (int o = 16; o > 0; o >>= 1) {
				const float ob = __shfl_xor_sync(0xffffffffu, best, o);
				const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
				if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
			}
			if (lane == 0) { red[warp] = best; redi[warp] = bi; }
			__syncthreads();
			if (threadIdx.x == 0) {
				float b = -1.f;
				int p = 0;
				for (int q = 0; q < 8; q++)
					if (red[q] > b || (red[q] == b && redi[q] < p)) { b = red[q]; p = redi[q]; }
				s_best = b;
				s_piv = p;
			}
			__syncthreads();
			if (s_best < 1e-4f) break;
			if (d == kTcNullMax) {
				if (threadIdx.x == 0) s_bad = 1;
				break;
			}
			const int p = s_piv;
			const float inv = rsqrtf(s_best);
			// column p of M minus the earlier factor columns: L_d = (e_p - S^T S(:, p) - sum_j L_j L_j(p)) / sqrt(M_pp)
			for (int k = threadIdx.x; k < n; k += blockDim.x) vp[k] = T[k * sk + p * si];
			__syncthreads();
			tc_cols_dot(T, sk, si, n, vp, col);
			__syncthreads();
			for (int i = threadIdx.x; i < n; i += blockDim.x) {
				float v = (i == p ? 1.f : 0.f) - col[i];
				for (int j = 0; j < d; j++) v -= Lv[m][j][i] * Lv[m][j][p];
				v *= inv;
				Lv[m][d][i] = v;
				dg[i] -= v * v;
			}
			d++;
		}
		if (threadIdx.x == 0) s_d[m] = d;
		__syncthreads();
	}
	if (s_bad || s_d[0] != s_d[1] || s_d[0] == 0) return;
	const int d = s_d[0];
	// the bases must be orthonormal already; then two Gram-Schmidt passes make them so to rounding
	for (int m = 0; m < 2; m++) {
		for (int a = 0; a < d; a++)
			for (int b = 0; b <= a; b++) {
				float v = 0.f;
				for (int i = threadIdx.x; i < n; i += blockDim.x) v += Lv[m][a][i] * Lv[m][b][i];
				v = block_sum256(v, red);
				if (fabsf(v - (a == b ? 1.f : 0.f)) > 1e-3f) {
					if (threadIdx.x == 0) s_bad = 1;
				}
			}
		__syncthreads();
		if (s_bad) return;
		for (int a = 0; a < d; a++) {
			for (int pass = 0; pass < 2; pass++)
				for (int b = 0; b < a; b++) {
					float v = 0.f;
					for (int i = threadIdx.x; i < n; i += blockDim.x) v += Lv[m][a][i] * Lv[m][b][i];
					v = block_sum256(v, red);
					for (int i = threadIdx.x; i < n; i += blockDim.x) Lv[m][a][i] -= v * Lv[m][b][i];
					__syncthreads();
				}
			float v = 0.f;
			for (int i = threadIdx.x; i < n; i += blockDim.x) v += Lv[m][a][i] * Lv[m][a][i];
			v = rsqrtf(block_sum256(v, red));
			for (int i = threadIdx.x; i < n; i += blockDim.x) Lv[m][a][i] *= v;
			__syncthreads();
		}
	}
	// T <- (I - U_0 U_0^T) T + U_0 V_0^T  (U_0 = the left null basis from F, V_0 from E): first the
	// coefficients c(a, j) = U_0(:, a)^T T(:, j) of every column (one thread per column for row-major
	// T, one warp per column for column-major T), then every entry independently
	if (tj == 1) {
		for (int j = threadIdx.x; j < n; j += blockDim.x) {
			float c[kTcNullMax];
#pragma unroll
			for (int a = 0; a < kTcNullMax; a++) c[a] = 0.f;
			for (int i = 0; i < n; i++) {
				const float t = T[i * ti + j];
#pragma unroll
				for (int a = 0; a < kTcNullMax; a++)
					if (a < d) c[a] = fmaf(Lv[1][a][i], t, c[a]);
			}
#pragma unroll
			for (int a = 0; a < kTcNullMax; a++)
				if (a < d) Cs[a * n + j] = c[a];
		}
	} else {
		for (int j = warp; j < n; j += blockDim.x >> 5) {
			float c[kTcNullMax];
#pragma unroll
			for (int a = 0; a < kTcNullMax; a++) c[a] = 0.f;
			for (int i = lane; i < n; i += 32) {
				const float t = T[i + j * tj];
#pragma unroll
				for (int a = 0; a < kTcNullMax; a++)
					if (a < d) c[a] = fmaf(Lv[1][a][i], t, c[a]);
			}
#pragma unroll
			for (int a = 0; a < kTcNullMax; a++)
				if (a < d) {
					const float sum = warp_sum(c[a]);
					if (lane == 0) Cs[a * n + j] = sum;
				}
		}
	}
	__syncthreads();
	for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
		const int r = (int)(e / n), q = (int)(e - (int64_t)r * n);
		const int i = t_rowmajor ? r : q, j = t_rowmajor ? q : r;
		float v = T[e];
		for (int a = 0; a < d; a++) v += Lv[1][a][i] * (Lv[0][a][j] - Cs[a * n + j]);
		T[e] = v;
	}
	if (threadIdx.x == 0) {
		SlStats st = stats[w.slot];
		st.flags = (st.flags & ~kFlagIllCond) | kFlagCompleted;
		stats[w.slot] = st;
	}
}

// Row-major FP32 n x n (leading dimension n) -> the iteration's two core-tiled FP16 planes of np x
// np; unpack reverses it ((hi + mid) / 2^12).  Used by the product self-test.
__global__ void k_tc_pack(const float *__restrict__ M, int n, int np, __nv_bfloat16 *__restrict__ planes) {
	const int npg = np >> 3;
	const int64_t pe = (int64_t)np * np;
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)np * npg; e += (int64_t)gridDim.x * blockDim.x) {
		const int row = (int)(e / npg), cg = (int)(e - (int64_t)row * npg);
		float v[8];
		for (int q = 0; q < 8; q++) {
			const int col = 8 * cg + q;
			v[q] = (row < n && col < n) ? M[(int64_t)row * n + col] : 0.f;
		}
		const int64_t o = ((int64_t)(row >> 3) * npg + cg) * 64 + (row & 7) * 8;
		store_split8h(v, planes + o, planes + pe + o);
	}
}
__global__ void k_tc_unpack(const __nv_bfloat16 *__restrict__ planes, int n, int np, float *__restrict__ M) {
	const int npg = np >> 3;
	const int64_t pe = (int64_t)np * np;
	for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n; e += (int64_t)gridDim.x * blockDim.x) {
		const int row = (int)(e / n), col = (int)(e - (int64_t)row * n);
		const int64_t o = ((int64_t)(row >> 3) * npg + (col >> 3)) * 64 + (row & 7) * 8 + (col & 7);
		const __half *hp = reinterpret_cast<const __half *>(planes);
		M[e] = (__half2float(hp[o]) + __half2float(hp[pe + o])) * (1.f / kTcOpScale);
	}
}

}  // namespace hab200
