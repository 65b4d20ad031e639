// ha_b200_mlp.cuh -- the learned (alpha, PC count) proposal: a 3-layer perceptron trained and run
// on the GPU by the kernels below.  No reference counterpart (the reference only has the full
// grid search, csrc/ha_ridge.c:97-345).
//
// Network: x (65 = 64 normalised singular values + log n) -> 128 GELU -> 128 GELU -> C logits,
// softmax over the C grid points (C = n_alphas * n_npcs, grid order g = a * n_npcs + p).
// Parameters, float32, packed: W1[65][128], b1[128], W2[128][128], b2[128], W3[128][C], b3[C]
// (W[i][j] = weight from input i to output j, row-major).
//
// Training: mean cross-entropy over a mini-batch; k_mlp_fwdbwd computes the forward and backward
// pass of 32 samples per CTA and writes that CTA's gradient sum; k_mlp_adam adds the CTA sums in
// CTA order (deterministic) and applies an Adam step.  Inference (k_mlp_infer) reads bfloat16
// copies of the weights and the features and accumulates in float32.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace hab200 {

constexpr int kMlpIn = 65;
constexpr int kMlpHidden = 128;
constexpr int kMlpMaxClasses = 64;
constexpr int kMlpSamples = 32;  // samples per CTA

struct MlpLayout {
	int64_t W1, b1, W2, b2, W3, b3, total;
	__host__ __device__ static MlpLayout make(int C) {
		MlpLayout L;
		int64_t o = 0;
		L.W1 = o; o += (int64_t)kMlpIn * kMlpHidden;
		L.b1 = o; o += kMlpHidden;
		L.W2 = o; o += (int64_t)kMlpHidden * kMlpHidden;
		L.b2 = o; o += kMlpHidden;
		L.W3 = o; o += (int64_t)kMlpHidden * C;
		L.b3 = o; o += C;
		L.total = o;
		return L;
	}
};

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
	return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Dense layer for the CTA's samples: out[s][j] = b[j] + sum_i in[s][i] W[i][j] (then GELU when
// act), in/out in shared memory with row strides ldi / ldo.  Threads take output units j (coalesced
// weight reads) and a strided subset of the samples.
template <typename WT>
__device__ __forceinline__ void mlp_dense(const float *in, int ldi, int nin, const WT *W, const WT *b, int nout,
                                          float *zout, float *hout, int ldo, int ns) {
	// work items: (unit j, sample group); each thread keeps up to kMlpSamples accumulators
	const int groups = (int)blockDim.x / nout;  // thread groups over the samples (nout <= blockDim.x)
	const int t = threadIdx.x;
	const int j = t % nout, grp = t / nout;
	if (grp >= groups || t >= groups * nout) return;
	float acc[kMlpSamples];
#pragma unroll
	for (int q = 0; q < kMlpSamples; q++) acc[q] = 0.0f;
	for (int i = 0; i < nin; i++) {
		const float w = (float)W[(int64_t)i * nout + j];
#pragma unroll
		for (int q = 0; q < kMlpSamples; q++) {
			const int s = grp + q * groups;
			if (s < ns) acc[q] += in[s * ldi + i] * w;
		}
	}
	const float bj = (float)b[j];
#pragma unroll
	for (int q = 0; q < kMlpSamples; q++) {
		const int s = grp + q * groups;
		if (s < ns) {
			const float z = acc[q] + bj;
			zout[s * ldo + j] = z;
			if (hout) hout[s * ldo + j] = gelu_f(z);
		}
	}
}

// Forward and backward pass of up to 32 samples per CTA.  idx (may be null) lists the samples of
// the mini-batch (sample k of the batch is idx[k], else k); scale multiplies the per-sample
// gradients (1 / batch size for the mean loss).  grad_part[blockIdx.x][P] receives the CTA's
// gradient sum and loss_part[blockIdx.x] its summed cross-entropy.
__global__ void __launch_bounds__(256) k_mlp_fwdbwd(const float *__restrict__ prm, int C, const float *__restrict__ X,
                                                    const int32_t *__restrict__ Y, const int32_t *__restrict__ idx,
                                                    int nb, float scale, float *__restrict__ grad_part,
                                                    float *__restrict__ loss_part) {
	extern __shared__ __align__(16) float sm[];
	const MlpLayout L = MlpLayout::make(C);
	const int s0 = blockIdx.x * kMlpSamples;
	const int ns = min(kMlpSamples, nb - s0);
	float *xs = sm;                                   // [32][65]
	float *z1 = xs + kMlpSamples * kMlpIn;            // [32][128]
	float *h1 = z1 + kMlpSamples * kMlpHidden;
	float *z2 = h1 + kMlpSamples * kMlpHidden;
	float *h2 = z2 + kMlpSamples * kMlpHidden;
	float *d3 = h2 + kMlpSamples * kMlpHidden;        // [32][C]
	__shared__ int ys[kMlpSamples];
	__shared__ float lsum[kMlpSamples];
	for (int e = threadIdx.x; e < ns * kMlpIn; e += blockDim.x) {
		const int s = e / kMlpIn, i = e - s * kMlpIn;
		const int g = idx ? idx[s0 + s] : s0 + s;
		xs[e] = X[(int64_t)g * kMlpIn + i];
	}
	for (int s = threadIdx.x; s < ns; s += blockDim.x) ys[s] = Y[idx ? idx[s0 + s] : s0 + s];
	__syncthreads();
	mlp_dense<float>(xs, kMlpIn, kMlpIn, prm + L.W1, prm + L.b1, kMlpHidden, z1, h1, kMlpHidden, ns);
	__syncthreads();
	mlp_dense<float>(h1, kMlpHidden, kMlpHidden, prm + L.W2, prm + L.b2, kMlpHidden, z2, h2, kMlpHidden, ns);
	__syncthreads();
	mlp_dense<float>(h2, kMlpHidden, kMlpHidden, prm + L.W3, prm + L.b3, C, d3, nullptr, C, ns);
	__syncthreads();
	// softmax and cross-entropy per sample (one warp per sample); d3 <- (p - onehot) * scale
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	for (int s = warp; s < ns; s += nwarp) {
		float *z = d3 + s * C;
		float mx = -INFINITY;
		for (int c = lane; c < C; c += 32) mx = fmaxf(mx, z[c]);
		for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
		float se = 0.0f;
		for (int c = lane; c < C; c += 32) se += expf(z[c] - mx);
		for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
		const float lse = mx + logf(se);
		const int y = ys[s];
		if (lane == 0) lsum[s] = lse - z[y];
		__syncwarp();
		for (int c = lane; c < C; c += 32) {
			const float p = expf(z[c] - lse);
			z[c] = (p - (c == y ? 1.0f : 0.0f)) * scale;
		}
	}
	__syncthreads();
	float *G = grad_part + (int64_t)blockIdx.x * L.total;
	// layer 3: dW3[k][c] = sum_s h2[s][k] d3[s][c], db3[c] = sum_s d3[s][c]
	for (int e = threadIdx.x; e < kMlpHidden * C; e += blockDim.x) {
		const int k = e / C, c = e - k * C;
		float a = 0.0f;
		for (int s = 0; s < ns; s++) a += h2[s * kMlpHidden + k] * d3[s * C + c];
		G[L.W3 + e] = a;
	}
	for (int c = threadIdx.x; c < C; c += blockDim.x) {
		float a = 0.0f;
		for (int s = 0; s < ns; s++) a += d3[s * C + c];
		G[L.b3 + c] = a;
	}
	// dz2[s][k] = (sum_c d3[s][c] W3[k][c]) * gelu'(z2[s][k])  -> stored over h2
	const float *W3 = prm + L.W3;
	__syncthreads();
	for (int e = threadIdx.x; e < ns * kMlpHidden; e += blockDim.x) {
		const int s = e / kMlpHidden, k = e - s * kMlpHidden;
		float a = 0.0f;
		for (int c = 0; c < C; c++) a += d3[s * C + c] * W3[(int64_t)k * C + c];
		h2[e] = a * gelu_grad(z2[e]);
	}
	__syncthreads();
	// layer 2: dW2[i][k] = sum_s h1[s][i] dz2[s][k], db2[k]
	for (int e = threadIdx.x; e < kMlpHidden * kMlpHidden; e += blockDim.x) {
		const int i = e / kMlpHidden, k = e - i * kMlpHidden;
		float a = 0.0f;
		for (int s = 0; s < ns; s++) a += h1[s * kMlpHidden + i] * h2[s * kMlpHidden + k];
		G[L.W2 + e] = a;
	}
	for (int k = threadIdx.x; k < kMlpHidden; k += blockDim.x) {
		float a = 0.0f;
		for (int s = 0; s < ns; s++) a += h2[s * kMlpHidden + k];
		G[L.b2 + k] = a;
	}
	// dz1[s][i] = (sum_k dz2[s][k] W2[i][k]) * gelu'(z1[s][i])  -> stored over h1
	const float *W2 = prm + L.W2;
	__syncthreads();
	for (int e = threadIdx.x; e < ns * kMlpHidden; e += blockDim.x) {
		const int s = e / kMlpHidden, i = e - s * kMlpHidden;
		float a = 0.0f;
		for (int k = 0; k < kMlpHidden; k++) a += h2[s * kMlpHidden + k] * W2[(int64_t)i * kMlpHidden + k];
		h1[e] = a * gelu_grad(z1[e]);
	}
	__syncthreads();
	// layer 1: dW1[i][j] = sum_s x[s][i] dz1[s][j], db1[j]
	for (int e = threadIdx.x; e < kMlpIn * kMlpHidden; e += blockDim.x) {
		const int i = e / kMlpHidden, j = e - i * kMlpHidden;
		float a = 0.0f;
		for (int s = 0; s < ns; s++) a += xs[s * kMlpIn + i] * h1[s * kMlpHidden + j];
		G[L.W1 + e] = a;
	}
	for (int j = threadIdx.x; j < kMlpHidden; j += blockDim.x) {
		float a = 0.0f;
		for (int s = 0; s < ns; s++) a += h1[s * kMlpHidden + j];
		G[L.b1 + j] = a;
	}
	if (threadIdx.x == 0) {
		float a = 0.0f;
		for (int s = 0; s < ns; s++) a += lsum[s];
		loss_part[blockIdx.x] = a;
	}
}

// g = sum over the nparts CTA gradients (in CTA order); then either out = g (grad_out) or an Adam
// step on the parameters (m, v moments; bias corrections bc1 = 1 - beta1^t, bc2 = 1 - beta2^t).
__global__ void k_mlp_adam(float *__restrict__ prm, const float *__restrict__ grad_part, int nparts, int64_t P,
                           float *__restrict__ m, float *__restrict__ v, float lr, float beta1, float beta2, float eps,
                           float bc1, float bc2, float *__restrict__ grad_out) {
	const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= P) return;
	float g = 0.0f;
	for (int b = 0; b < nparts; b++) g += grad_part[(int64_t)b * P + p];
	if (grad_out) {
		grad_out[p] = g;
		return;
	}
	const float mm = beta1 * m[p] + (1.0f - beta1) * g;
	const float vv = beta2 * v[p] + (1.0f - beta2) * g * g;
	m[p] = mm;
	v[p] = vv;
	prm[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

__global__ void k_f32_to_bf16(const float *__restrict__ in, __nv_bfloat16 *__restrict__ out, int64_t n) {
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = __float2bfloat16_rn(in[i]);
}

// Inference with bfloat16 weights and features (float32 accumulation): the most probable grid
// point (ties to the lower index) and its softmax probability.
__global__ void __launch_bounds__(256) k_mlp_infer(const __nv_bfloat16 *__restrict__ prm, int C,
                                                   const float *__restrict__ X, int n, int32_t *__restrict__ cls,
                                                   float *__restrict__ prob) {
	extern __shared__ __align__(16) float sm[];
	const MlpLayout L = MlpLayout::make(C);
	const int s0 = blockIdx.x * kMlpSamples;
	const int ns = min(kMlpSamples, n - s0);
	float *xs = sm;
	float *z1 = xs + kMlpSamples * kMlpIn;
	float *h1 = z1 + kMlpSamples * kMlpHidden;
	float *z2 = h1 + kMlpSamples * kMlpHidden;
	float *h2 = z2 + kMlpSamples * kMlpHidden;
	float *z3 = h2 + kMlpSamples * kMlpHidden;
	for (int e = threadIdx.x; e < ns * kMlpIn; e += blockDim.x)
		xs[e] = __bfloat162float(__float2bfloat16_rn(X[(int64_t)s0 * kMlpIn + e]));
	__syncthreads();
	mlp_dense<__nv_bfloat16>(xs, kMlpIn, kMlpIn, prm + L.W1, prm + L.b1, kMlpHidden, z1, h1, kMlpHidden, ns);
	__syncthreads();
	mlp_dense<__nv_bfloat16>(h1, kMlpHidden, kMlpHidden, prm + L.W2, prm + L.b2, kMlpHidden, z2, h2, kMlpHidden, ns);
	__syncthreads();
	mlp_dense<__nv_bfloat16>(h2, kMlpHidden, kMlpHidden, prm + L.W3, prm + L.b3, C, z3, nullptr, C, ns);
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
	for (int s = warp; s < ns; s += nwarp) {
		const float *z = z3 + s * C;
		float mx = -INFINITY;
		int am = 0x7fffffff;
		for (int c = lane; c < C; c += 32)
			if (z[c] > mx) { mx = z[c]; am = c; }
		for (int o = 16; o > 0; o >>= 1) {
			const float om = __shfl_xor_sync(0xffffffffu, mx, o);
			const int oa = __shfl_xor_sync(0xffffffffu, am, o);
			if (om > mx || (om == mx && oa < am)) { mx = om; am = oa; }
		}
		float se = 0.0f;
		for (int c = lane; c < C; c += 32) se += expf(z[c] - mx);
		for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
		if (lane == 0) {
			cls[s0 + s] = am;
			prob[s0 + s] = 1.0f / se;
		}
	}
}

}  // namespace hab200
