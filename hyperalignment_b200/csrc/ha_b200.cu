// ha_b200.cu -- host side of the B200 searchlight alignment backend: plans, launches and the C ABI.
//
// A plan holds everything that depends only on the searchlight geometry (weights, per-vertex
// membership lists, the symmetric CSC pattern, size buckets, scratch layout).  A run converts
// the float64 inputs on the device, solves every searchlight (cross-covariance, Jacobi polar,
// refinement, reflection fix) chunk by chunk, and reduces the weighted local transforms into
// the pattern's values with a deterministic segmented reduction.

#include "../../include/hyperalignment_b200.h"
#include "ha_b200_kernels.cuh"
#include "ha_b200_grid.cuh"
#include "ha_b200_mlp.cuh"
#include "ha_b200_tc.cuh"
#include "ha_b200_pca.cuh"

#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

using namespace hab200;

namespace {

constexpr int kBlock = 256;
constexpr size_t kSmemMax = 220 * 1024;  // dynamic shared memory budget per CTA (B200 opt-in max is 227 KB)

#define HA_CUDA(call)                                                                              \
	do {                                                                                           \
		cudaError_t e_ = (call);                                                                   \
		if (e_ != cudaSuccess) {                                                                   \
			fprintf(stderr, "ha_b200: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_),     \
			        __FILE__, __LINE__);                                                           \
			return kHaErrorInternal;                                                               \
		}                                                                                          \
	} while (0)

std::recursive_mutex g_mu;
bool g_inited = false;
int g_threads = 0;

// ---- launch tracing: optional CUDA events around every launch, and a launch counter ----
int64_t g_launches = 0;
bool g_timing = false;
struct TimedLaunch {
	int kind;
	cudaEvent_t a, b;
};
std::vector<TimedLaunch> g_timed;
cudaEvent_t g_time_base = nullptr;  // recorded when timing starts and after every read-out
double g_kernel_ms[kHaB200NumKernelKinds] = {0};
int64_t g_kernel_n[kHaB200NumKernelKinds] = {0};

struct LaunchScope {
	int kind;
	cudaStream_t st;
	cudaEvent_t a = nullptr, b = nullptr;
	LaunchScope(int k, cudaStream_t s) : kind(k), st(s) {
		g_launches++;
		g_kernel_n[k]++;
		if (g_timing && cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess)
			cudaEventRecord(a, st);
	}
	~LaunchScope() {
		if (a && b) {
			cudaEventRecord(b, st);
			g_timed.push_back({kind, a, b});
		}
	}
};
#define HA_LAUNCH(kind, st) LaunchScope ha_scope_##__LINE__((kind), (st))

template <typename T>
struct DevArr {
	T *p = nullptr;
	size_t n = 0;  // capacity in elements
	int ensure(size_t count) {
		if (count <= n && p) return kHaSuccess;
		if (p) cudaFree(p);
		p = nullptr;
		n = 0;
		size_t want = std::max<size_t>(count, 1);
		if (cudaMalloc(&p, want * sizeof(T)) != cudaSuccess) {
			cudaGetLastError();
			fprintf(stderr, "ha_b200: cudaMalloc of %zu bytes failed\n", want * sizeof(T));
			p = nullptr;
			return kHaErrorAlloc;
		}
		n = want;
		return kHaSuccess;
	}
	void release() {
		if (p) cudaFree(p);
		p = nullptr;
		n = 0;
	}
};

// Buffers for the host-memory entry points (inputs, outputs), kept between calls.
struct HostCallBufs {
	DevArr<double> X64, Y64, Xtmp, vals;
	std::vector<double> h_vals;
	void release() {
		X64.release(); Y64.release(); Xtmp.release(); vals.release();
		std::vector<double>().swap(h_vals);
	}
} g_bufs;

size_t real_bytes(bool fp64) { return fp64 ? 8 : 4; }

// Jacobi kernel instances: rows per lane (column length <= 32 * rpl)
const int kRplSet[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16};
int rpl_for(int n) {
	for (int r : kRplSet)
		if (n <= 32 * r) return r;
	return -1;
}

// Shared memory of k_jacobi for 2*b staged columns (plus the zero pair) of LD rows: A and V
// columns, norms and the GEMM tiles of the polar factor; in eigenvector mode (no V) A and norms.
size_t jacobi_smem(int b, int ld, size_t rb, bool with_v = true) {
	const size_t mst = (size_t)2 * b + 2;
	if (!with_v) return (mst * ld + mst + 2 + 8) * rb;
	return (2 * mst * ld + mst + 2 + 2 * 16 * 65 + 8) * rb;
}

// Jacobi block layout for a searchlight of n vertices in a given precision: resident (two
// blocks covering all columns stay in shared memory) when it fits, else blocked with the
// widest block that fits.
// Eigenvector mode (no V) stages twice the columns in the same memory, so its blocks may be wider.
void jacobi_layout(int n, bool fp64, int &bsz, int &nblk, size_t &smem, size_t budget, bool with_v = true) {
	const size_t rb = real_bytes(fp64);
	const int ld = 32 * std::max(1, rpl_for(n));
	int h = (n + 1) / 2;
	size_t res = jacobi_smem(h, ld, rb, with_v);
	if (res <= budget) {
		bsz = h;
		nblk = 2;
		smem = res;
		return;
	}
	int b = with_v ? 32 : 64;
	while (b > 2 && jacobi_smem(b, ld, rb, with_v) > budget) b--;
	b -= b & 1;  // even blocks: the round robin inside one block needs an even column count
	bsz = b;
	nblk = (n + b - 1) / b;
	if (nblk & 1) nblk++;
	smem = jacobi_smem(b, ld, rb, with_v);
}

void jacobi_layout(int n, bool fp64, int &bsz, int &nblk, size_t &smem) {
	jacobi_layout(n, fp64, bsz, nblk, smem, kSmemMax);
}

// Shared-memory budget of the plan's FP32 Jacobi buckets: small enough for two CTAs per SM
// (the float instances are register-bounded to two 512-thread CTAs), so more searchlights run
// in blocked mode through L2 but twice as many warps hide the rotation latencies.
// HA_B200_JACOBI_SMEM_KB overrides it (upper bound 220).
size_t fp32_jacobi_budget() {
	static size_t b = 0;
	if (!b) {
		const char *e = getenv("HA_B200_JACOBI_SMEM_KB");
		double kb = e ? atof(e) : 110.0;
		if (!(kb >= 16.0)) kb = 110.0;
		b = std::min(kSmemMax, (size_t)(kb * 1024.0));
	}
	return b;
}

// Side streams for the size buckets of a chunk.  Buckets own disjoint scratch regions, so their
// kernels may overlap and fill the SMs that one bucket's last wave leaves idle; begin() makes
// every side stream wait for the caller's stream, end() makes the caller's stream wait for all.
struct StreamFan {
	static constexpr int kN = 6;
	cudaStream_t s[kN] = {};
	cudaEvent_t fork = nullptr, join[kN] = {};
	bool ready = false;
	int init() {
		if (ready) return kHaSuccess;
		for (int i = 0; i < kN; i++) {
			HA_CUDA(cudaStreamCreateWithFlags(&s[i], cudaStreamNonBlocking));
			HA_CUDA(cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming));
		}
		HA_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
		ready = true;
		return kHaSuccess;
	}
	int begin(cudaStream_t main) {
		int rc = init();
		if (rc != kHaSuccess) return rc;
		HA_CUDA(cudaEventRecord(fork, main));
		for (int i = 0; i < kN; i++) HA_CUDA(cudaStreamWaitEvent(s[i], fork, 0));
		return kHaSuccess;
	}
	cudaStream_t at(int i) const { return s[i % kN]; }
	int end(cudaStream_t main) {
		for (int i = 0; i < kN; i++) {
			HA_CUDA(cudaEventRecord(join[i], s[i]));
			HA_CUDA(cudaStreamWaitEvent(main, join[i], 0));
		}
		return kHaSuccess;
	}
	void release() {
		if (!ready) return;
		for (int i = 0; i < kN; i++) {
			cudaStreamDestroy(s[i]);
			cudaEventDestroy(join[i]);
		}
		cudaEventDestroy(fork);
		ready = false;
	}
} g_fan;

struct Bucket {
	int first, count;  // range in the chunk's work array
	size_t smem;
	bool blocked;
	int threads;       // Jacobi block size: about two column pairs per warp per round
	int rpl;           // rows per lane of the Jacobi kernel instance (n <= 32 * rpl)
};

template <typename Real>
int launch_jacobi(int rpl, int grid, int threads, size_t smem, cudaStream_t st, const SlWork *wk, Real *A, Real *V,
                  float *T, SlStats *stats, double *uv, JacobiParams jp) {
	switch (rpl) {
#define HA_RPL_CASE(R) \
	case R: k_jacobi<Real, R><<<grid, std::min(threads, JacobiBounds<Real, R>::threads), smem, st>>>(wk, A, V, T, stats, uv, jp); break;
		HA_RPL_CASE(1) HA_RPL_CASE(2) HA_RPL_CASE(3) HA_RPL_CASE(4) HA_RPL_CASE(5)
		HA_RPL_CASE(6) HA_RPL_CASE(8) HA_RPL_CASE(10) HA_RPL_CASE(12) HA_RPL_CASE(16)
#undef HA_RPL_CASE
	default:
		fprintf(stderr, "ha_b200: no Jacobi kernel for %d rows per lane\n", rpl);
		return kHaErrorArg;
	}
	return kHaSuccess;
}

template <typename Real>
int set_jacobi_attrs() {
	const int m = (int)kSmemMax;
#define HA_RPL_ATTR(R) \
	if (cudaFuncSetAttribute(k_jacobi<Real, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, m) != cudaSuccess) \
		return kHaErrorInternal;
	HA_RPL_ATTR(1) HA_RPL_ATTR(2) HA_RPL_ATTR(3) HA_RPL_ATTR(4) HA_RPL_ATTR(5)
	HA_RPL_ATTR(6) HA_RPL_ATTR(8) HA_RPL_ATTR(10) HA_RPL_ATTR(12) HA_RPL_ATTR(16)
#undef HA_RPL_ATTR
	return kHaSuccess;
}

int jacobi_threads(int bsz, bool fp64) {
	int warps = (bsz + 1) / 2;
	(void)fp64;
	warps = std::max(8, std::min(16, warps));
	return warps * 32;
}

struct Chunk {
	int s0, s1;
	std::vector<SlWork> w32, w64, weig;  // float32 polar, float64 polar, float64 eigenvector mode
	std::vector<Bucket> b32, b64, beig;
	std::vector<SlWork> weig32;  // float32 eigenvector mode (the plain FP32 grid search)
	std::vector<Bucket> beig32;
	std::vector<int64_t> tofs;  // per slot
	int64_t scratch_elems8;     // scratch size in 8-byte units (A and V each)
	int64_t t_elems;            // T scratch floats
	int64_t uv_elems;
	SlWork *d_w32 = nullptr, *d_w64 = nullptr, *d_weig = nullptr, *d_weig32 = nullptr;
	int64_t *d_tofs = nullptr;
	// tensor-core solve: one work item per searchlight (slot order), 128-row tiles in two size
	// classes (np <= 256: two CTAs per SM; np > 256), largest searchlights first
	std::vector<TcWork> tcw;
	std::vector<TcTile> tct[2];
	TcWork *d_tcw = nullptr;
	TcTile *d_tct[2] = {nullptr, nullptr};
	std::vector<int32_t> tco[2];  // persistent solve: work indices per size class, largest first
	int32_t *d_tco[2] = {nullptr, nullptr};
	// the tensor-core iteration loop of this chunk captured as a CUDA graph, and what it was
	// captured for (output order, layouts); replayed while those are unchanged
	cudaGraphExec_t tc_graph = nullptr;
	int tc_graph_key[3] = {-1, -1, -1};
	int tc_graph_kernels = 0;
	int64_t tc_x_elems = 0, tc_a_elems = 0;
};

}  // namespace

struct HaB200Plan {
	int nt = 0, nv = 0, count = 0;
	int64_t total = 0;
	int max_n = 0;
	std::vector<int32_t> h_off, h_idx;
	std::vector<double> h_w;
	bool has_weights = true;
	// device geometry
	DevArr<int32_t> idx, off, lo, hi;
	DevArr<double> w;
	DevArr<int64_t> vlptr;
	DevArr<int2> vlent;
	DevArr<int64_t> patptr;
	DevArr<int32_t> patcol;
	int64_t nnz = 0;
	int max_row = 0;
	std::vector<int64_t> h_patptr;
	std::vector<int32_t> h_patcol;
	// chunks and scratch
	std::vector<Chunk> chunks;
	DevArr<double> scrA, scrV;  // 8-byte units, reinterpreted per precision
	DevArr<float> scrT;
	DevArr<double> scrT64;  // float64 local results (ridge), allocated on first use
	DevArr<double> uv, scale;
	DevArr<SlStats> stats;
	int max_slots = 0;
	// per-run data
	DevArr<float> X32, Y32;
	DevArr<double> var;
	DevArr<int32_t> counters;  // [n_fp64, n_unconverged, sweeps sum, sweeps max, tensor-core wait failures]
	// tensor-core solve, allocated on first use: vertex-major bf16 planes of X and Y, iterate and P
	// planes, cross-covariance, iteration state (two copies) and residual partials
	DevArr<__nv_bfloat16> tcXb, tcYb, tcXp, tcXq, tcPp;
	DevArr<float> tcA, tcRes;
	DevArr<TcState> tcSt;
	DevArr<float> tcSched;      // c1[maxit], c3[maxit] of the iteration schedule
	DevArr<int32_t> tcPlain;    // plain[maxit]
	DevArr<int32_t> tcQueue;    // work queue positions of the persistent solve (two size classes)
	bool tc_ready = false;
	// tile layout of the per-phase launches per size class (tiles of <= 128 columns, of 129-256):
	// dynamic shared memory per CTA, which sets the CTAs per SM and the pipeline depth; chosen by
	// timing the candidates on the plan's first tensor-core run (autotune_tc), or pinned
	int tc_smem[2] = {110 * 1024, 110 * 1024};
	bool tc_tuned = false;
	// the ridge grid search captured as a CUDA graph, and the key it was captured for
	cudaGraphExec_t grid_graph = nullptr;
	std::vector<uint64_t> grid_key;
	int grid_bits = 64;  // arithmetic of ha_b200_plan_ridge_grid_device: 64 (float64) or 32 (plain FP32)
	int64_t grid_graph_launches = 0;
	double tc_tune_ms[2][3] = {{0}};  // measured Gram-launch times of the candidates
	// ridge grid search: scratch and the uploaded grid / CV description, allocated on first use
	DevArr<double> gridscr, galpha, gwinv;
	DevArr<int64_t> gbase;
	DevArr<int32_t> gnpcs, grows, gtpos, gurows, guntested;
	DevArr<GridModel> gmdl;
	DevArr<int32_t> gfit;      // fit rows of the learned form / the features
	DevArr<float> gfeat;       // features of the learned form
	DevArr<SlWork> gwork;      // fallback work list of the learned form
	int last_chunk = -1;
	int last_rowmajor = 1;
};

namespace {

int check_cuda_ready() {
	if (!g_inited) {
		int rc = ha_b200_init();
		if (rc != kHaSuccess) return rc;
	}
	return kHaSuccess;
}

uint64_t fnv1a(const void *data, size_t bytes, uint64_t h) {
	const unsigned char *p = (const unsigned char *)data;
	for (size_t i = 0; i < bytes; i++) {
		h ^= p[i];
		h *= 1099511628211ULL;
	}
	return h;
}

// Flat weights exactly as csrc/ha_searchlight.c:970-1001 (same operation order, float64).
void compute_weights(const int32_t *idx, const int32_t *off, const double *dists, int32_t count, double radius,
                     int32_t nv, double *out) {
	const int64_t total = off[count];
	std::vector<double> vsum((size_t)nv, 0.0);
	if (dists == nullptr) {
		for (int64_t k = 0; k < total; k++) vsum[idx[k]] += 1.0;
		for (int64_t k = 0; k < total; k++) out[k] = 1.0 / vsum[idx[k]];
	} else {
		for (int64_t k = 0; k < total; k++) {
			double w = (radius - dists[k]) / radius;
			vsum[idx[k]] += w;
		}
		for (int64_t k = 0; k < total; k++) {
			double w = (radius - dists[k]) / radius;
			out[k] = w / vsum[idx[k]];
		}
	}
}

int validate_searchlights(const int32_t *idx, const int32_t *off, int32_t count, int32_t nv) {
	if (!idx || !off || count <= 0 || nv <= 0) return kHaErrorArg;
	if (off[0] != 0) {
		fprintf(stderr, "ha_b200: sl_offsets[0] must be 0\n");
		return kHaErrorArg;
	}
	std::vector<int32_t> mark((size_t)nv, -1);
	for (int32_t s = 0; s < count; s++) {
		if (off[s + 1] <= off[s]) {
			fprintf(stderr, "ha_b200: searchlight %d is empty or offsets decrease\n", s);
			return kHaErrorArg;
		}
		for (int32_t k = off[s]; k < off[s + 1]; k++) {
			int32_t v = idx[k];
			if (v < 0 || v >= nv) {
				fprintf(stderr, "ha_b200: searchlight %d has vertex %d outside [0, %d)\n", s, v, nv);
				return kHaErrorArg;
			}
			if (mark[v] == s) {
				fprintf(stderr, "ha_b200: searchlight %d lists vertex %d twice\n", s, v);
				return kHaErrorArg;
			}
			mark[v] = s;
		}
	}
	return kHaSuccess;
}

size_t scratch_budget_bytes() {
	const char *e = getenv("HA_B200_SCRATCH_GB");
	double gb = e ? atof(e) : 16.0;
	if (!(gb > 0.01)) gb = 16.0;
	return (size_t)(gb * 1073741824.0);
}

// Sort work items by Jacobi class (resident or blocked, rows per lane), largest first inside a
// class, and cut them into buckets of one Jacobi kernel instance each.  prec: 0 float32 polar,
// 1 float64 polar, 2 float64 eigenvector mode, 3 float32 eigenvector mode.
std::vector<Bucket> bucketize(std::vector<SlWork> &items, int prec) {
	auto key = [](const SlWork &w) { return (w.nblk == 2 ? 0 : 32) + rpl_for(w.n); };
	std::stable_sort(items.begin(), items.end(), [&](const SlWork &a, const SlWork &b) {
		int ka = key(a), kb = key(b);
		if (ka != kb) return ka < kb;
		return a.n > b.n;
	});
	std::vector<Bucket> buckets;
	for (int i = 0; i < (int)items.size();) {
		int j = i;
		size_t smem = 0;
		while (j < (int)items.size() && key(items[j]) == key(items[i])) {
			int bb, kk;
			size_t mm;
			const bool f64 = prec == 1 || prec == 2;
			jacobi_layout(items[j].n, f64, bb, kk, mm, f64 ? kSmemMax : fp32_jacobi_budget(), prec < 2);
			smem = std::max(smem, mm);
			j++;
		}
		Bucket b;
		b.first = i;
		b.count = j - i;
		b.smem = smem;
		b.blocked = items[i].nblk != 2;
		b.threads = jacobi_threads(items[i].bsz, prec == 1 || prec == 2);
		b.rpl = rpl_for(items[i].n);
		buckets.push_back(b);
		i = j;
	}
	return buckets;
}

int build_chunks(HaB200Plan *P) {
	const size_t budget = scratch_budget_bytes();
	P->chunks.clear();
	int s = 0;
	while (s < P->count) {
		Chunk ch;
		ch.s0 = s;
		int64_t acc8 = 0, tacc = 0, uvacc = 0;
		std::vector<int64_t> tofs;
		std::vector<int64_t> aofs8;
		std::vector<int> bs32, nb32, bs64, nb64, bse, nbe, bse32, nbe32;
		std::vector<size_t> sm32, sm64;
		while (s < P->count) {
			int n = P->h_off[s + 1] - P->h_off[s];
			int b32, k32, b64, k64;
			size_t m32, m64;
			jacobi_layout(n, false, b32, k32, m32, fp32_jacobi_budget());
			jacobi_layout(n, true, b64, k64, m64);
			int be, ke;
			size_t me;
			jacobi_layout(n, true, be, ke, me, kSmemMax, false);
			int be32, ke32;
			jacobi_layout(n, false, be32, ke32, me, fp32_jacobi_budget(), false);
			int64_t e32 = ((int64_t)n * k32 * b32 * 4 + 7) / 8;
			int64_t e64 = (int64_t)n * k64 * b64;
			int64_t eeig = (int64_t)n * ke * be;
			int64_t eeig32 = ((int64_t)n * ke32 * be32 * 4 + 7) / 8;
			int64_t region = std::max<int64_t>(std::max(std::max(e32, e64), std::max(eeig, eeig32)), (int64_t)n * n);
			region = (region + 31) & ~(int64_t)31;
			size_t bytes_if = (size_t)(acc8 + region) * 8 * 2 + (size_t)(tacc + (int64_t)n * n) * 4;
			if (!tofs.empty() && bytes_if > budget) break;
			aofs8.push_back(acc8);
			tofs.push_back(tacc);
			acc8 += region;
			tacc += (int64_t)n * n;
			bs32.push_back(b32); nb32.push_back(k32); sm32.push_back(m32);
			bs64.push_back(b64); nb64.push_back(k64); sm64.push_back(m64);
			bse.push_back(be); nbe.push_back(ke);
			bse32.push_back(be32); nbe32.push_back(ke32);
			uvacc += 2 * (int64_t)n;
			s++;
		}
		ch.s1 = s;
		ch.scratch_elems8 = acc8;
		ch.t_elems = tacc;
		ch.uv_elems = uvacc;
		ch.tofs = tofs;
		const int nsl = ch.s1 - ch.s0;
		// work items, bucketed by (mode, n range), largest first inside a bucket
		for (int prec = 0; prec < 4; prec++) {  // float32, float64, float64 / float32 eigenvector mode
			std::vector<SlWork> items;
			int64_t uvo = 0;
			for (int q = 0; q < nsl; q++) {
				int sidx = ch.s0 + q;
				int n = P->h_off[sidx + 1] - P->h_off[sidx];
				SlWork w;
				w.s = sidx;
				w.n = n;
				w.bsz = prec == 3 ? bse32[q] : prec == 2 ? bse[q] : (prec ? bs64[q] : bs32[q]);
				w.nblk = prec == 3 ? nbe32[q] : prec == 2 ? nbe[q] : (prec ? nb64[q] : nb32[q]);
				w.aofs = (prec == 1 || prec == 2) ? aofs8[q] : aofs8[q] * 2;
				w.tofs = tofs[q];
				w.sofs = P->h_off[sidx];
				w.slot = q;
				w.uvofs = uvo;
				uvo += 2 * (int64_t)n;
				items.push_back(w);
			}
			std::vector<Bucket> buckets = bucketize(items, prec);
			if (prec == 0) { ch.w32 = items; ch.b32 = buckets; }
			else if (prec == 1) { ch.w64 = items; ch.b64 = buckets; }
			else if (prec == 2) { ch.weig = items; ch.beig = buckets; }
			else { ch.weig32 = items; ch.beig32 = buckets; }
		}
		P->chunks.push_back(std::move(ch));
	}
	// device copies of the work lists
	for (auto &ch : P->chunks) {
		size_t n32 = ch.w32.size(), n64 = ch.w64.size(), ne = ch.weig.size();
		if (cudaMalloc(&ch.d_w32, n32 * sizeof(SlWork)) != cudaSuccess) return kHaErrorAlloc;
		if (cudaMalloc(&ch.d_w64, n64 * sizeof(SlWork)) != cudaSuccess) return kHaErrorAlloc;
		if (cudaMalloc(&ch.d_weig, ne * sizeof(SlWork)) != cudaSuccess) return kHaErrorAlloc;
		HA_CUDA(cudaMemcpy(ch.d_weig, ch.weig.data(), ne * sizeof(SlWork), cudaMemcpyHostToDevice));
		if (cudaMalloc(&ch.d_weig32, ch.weig32.size() * sizeof(SlWork)) != cudaSuccess) return kHaErrorAlloc;
		HA_CUDA(cudaMemcpy(ch.d_weig32, ch.weig32.data(), ch.weig32.size() * sizeof(SlWork), cudaMemcpyHostToDevice));
		if (cudaMalloc(&ch.d_tofs, ch.tofs.size() * sizeof(int64_t)) != cudaSuccess) return kHaErrorAlloc;
		HA_CUDA(cudaMemcpy(ch.d_w32, ch.w32.data(), n32 * sizeof(SlWork), cudaMemcpyHostToDevice));
		HA_CUDA(cudaMemcpy(ch.d_w64, ch.w64.data(), n64 * sizeof(SlWork), cudaMemcpyHostToDevice));
		HA_CUDA(cudaMemcpy(ch.d_tofs, ch.tofs.data(), ch.tofs.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
	}
	int64_t max8 = 1, maxT = 1, maxUV = 1;
	int max_slots = 1;
	for (auto &ch : P->chunks) {
		max8 = std::max(max8, ch.scratch_elems8);
		maxT = std::max(maxT, ch.t_elems);
		maxUV = std::max(maxUV, ch.uv_elems);
		max_slots = std::max(max_slots, ch.s1 - ch.s0);
	}
	int rc;
	if ((rc = P->scrA.ensure((size_t)max8)) != kHaSuccess) return rc;
	if ((rc = P->scrV.ensure((size_t)max8)) != kHaSuccess) return rc;
	if ((rc = P->scrT.ensure((size_t)maxT)) != kHaSuccess) return rc;
	if ((rc = P->uv.ensure((size_t)maxUV)) != kHaSuccess) return rc;
	if ((rc = P->scale.ensure((size_t)max_slots)) != kHaSuccess) return rc;
	if ((rc = P->stats.ensure((size_t)max_slots)) != kHaSuccess) return rc;
	if ((rc = P->counters.ensure(5)) != kHaSuccess) return rc;
	P->max_slots = max_slots;
	return kHaSuccess;
}

__global__ void k_count_flags(const SlStats *__restrict__ st, int n, int32_t *__restrict__ counters) {
	int q = blockIdx.x * blockDim.x + threadIdx.x;
	if (q >= n) return;
	int f = st[q].flags;
	if (f & kFlagFP64) atomicAdd(&counters[0], 1);
	if (f & kFlagUnconverged) atomicAdd(&counters[1], 1);
	atomicAdd(&counters[2], st[q].sweeps);
	atomicMax(&counters[3], st[q].sweeps);
}

int set_smem_attrs() {
	static bool done = false;
	if (done) return kHaSuccess;
	if (set_jacobi_attrs<float>() != kHaSuccess || set_jacobi_attrs<double>() != kHaSuccess) {
		fprintf(stderr, "ha_b200: cudaFuncSetAttribute on the Jacobi kernels failed\n");
		return kHaErrorInternal;
	}
	HA_CUDA(cudaFuncSetAttribute(k_reduce<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax));
	HA_CUDA(cudaFuncSetAttribute(k_reduce<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax));
	HA_CUDA(cudaFuncSetAttribute(k_pattern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax));
	HA_CUDA(cudaFuncSetAttribute(k_pchol<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kPcholNb * kGridMaxN * 8)));
	HA_CUDA(cudaFuncSetAttribute(k_pchol<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kPcholNb * kGridMaxN * 4)));
	done = true;
	return kHaSuccess;
}

int build_pattern(HaB200Plan *P) {
	const int nv = P->nv;
	const size_t words = (size_t)nv / 32 + 2;
	if (words * 4 > kSmemMax) {
		fprintf(stderr, "ha_b200: nv = %d exceeds the pattern builder's limit\n", nv);
		return kHaErrorArg;
	}
	int rc;
	DevArr<int64_t> len;
	if ((rc = len.ensure(nv)) != kHaSuccess) return rc;
	if ((rc = P->patptr.ensure((size_t)nv + 1)) != kHaSuccess) { len.release(); return rc; }
	{ HA_LAUNCH(kHaB200KPattern, 0); k_pattern<<<nv, kBlock, words * 4>>>(P->vlptr.p, P->vlent.p, P->off.p, P->idx.p, P->lo.p, P->hi.p, nv, 0,
	                                     len.p, nullptr, nullptr); }
	HA_CUDA(cudaGetLastError());
	std::vector<int64_t> hl((size_t)nv);
	HA_CUDA(cudaMemcpy(hl.data(), len.p, (size_t)nv * sizeof(int64_t), cudaMemcpyDeviceToHost));
	P->h_patptr.assign((size_t)nv + 1, 0);
	int max_row = 0;
	for (int v = 0; v < nv; v++) {
		P->h_patptr[v + 1] = P->h_patptr[v] + hl[v];
		max_row = std::max<int>(max_row, (int)hl[v]);
	}
	P->nnz = P->h_patptr[nv];
	P->max_row = max_row;
	HA_CUDA(cudaMemcpy(P->patptr.p, P->h_patptr.data(), ((size_t)nv + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
	if ((rc = P->patcol.ensure((size_t)P->nnz)) != kHaSuccess) { len.release(); return rc; }
	{ HA_LAUNCH(kHaB200KPattern, 0); k_pattern<<<nv, kBlock, words * 4>>>(P->vlptr.p, P->vlent.p, P->off.p, P->idx.p, P->lo.p, P->hi.p, nv, 1,
	                                     len.p, P->patptr.p, P->patcol.p); }
	HA_CUDA(cudaGetLastError());
	HA_CUDA(cudaDeviceSynchronize());
	len.release();
	return kHaSuccess;
}

int plan_create_impl(int32_t nt, int32_t nv, const int32_t *sl_indices, const int32_t *sl_offsets,
                     const double *sl_dists, int32_t count, double radius, const double *weights,
                     bool unweighted, HaB200Plan **out) {
	*out = nullptr;
	int rc = validate_searchlights(sl_indices, sl_offsets, count, nv);
	if (rc != kHaSuccess) return rc;
	if (nt <= 0) return kHaErrorArg;
	if (sl_dists && !(radius > 0)) {
		fprintf(stderr, "ha_b200: radius must be positive with distance weighting\n");
		return kHaErrorArg;
	}
	if ((rc = set_smem_attrs()) != kHaSuccess) return rc;
	HaB200Plan *P = new (std::nothrow) HaB200Plan();
	if (!P) return kHaErrorAlloc;
	P->nt = nt;
	P->nv = nv;
	P->count = count;
	P->total = sl_offsets[count];
	P->h_off.assign(sl_offsets, sl_offsets + count + 1);
	P->h_idx.assign(sl_indices, sl_indices + P->total);
	P->h_w.resize((size_t)P->total);
	P->has_weights = !unweighted;
	if (weights)
		memcpy(P->h_w.data(), weights, (size_t)P->total * sizeof(double));
	else if (!unweighted)
		compute_weights(sl_indices, sl_offsets, sl_dists, count, radius, nv, P->h_w.data());
	for (int s = 0; s < count; s++) P->max_n = std::max(P->max_n, sl_offsets[s + 1] - sl_offsets[s]);
	if (rpl_for(P->max_n) < 0) {
		fprintf(stderr, "ha_b200: searchlight of %d vertices exceeds the supported maximum of %d\n", P->max_n,
		        32 * kRplSet[sizeof(kRplSet) / sizeof(kRplSet[0]) - 1]);
		delete P;
		return kHaErrorArg;
	}
	// per-vertex membership lists, sorted by searchlight (counting sort over flat order)
	std::vector<int64_t> vptr((size_t)nv + 1, 0);
	for (int64_t k = 0; k < P->total; k++) vptr[(size_t)sl_indices[k] + 1]++;
	for (int v = 0; v < nv; v++) vptr[v + 1] += vptr[v];
	std::vector<int2> vent((size_t)P->total);
	std::vector<int64_t> cur(vptr.begin(), vptr.end() - 1);
	std::vector<int32_t> slo((size_t)count), shi((size_t)count);
	for (int s = 0; s < count; s++) {
		int lo = nv, hi = -1;
		for (int32_t k = sl_offsets[s]; k < sl_offsets[s + 1]; k++) {
			int v = sl_indices[k];
			vent[(size_t)cur[v]++] = make_int2(s, k - sl_offsets[s]);
			lo = std::min(lo, v);
			hi = std::max(hi, v);
		}
		slo[s] = lo;
		shi[s] = hi;
	}
	auto fail = [&](int code) {
		ha_b200_plan_destroy(P);
		return code;
	};
	if ((rc = P->idx.ensure((size_t)P->total)) != kHaSuccess) return fail(rc);
	if ((rc = P->off.ensure((size_t)count + 1)) != kHaSuccess) return fail(rc);
	if ((rc = P->lo.ensure((size_t)count)) != kHaSuccess) return fail(rc);
	if ((rc = P->hi.ensure((size_t)count)) != kHaSuccess) return fail(rc);
	if ((rc = P->w.ensure((size_t)P->total)) != kHaSuccess) return fail(rc);
	if ((rc = P->vlptr.ensure((size_t)nv + 1)) != kHaSuccess) return fail(rc);
	if ((rc = P->vlent.ensure((size_t)P->total)) != kHaSuccess) return fail(rc);
	if (cudaMemcpy(P->idx.p, sl_indices, (size_t)P->total * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(P->off.p, sl_offsets, ((size_t)count + 1) * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(P->lo.p, slo.data(), (size_t)count * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(P->hi.p, shi.data(), (size_t)count * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(P->w.p, P->h_w.data(), (size_t)P->total * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(P->vlptr.p, vptr.data(), ((size_t)nv + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(P->vlent.p, vent.data(), (size_t)P->total * sizeof(int2), cudaMemcpyHostToDevice) != cudaSuccess) {
		fprintf(stderr, "ha_b200: upload of the searchlight geometry failed: %s\n", cudaGetErrorString(cudaGetLastError()));
		return fail(kHaErrorInternal);
	}
	if ((rc = build_pattern(P)) != kHaSuccess) return fail(rc);
	*out = P;
	return kHaSuccess;
}

// sigma_min / sigma_max below which the mixed solver re-solves a searchlight in float64
// (HA_B200_ILL_RATIO overrides the default).  Measured on the hemisphere template workload
// (10242 searchlights, float64 oracle): FP32 Jacobi + refinement stays within 1.4e-5
// relative Frobenius for every searchlight with ratio >= 3e-5 and fails some below it; 5e-5
// keeps a margin.
double ill_ratio() {
	static double r = -1.0;
	if (r < 0.0) {
		const char *e = getenv("HA_B200_ILL_RATIO");
		r = e ? atof(e) : 5e-5;
		if (!(r >= 0.0)) r = 5e-5;
	}
	return r;
}

// Early stop of the float32 solves: a sweep whose largest |cos| is at most this is the last
// (HA_B200_STOP_COS overrides the default 1e-2; 0 turns it off).  Measured in float32 on template
// searchlights: the sweep after one with |cos| <= 1e-2 only confirms convergence (its largest |cos|
// is ~1e-6), and stopping without it leaves the per-T error unchanged.
double fp32_stop_cos() {
	static double r = -1.0;
	if (r < 0.0) {
		const char *e = getenv("HA_B200_STOP_COS");
		r = e ? atof(e) : 1e-2;
		if (!(r >= 0.0)) r = 1e-2;
	}
	return r;
}

// The same for the float64 solves (HA_B200_STOP_COS64 overrides the default 1e-8): measured in
// float64, the sweep after one with |cos| <= 1e-6 changes T by less than 1e-14.
double fp64_stop_cos() {
	static double r = -1.0;
	if (r < 0.0) {
		const char *e = getenv("HA_B200_STOP_COS64");
		r = e ? atof(e) : 1e-8;
		if (!(r >= 0.0)) r = 1e-8;
	}
	return r;
}

// Weak-column factor of k_jacobi (HA_B200_WEAK_FACTOR overrides the default).
double weak_factor() {
	static double r = -1.0;
	if (r < 0.0) {
		const char *e = getenv("HA_B200_WEAK_FACTOR");
		r = e ? atof(e) : 1000.0;
		if (!(r >= 0.0)) r = 1000.0;
	}
	return r;
}

// ---- tensor-core Newton-Schulz solver ----

// Dynamic shared memory of the tile-product launches: np <= 256 runs two CTAs per SM (two
// 110 KB stage rings plus static and reserved shared memory within the SM's 228 KB, 2 x 256
// tensor-memory columns), np > 256 one CTA per SM.
constexpr int kTcSmemSmall = 110 * 1024;
constexpr int kTcSmemLarge = 200 * 1024;

double env_double(const char *name, double dflt, double lo, double hi) {
	const char *e = getenv(name);
	if (!e) return dflt;
	const double v = atof(e);
	return (v >= lo && v <= hi) ? v : dflt;
}

// Iteration schedule, shared by every searchlight.  X_0 = A / u has its singular values in
// [l0, 1] for a condition number up to 1/l0 (u overestimates sigma_max by a few units, which the
// bound absorbs).  l0 = 3e-5 and cap 1.65 minimise the mean iteration count on template
// searchlights (15.4, from the singular values of 400 of them; 17.1 with 1e-5 and 1.6) at the same
// accuracy (a three-part-split emulation on the ten worst conditioned: max 3.5e-7 vs float64).  Each step is the scaled cubic step of the lower bound l:
// a = sqrt(3 / (1 + l + l^2)), capped at `cap` (larger scalings map the largest singular values
// near zero and lose their precision), l <- a l (3 - a^2 l^2) / 2; once a < 1.02 the steps are the
// plain ones (a = 1) until the residual criterion ends each searchlight.  HA_B200_NS_L0,
// HA_B200_NS_CAP and HA_B200_NS_MAXIT override the defaults.
struct NsStep {
	float c1, c3;
	int plain;
};
std::vector<NsStep> ns_schedule() {
	const double l0 = env_double("HA_B200_NS_L0", 3e-5, 1e-12, 0.5);
	const double cap = env_double("HA_B200_NS_CAP", 1.65, 1.0, 1.7);
	const int maxit = (int)env_double("HA_B200_NS_MAXIT", 40, 4, 200);
	std::vector<NsStep> out;
	double l = l0;
	bool plain = false;
	for (int k = 0; k < maxit; k++) {
		double a = 1.0;
		if (!plain) {
			a = std::min(std::sqrt(3.0 / (1.0 + l + l * l)), cap);
			if (a < 1.02) {
				plain = true;
				a = 1.0;
			}
		}
		out.push_back({(float)(1.5 * a), (float)(-0.5 * a * a * a), plain ? 1 : 0});
		l = std::min(1.0, 0.5 * a * l * (3.0 - a * a * l * l));
	}
	return out;
}

// Residual ||G - I||_F / sqrt(n) below which a plain step is the last (HA_B200_NS_TOL).  The
// largest |1 - sigma^2| is then below 1e-4 sqrt(n); the final step squares it.
double ns_tol() { return env_double("HA_B200_NS_TOL", 1e-4, 1e-7, 1e-1); }

// One launch per phase and iteration (default), or the persistent solve (HA_B200_TC_PERSIST=1: one
// CTA runs whole searchlights, their planes stay in L2; measured 3% slower on the template pair).
bool tc_persistent() {
	static int v = -1;
	if (v < 0) {
		const char *e = getenv("HA_B200_TC_PERSIST");
		v = (e && e[0] == '1') ? 1 : 0;
	}
	return v == 1;
}

int g_num_sms = 148;

// CTAs per SM of the persistent solve for searchlights of np <= 256: two (110 KB of stages each)
// or one (200 KB, so deeper pipelines, and half the planes live in L2 at a time).
// HA_B200_TC_CTAS overrides the default.
int tc_small_ctas_per_sm() {
	static int v = 0;
	if (!v) {
		const char *e = getenv("HA_B200_TC_CTAS");
		v = (e && e[0] == '1') ? 1 : 2;
	}
	return v;
}

int set_tc_attrs() {
	static bool done = false;
	if (done) return kHaSuccess;
	HA_CUDA(cudaFuncSetAttribute(k_tc_gemm<kTcPhaseXcov>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemLarge));
	HA_CUDA(cudaFuncSetAttribute(k_tc_gemm<kTcPhaseGram>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemLarge));
	HA_CUDA(cudaFuncSetAttribute(k_tc_gemm<kTcPhaseUpdate>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemLarge));
	HA_CUDA(cudaFuncSetAttribute(k_tc_gemm<kTcPhaseGram, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemLarge));
	HA_CUDA(cudaFuncSetAttribute(k_tc_iter<kTcPhaseGram>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax));
	HA_CUDA(cudaFuncSetAttribute(k_tc_iter<kTcPhaseUpdate>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax));
	HA_CUDA(cudaFuncSetAttribute(k_tc_gemm<kTcPhaseUpdate, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemLarge));
	HA_CUDA(cudaFuncSetAttribute(k_tc_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmemLarge));
	done = true;
	return kHaSuccess;
}

// Work lists and buffers of the tensor-core solve (once per plan).
int build_tc(HaB200Plan *P) {
	if (P->tc_ready) return kHaSuccess;
	int rc;
	if ((rc = set_tc_attrs()) != kHaSuccess) return rc;
	int64_t maxX = 1, maxA = 1;
	for (auto &ch : P->chunks) {
		const int nsl = ch.s1 - ch.s0;
		ch.tcw.clear();
		int64_t xacc = 0, aacc = 0;
		for (int q = 0; q < nsl; q++) {
			const int s = ch.s0 + q;
			const int n = P->h_off[s + 1] - P->h_off[s];
			const int np = (n + 15) & ~15;
			if (np > kTcMaxNp) return kHaErrorArg;
			TcWork w = {};
			w.s = s;
			w.slot = q;
			w.n = n;
			w.np = np;
			w.sofs = P->h_off[s];
			w.xofs = xacc;
			w.pofs = xacc;
			w.aofs = aacc;
			w.tofs = ch.tofs[q];
			xacc += 2 * (int64_t)np * np;  // the iteration's two FP16 planes
			aacc += (int64_t)np * np;
			ch.tcw.push_back(w);
		}
		ch.tc_x_elems = xacc;
		ch.tc_a_elems = aacc;
		maxX = std::max(maxX, xacc);
		maxA = std::max(maxA, aacc);
		std::vector<int> order((size_t)nsl);
		for (int q = 0; q < nsl; q++) order[q] = q;
		std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return ch.tcw[x].n > ch.tcw[y].n; });
		for (int c = 0; c < 2; c++) {
			ch.tct[c].clear();
			ch.tco[c].clear();
		}
		for (int q : order) {
			const int np = ch.tcw[q].np;
			const int c = np > 256 ? 1 : 0;
			// per-phase launches: tiles of at most 256 columns (two halves when np > 256), in two
			// classes by column count (<= 128: 128 tensor-memory columns a CTA; 129-256)
			const int h0 = np > 256 ? ((np / 2 + 15) & ~15) : np;
			for (int t = 0; t * 128 < np; t++) {
				ch.tct[h0 <= 128 ? 0 : 1].push_back({q, t, 0, h0});
				if (h0 < np) ch.tct[np - h0 <= 128 ? 0 : 1].push_back({q, t, h0, np - h0});
			}
			ch.tco[c].push_back(q);
		}
		if (cudaMalloc(&ch.d_tcw, (size_t)nsl * sizeof(TcWork)) != cudaSuccess) return kHaErrorAlloc;
		HA_CUDA(cudaMemcpy(ch.d_tcw, ch.tcw.data(), (size_t)nsl * sizeof(TcWork), cudaMemcpyHostToDevice));
		for (int c = 0; c < 2; c++) {
			const size_t cnt = std::max<size_t>(ch.tct[c].size(), 1);
			if (cudaMalloc(&ch.d_tct[c], cnt * sizeof(TcTile)) != cudaSuccess) return kHaErrorAlloc;
			if (!ch.tct[c].empty())
				HA_CUDA(cudaMemcpy(ch.d_tct[c], ch.tct[c].data(), ch.tct[c].size() * sizeof(TcTile), cudaMemcpyHostToDevice));
			const size_t co = std::max<size_t>(ch.tco[c].size(), 1);
			if (cudaMalloc(&ch.d_tco[c], co * sizeof(int32_t)) != cudaSuccess) return kHaErrorAlloc;
			if (!ch.tco[c].empty())
				HA_CUDA(cudaMemcpy(ch.d_tco[c], ch.tco[c].data(), ch.tco[c].size() * sizeof(int32_t), cudaMemcpyHostToDevice));
		}
	}
	if ((rc = P->tcXp.ensure((size_t)maxX)) != kHaSuccess) return rc;
	if ((rc = P->tcXq.ensure((size_t)maxX)) != kHaSuccess) return rc;
	if ((rc = P->tcPp.ensure((size_t)maxX)) != kHaSuccess) return rc;
	if ((rc = P->tcA.ensure((size_t)maxA)) != kHaSuccess) return rc;
	if ((rc = P->tcRes.ensure((size_t)P->max_slots * kTcResSlots)) != kHaSuccess) return rc;
	if ((rc = P->tcSt.ensure((size_t)P->max_slots * 2)) != kHaSuccess) return rc;
	{
		const std::vector<NsStep> sched = ns_schedule();
		const size_t m = sched.size();
		std::vector<float> hc((size_t)2 * m);
		std::vector<int32_t> hp(m);
		for (size_t k = 0; k < m; k++) {
			hc[k] = sched[k].c1;
			hc[m + k] = sched[k].c3;
			hp[k] = sched[k].plain;
		}
		if ((rc = P->tcSched.ensure(2 * m)) != kHaSuccess) return rc;
		if ((rc = P->tcPlain.ensure(m)) != kHaSuccess) return rc;
		if ((rc = P->tcQueue.ensure(2)) != kHaSuccess) return rc;
		HA_CUDA(cudaMemcpy(P->tcSched.p, hc.data(), hc.size() * sizeof(float), cudaMemcpyHostToDevice));
		HA_CUDA(cudaMemcpy(P->tcPlain.p, hp.data(), hp.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
	}
	P->tc_ready = true;
	return kHaSuccess;
}

// Which of the iteration's products fill their stages with bulk copies from a producer warp
// rather than with per-thread loads: bit 0 the Gram, bit 1 the update (HA_B200_TC_BULK, default
// 1).  On the full template hemisphere the bulk Gram takes 1.32 ms a launch against 1.37, while the
// bulk update takes 1.80 against 1.37: its K-major A tile arrives as 16 strided 256-byte pieces
// per plane, which the copy engine streams from DRAM more slowly than 128 threads' loads.
int tc_bulk_mask() {
	static int v = -1;
	if (v < 0) {
		const char *e = getenv("HA_B200_TC_BULK");
		v = e ? (atoi(e) & 3) : 1;
	}
	return v;
}

// The first iteration whose products run in the persistent kernel (one CTA per SM walking the
// tiles; loads, products and epilogues overlapped across tiles); earlier iterations launch one CTA
// per tile.  While every searchlight is active the per-tile launches are faster (their tails
// overlap the next launch); once most have converged, a per-tile launch still starts every tile's
// CTA (about 0.25 ms for the template hemisphere's 24,054 tiles) where the persistent launch reads
// a short tile list (8-18 us).  Both compute identical bits.  HA_B200_TC_ITER_FROM overrides the
// default 16 (0: always persistent, also in the product self-test; 1000: never).
int tc_iter_from() {
	static int v = -1;
	if (v < 0) {
		const char *e = getenv("HA_B200_TC_ITER_FROM");
		v = e ? std::max(0, atoi(e)) : 16;
	}
	return v;
}

// One launch of the tile product of PHASE over `ntiles` tiles of at most `nmax` columns, by the
// persistent kernel when `persist`.
template <int PHASE>
void launch_tc_tiles(int ntiles, TcArgs a, cudaStream_t st, int nmax, bool persist) {
	if constexpr (PHASE != kTcPhaseXcov) {
		if (persist) {
			// stages for the tiles' widest B, then the CTA's tile list; enough CTAs that none holds
			// more than kTcIterMaxTiles tiles (beyond one per SM they run in later waves)
			const int stage = 2 * 4096 + 64 * nmax;
			const int list = kTcIterMaxTiles * (int)sizeof(TcIterTile);
			a.smem_bytes = std::min(kTcMaxStages, (int)(kSmemMax - list) / stage) * stage + list;
			const int grid = std::min(ntiles, std::max(g_num_sms, (ntiles + kTcIterMaxTiles - 1) / kTcIterMaxTiles));
			k_tc_iter<PHASE><<<grid, kTcIterThreads, a.smem_bytes, st>>>(a, ntiles, nmax);
			return;
		}
	}
	if (PHASE != kTcPhaseXcov && (tc_bulk_mask() >> (PHASE > 0 ? PHASE - 1 : 0) & 1))
		k_tc_gemm<PHASE, PHASE != kTcPhaseXcov><<<ntiles, kTcThreads, a.smem_bytes, st>>>(a);
	else
		k_tc_gemm<PHASE><<<ntiles, kTcThreads, a.smem_bytes, st>>>(a);
}

// Launch one phase of the tile product over the size classes of a chunk (only class `only` when
// it is 0 or 1), each with its layout's shared memory.
template <int PHASE>
int launch_tc(const Chunk &ch, TcArgs a, cudaStream_t st, int kind, const int *smem, int only = -1,
              bool persist = false) {
	for (int c = 0; c < 2; c++) {
		const int ntiles = (int)ch.tct[c].size();
		if (!ntiles || (only >= 0 && c != only)) continue;
		a.tiles = ch.d_tct[c];
		a.smem_bytes = smem[c];
		HA_LAUNCH(kind, st);
		launch_tc_tiles<PHASE>(ntiles, a, st, c ? 256 : 128, persist);
	}
	HA_CUDA(cudaGetLastError());
	return kHaSuccess;
}

// Layout candidates per size class (dynamic shared memory per CTA): tiles of <= 128 columns hold
// 128 tensor-memory columns, so two, three or four CTAs fit an SM (4, 3 or 2 pipeline stages);
// tiles of 129-256 columns run two CTAs per SM (110 KB, 3-4 stages) or one (200 KB, 5-7 stages).
const int kTcCand[2][3] = {{110 * 1024, 72 * 1024, 53 * 1024}, {110 * 1024, 200 * 1024, 0}};

// CUDA-graph replay of captured launch sequences (ha_b200_set_graphs; on by default,
// HA_B200_GRAPHS=0 turns it off).
int g_graphs = -1;
bool graphs_enabled() {
	if (g_graphs < 0) {
		const char *e = getenv("HA_B200_GRAPHS");
		g_graphs = (e && e[0] == '0') ? 0 : 1;
	}
	return g_graphs == 1;
}

// A private non-blocking stream for captures (the legacy default stream cannot be captured).
cudaStream_t capture_stream() {
	static cudaStream_t s = nullptr;
	if (!s && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
		cudaGetLastError();
		s = nullptr;
	}
	return s;
}

bool autotune_enabled() {
	static int v = -1;
	if (v < 0) {
		const char *e = getenv("HA_B200_AUTOTUNE");
		v = (e && e[0] == '0') ? 0 : 1;
	}
	return v == 1;
}

// Time one Gram launch of every candidate layout per size class on the chunk's current iterate
// (the launches only write P and the residual partials, which the iteration then recomputes) and
// keep the fastest.  Synchronises the stream once.
int autotune_tc(HaB200Plan *P, const Chunk &ch, TcArgs a, cudaStream_t st) {
	cudaEvent_t e0, e1;
	HA_CUDA(cudaEventCreate(&e0));
	HA_CUDA(cudaEventCreate(&e1));
	for (int c = 0; c < 2; c++) {
		if (ch.tct[c].empty()) continue;
		double best = 1e300;
		for (int i = 0; i < 3 && kTcCand[c][i]; i++) {
			int smem[2] = {P->tc_smem[0], P->tc_smem[1]};
			smem[c] = kTcCand[c][i];
			double tmin = 1e300;
			for (int rep = 0; rep < 2; rep++) {
				HA_CUDA(cudaEventRecord(e0, st));
				int rc = launch_tc<kTcPhaseGram>(ch, a, st, kHaB200KTcNs, smem, c);
				HA_CUDA(cudaEventRecord(e1, st));
				if (rc != kHaSuccess) return rc;
				HA_CUDA(cudaEventSynchronize(e1));
				float ms = 0.f;
				HA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
				tmin = std::min(tmin, (double)ms);
			}
			P->tc_tune_ms[c][i] = tmin;
			if (tmin < best) {
				best = tmin;
				P->tc_smem[c] = kTcCand[c][i];
			}
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	P->tc_tuned = true;
	return kHaSuccess;
}

// Enqueue one tensor-core solve + reduction over all chunks: split-BF16 cross-covariance,
// Newton-Schulz polar, float64 Jacobi re-solve of the searchlights whose iteration did not
// converge (exactly singular A), scaling, reduction.  Reflection is allowed (isReflection).
int run_procrustes_tc(HaB200Plan *P, const double *d_X, const double *d_Y, bool scal, int out_kind, double *d_vals,
                      cudaStream_t st) {
	const int nt = P->nt, nv = P->nv;
	const int ntp = (nt + 15) & ~15;
	const int rowmajor = out_kind == kHaB200OutCSR ? 1 : 0;
	int rc;
	if (P->chunks.empty() && (rc = build_chunks(P)) != kHaSuccess) return rc;
	if ((rc = build_tc(P)) != kHaSuccess) return rc;
	const int64_t vplane = (int64_t)nv * ntp;
	if ((rc = P->tcXb.ensure((size_t)(3 * vplane))) != kHaSuccess) return rc;
	if ((rc = P->tcYb.ensure((size_t)(3 * vplane))) != kHaSuccess) return rc;
	{ HA_LAUNCH(kHaB200KConvert, st); k_split3_vertex_major<<<148 * 8, kBlock, 0, st>>>(d_X, nt, nv, ntp, P->tcXb.p); }
	{ HA_LAUNCH(kHaB200KConvert, st); k_split3_vertex_major<<<148 * 8, kBlock, 0, st>>>(d_Y, nt, nv, ntp, P->tcYb.p); }
	if (scal) {
		if ((rc = P->var.ensure((size_t)nv)) != kHaSuccess) return rc;
		{ HA_LAUNCH(kHaB200KColVar, st); k_col_var_over_nt<<<(nv + 127) / 128, 128, 0, st>>>(d_X, nt, nv, P->var.p); }
	}
	HA_CUDA(cudaMemsetAsync(P->counters.p, 0, 5 * sizeof(int32_t), st));
	static const std::vector<NsStep> sched = ns_schedule();
	const int maxit = (int)sched.size();
	float *T = P->scrT.p;
	const int smem_cap = std::min(P->max_row, 16384);
	const size_t red_smem = (size_t)smem_cap * 12;
	for (size_t c = 0; c < P->chunks.size(); c++) {
		Chunk &ch = P->chunks[c];
		const int nsl = ch.s1 - ch.s0;
		HA_CUDA(cudaMemsetAsync(P->stats.p, 0, (size_t)nsl * sizeof(SlStats), st));
		TcArgs a = {};
		a.work = ch.d_tcw;
		a.Xb = P->tcXb.p;
		a.Yb = P->tcYb.p;
		a.vplane = vplane;
		a.ntp = ntp;
		a.sl_idx = P->idx.p;
		a.Xp = P->tcXp.p;
		a.Xw = P->tcXq.p;
		a.Pp = P->tcPp.p;
		a.A32 = P->tcA.p;
		a.T = T;
		a.t_rowmajor = rowmajor;
		a.res_part = P->tcRes.p;
		a.tol_stop = (float)ns_tol();
		a.err = P->counters.p + 4;
		if (tc_persistent()) {
			// one launch per size class; the larger searchlights first
			HA_CUDA(cudaMemsetAsync(P->tcQueue.p, 0, 2 * sizeof(int32_t), st));
			TcSolveArgs sa = {};
			sa.work = ch.d_tcw;
			sa.Xb = P->tcXb.p; sa.Yb = P->tcYb.p; sa.vplane = vplane; sa.ntp = ntp; sa.sl_idx = P->idx.p;
			sa.Xp = P->tcXp.p; sa.Pp = P->tcPp.p; sa.A32 = P->tcA.p; sa.T = T; sa.t_rowmajor = rowmajor;
			sa.c1 = P->tcSched.p; sa.c3 = P->tcSched.p + maxit; sa.plain = P->tcPlain.p; sa.maxit = maxit;
			sa.tol_stop = (float)ns_tol(); sa.stats = P->stats.p; sa.err = P->counters.p + 4;
			for (int c = 1; c >= 0; c--) {
				const int cnt = (int)ch.tco[c].size();
				if (!cnt) continue;
				sa.order = ch.d_tco[c];
				sa.count = cnt;
				sa.queue = P->tcQueue.p + c;
				const int per_sm = c ? 1 : tc_small_ctas_per_sm();
				sa.smem_bytes = per_sm == 2 ? kTcSmemSmall : kTcSmemLarge;
				const int grid = std::min(cnt, g_num_sms * per_sm);
				HA_LAUNCH(kHaB200KTcNs, st);
				k_tc_solve<<<grid, kTcThreads, sa.smem_bytes, st>>>(sa);
			}
			HA_CUDA(cudaGetLastError());
		} else {
		if ((rc = launch_tc<kTcPhaseXcov>(ch, a, st, kHaB200KTcXcov, P->tc_smem)) != kHaSuccess) return rc;
		{ HA_LAUNCH(kHaB200KTcNs, st); k_tc_ns_init<<<nsl, 256, 0, st>>>(ch.d_tcw, P->tcA.p, P->tcXp.p, P->tcSt.p, P->tcRes.p); }
		if (!P->tc_tuned && autotune_enabled()) {
			a.st_in = P->tcSt.p;
			a.c1 = sched[0].c1;
			a.c3 = sched[0].c3;
			if ((rc = autotune_tc(P, ch, a, st)) != kHaSuccess) return rc;
		}
		// the iteration: 2 x maxit launches per size class, the same every call on this plan, so
		// captured once into a CUDA graph (on a private stream) and replayed on the caller's stream
		auto enqueue_loop = [&](cudaStream_t ls) -> int {
			for (int k = 0; k < maxit; k++) {
				a.st_in = P->tcSt.p + (size_t)(k & 1) * P->max_slots;
				a.st_out = P->tcSt.p + (size_t)((k + 1) & 1) * P->max_slots;
				a.Xp = (k & 1) ? P->tcXq.p : P->tcXp.p;
				a.Xw = (k & 1) ? P->tcXp.p : P->tcXq.p;
				a.c1 = sched[k].c1;
				a.c3 = sched[k].c3;
				a.plain = sched[k].plain;
				a.last = (k == maxit - 1) ? 1 : 0;
				const bool persist = k >= tc_iter_from();
				int r = launch_tc<kTcPhaseGram>(ch, a, ls, kHaB200KTcNs, P->tc_smem, -1, persist);
				if (r != kHaSuccess) return r;
				if ((r = launch_tc<kTcPhaseUpdate>(ch, a, ls, kHaB200KTcNs, P->tc_smem, -1, persist)) != kHaSuccess)
					return r;
			}
			return kHaSuccess;
		};
		if (!graphs_enabled() || g_timing) {
			if ((rc = enqueue_loop(st)) != kHaSuccess) return rc;
		} else {
			const int key[3] = {rowmajor, P->tc_smem[0], P->tc_smem[1]};
			if (!ch.tc_graph || memcmp(key, ch.tc_graph_key, sizeof(key)) != 0) {
				if (ch.tc_graph) cudaGraphExecDestroy(ch.tc_graph);
				ch.tc_graph = nullptr;
				cudaStream_t cs = capture_stream();
				if (!cs) return kHaErrorInternal;
				const int64_t l0 = g_launches, n0 = g_kernel_n[kHaB200KTcNs];
				HA_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
				rc = enqueue_loop(cs);
				cudaGraph_t gr = nullptr;
				const cudaError_t ce = cudaStreamEndCapture(cs, &gr);
				g_launches = l0;  // counted when the graph runs
				g_kernel_n[kHaB200KTcNs] = n0;
				if (rc != kHaSuccess || ce != cudaSuccess) {
					if (gr) cudaGraphDestroy(gr);
					fprintf(stderr, "ha_b200: capture of the tensor-core iteration failed: %s\n", cudaGetErrorString(ce));
					return rc != kHaSuccess ? rc : kHaErrorInternal;
				}
				const cudaError_t ie = cudaGraphInstantiate(&ch.tc_graph, gr, 0);
				size_t nodes = 0;
				cudaGraphGetNodes(gr, nullptr, &nodes);
				cudaGraphDestroy(gr);
				if (ie != cudaSuccess) {
					ch.tc_graph = nullptr;
					fprintf(stderr, "ha_b200: instantiating the tensor-core iteration graph failed: %s\n", cudaGetErrorString(ie));
					return kHaErrorInternal;
				}
				ch.tc_graph_kernels = (int)nodes;
				memcpy(ch.tc_graph_key, key, sizeof(key));
			}
			HA_CUDA(cudaGraphLaunch(ch.tc_graph, st));
			g_launches += ch.tc_graph_kernels;
			g_kernel_n[kHaB200KTcNs] += ch.tc_graph_kernels;
		}
		{ HA_LAUNCH(kHaB200KTcNs, st); k_tc_ns_finish<<<nsl, 256, 0, st>>>(ch.d_tcw, P->tcA.p, T, P->tcSt.p + (size_t)(maxit & 1) * P->max_slots,
		                                                              P->stats.p, rowmajor); }
		}
		{ HA_LAUNCH(kHaB200KTcNs, st); k_tc_complete<<<nsl, 256, 0, st>>>(ch.d_tcw, T, P->tcXp.p, P->tcPp.p, P->stats.p, rowmajor); }
		// float64 Jacobi re-solve of the searchlights still flagged (cold start)
		{
			JacobiParams jp;
			jp.max_sweeps = 40;
			jp.t_rowmajor = rowmajor;
			jp.ill_ratio = 0.0;
			jp.weak = weak_factor();
			jp.eig = 0;
			jp.keep_v = 0;
			jp.warm = 0;
			jp.only_flagged = 1;
			jp.stop_cos = fp64_stop_cos();
			double *A = P->scrA.p, *V = P->scrV.p;
			if ((rc = g_fan.begin(st)) != kHaSuccess) return rc;
			for (size_t bi = 0; bi < ch.b64.size(); bi++) {
				const Bucket &b = ch.b64[bi];
				const cudaStream_t bs = g_fan.at((int)bi);
				const SlWork *wk = ch.d_w64 + b.first;
				{ HA_LAUNCH(kHaB200KXcov64, bs); k_xcov<double, 16><<<b.count, kBlock, 0, bs>>>(wk, P->idx.p, d_X, d_Y, nt, nt, A, P->stats.p, 1); }
				{
					HA_LAUNCH(kHaB200KJacobi64, bs);
					if ((rc = launch_jacobi<double>(b.rpl, b.count, b.threads, b.smem, bs, wk, A, V, T, P->stats.p, P->uv.p, jp)) != kHaSuccess)
						return rc;
				}
				if (b.blocked) { HA_LAUNCH(kHaB200KFormT64, bs); k_form_t_global<double><<<b.count, kBlock, 0, bs>>>(wk, A, V, T, P->stats.p, rowmajor, 1); }
			}
			if ((rc = g_fan.end(st)) != kHaSuccess) return rc;
		}
		{ HA_LAUNCH(kHaB200KScale, st); k_scale<<<(nsl + 127) / 128, 128, 0, st>>>(ch.d_w64, nsl, P->idx.p, P->var.p, P->stats.p, nt, scal ? 1 : 0,
		                                          P->scale.p); }
		{ HA_LAUNCH(kHaB200KScale, st); k_count_flags<<<(nsl + 127) / 128, 128, 0, st>>>(P->stats.p, nsl, P->counters.p); }
		{ HA_LAUNCH(kHaB200KReduce, st); k_reduce<float><<<nv, kBlock, red_smem, st>>>(P->vlptr.p, P->vlent.p, P->off.p, P->idx.p,
		                                       P->has_weights ? P->w.p : nullptr, P->patptr.p, P->patcol.p, T,
		                                       ch.d_tofs, P->scale.p, ch.s0, ch.s1, out_kind == kHaB200OutCSC ? 1 : 0,
		                                       smem_cap, d_vals); }
		HA_CUDA(cudaGetLastError());
	}
	P->last_chunk = (int)P->chunks.size() - 1;
	P->last_rowmajor = rowmajor;
	return kHaSuccess;
}

// Enqueue one solve + reduction over all chunks.
int run_procrustes(HaB200Plan *P, const double *d_X, const double *d_Y, bool refl, bool scal, int solver,
                   int out_kind, double *d_vals, cudaStream_t st) {
	if (solver == kHaB200SolverTC) {
		// The reflection fix needs the smallest singular pair, which the polar iteration does not
		// produce: without reflection the mixed Jacobi solver runs instead.
		if (refl) return run_procrustes_tc(P, d_X, d_Y, scal, out_kind, d_vals, st);
		solver = kHaB200SolverMixed;
	}
	const int nt = P->nt, nv = P->nv;
	const int ntp = (nt + 31) & ~31;
	const bool use32 = solver != kHaB200SolverFP64;
	const int rowmajor = out_kind == kHaB200OutCSR ? 1 : 0;
	int rc;
	if (P->chunks.empty() && (rc = build_chunks(P)) != kHaSuccess) return rc;
	if (solver == kHaB200SolverMixed) {  // float64 temporaries of the re-solve's warm start
		int64_t maxT = 1;
		for (auto &ch : P->chunks) maxT = std::max(maxT, ch.t_elems);
		if ((rc = P->scrT64.ensure((size_t)maxT)) != kHaSuccess) return rc;
	}
	if (use32) {
		if ((rc = P->X32.ensure((size_t)nv * ntp)) != kHaSuccess) return rc;
		if ((rc = P->Y32.ensure((size_t)nv * ntp)) != kHaSuccess) return rc;
		int grid = 148 * 8;
		{ HA_LAUNCH(kHaB200KConvert, st); k_to_f32_vertex_major<<<grid, kBlock, 0, st>>>(d_X, nt, nv, ntp, P->X32.p); }
		{ HA_LAUNCH(kHaB200KConvert, st); k_to_f32_vertex_major<<<grid, kBlock, 0, st>>>(d_Y, nt, nv, ntp, P->Y32.p); }
	}
	if (scal) {
		if ((rc = P->var.ensure((size_t)nv)) != kHaSuccess) return rc;
		{ HA_LAUNCH(kHaB200KColVar, st); k_col_var_over_nt<<<(nv + 127) / 128, 128, 0, st>>>(d_X, nt, nv, P->var.p); }
	}
	HA_CUDA(cudaMemsetAsync(P->counters.p, 0, 5 * sizeof(int32_t), st));
	float *T = P->scrT.p;
	int smem_cap = std::min(P->max_row, 16384);
	size_t red_smem = (size_t)smem_cap * 12;
	for (size_t c = 0; c < P->chunks.size(); c++) {
		Chunk &ch = P->chunks[c];
		const int nsl = ch.s1 - ch.s0;
		HA_CUDA(cudaMemsetAsync(P->stats.p, 0, (size_t)nsl * sizeof(SlStats), st));
		JacobiParams jp;
		jp.max_sweeps = 40;
		jp.t_rowmajor = rowmajor;
		jp.ill_ratio = (solver == kHaB200SolverMixed) ? ill_ratio() : 0.0;
		jp.weak = weak_factor();
		jp.eig = 0;
		jp.keep_v = (solver == kHaB200SolverMixed) ? 1 : 0;
		jp.warm = 0;
		jp.stop_cos = fp32_stop_cos();
		if (use32) {
			float *A = reinterpret_cast<float *>(P->scrA.p);
			float *V = reinterpret_cast<float *>(P->scrV.p);
			jp.only_flagged = 0;
			if ((rc = g_fan.begin(st)) != kHaSuccess) return rc;
			for (size_t bi = 0; bi < ch.b32.size(); bi++) {
				const Bucket &b = ch.b32[bi];
				const cudaStream_t bs = g_fan.at((int)bi);
				const SlWork *wk = ch.d_w32 + b.first;
				{ HA_LAUNCH(kHaB200KXcov32, bs); k_xcov<float, 32><<<b.count, kBlock, 0, bs>>>(wk, P->idx.p, P->X32.p, P->Y32.p, ntp, nt, A, P->stats.p, 0); }
				{
					HA_LAUNCH(kHaB200KJacobi32, bs);
					if ((rc = launch_jacobi<float>(b.rpl, b.count, b.threads, b.smem, bs, wk, A, V, T, P->stats.p, P->uv.p, jp)) != kHaSuccess)
						return rc;
				}
				if (b.blocked) { HA_LAUNCH(kHaB200KFormT32, bs); k_form_t_global<float><<<b.count, kBlock, 0, bs>>>(wk, A, V, T, P->stats.p, rowmajor, 0); }
			}
			if ((rc = g_fan.end(st)) != kHaSuccess) return rc;
		}
		if (solver != kHaB200SolverFP32) {
			double *A = P->scrA.p, *V = P->scrV.p;
			const int only = (solver == kHaB200SolverMixed) ? 1 : 0;
			jp.only_flagged = only;
			jp.keep_v = 0;
			jp.warm = only;  // the mixed solver's re-solve starts from the float32 rotations
			jp.stop_cos = fp64_stop_cos();
			if ((rc = g_fan.begin(st)) != kHaSuccess) return rc;
			for (size_t bi = 0; bi < ch.b64.size(); bi++) {
				const Bucket &b = ch.b64[bi];
				const cudaStream_t bs = g_fan.at((int)bi);
				const SlWork *wk = ch.d_w64 + b.first;
				if (only) { HA_LAUNCH(kHaB200KRefine, bs); k_warm_v<<<b.count, kBlock, 0, bs>>>(wk, A, V, P->scrT64.p, P->stats.p); }
				{ HA_LAUNCH(kHaB200KXcov64, bs); k_xcov<double, 16><<<b.count, kBlock, 0, bs>>>(wk, P->idx.p, d_X, d_Y, nt, nt, A, P->stats.p, only); }
				if (only) { HA_LAUNCH(kHaB200KRefine, bs); k_warm_av<<<b.count, kBlock, 0, bs>>>(wk, A, V, P->scrT64.p, P->stats.p); }
				{
					HA_LAUNCH(kHaB200KJacobi64, bs);
					if ((rc = launch_jacobi<double>(b.rpl, b.count, b.threads, b.smem, bs, wk, A, V, T, P->stats.p, P->uv.p, jp)) != kHaSuccess)
						return rc;
				}
				if (b.blocked) { HA_LAUNCH(kHaB200KFormT64, bs); k_form_t_global<double><<<b.count, kBlock, 0, bs>>>(wk, A, V, T, P->stats.p, rowmajor, only); }
			}
			if ((rc = g_fan.end(st)) != kHaSuccess) return rc;
		}
		if (solver == kHaB200SolverMixed) {
			{ HA_LAUNCH(kHaB200KRefine, st); k_ns_refine<<<nsl, kBlock, 0, st>>>(ch.d_w32, T, reinterpret_cast<float *>(P->scrV.p),
			                                    reinterpret_cast<float *>(P->scrA.p), P->stats.p, rowmajor); }
		}
		if (!refl) { HA_LAUNCH(kHaB200KReflect, st); k_reflect_fix<<<nsl, kBlock, 0, st>>>(ch.d_w64, T, P->scrA.p, P->stats.p, P->uv.p, rowmajor); }
		{ HA_LAUNCH(kHaB200KScale, st); k_scale<<<(nsl + 127) / 128, 128, 0, st>>>(ch.d_w64, nsl, P->idx.p, P->var.p, P->stats.p, nt, scal ? 1 : 0,
		                                          P->scale.p); }
		{ HA_LAUNCH(kHaB200KScale, st); k_count_flags<<<(nsl + 127) / 128, 128, 0, st>>>(P->stats.p, nsl, P->counters.p); }
		{ HA_LAUNCH(kHaB200KReduce, st); k_reduce<float><<<nv, kBlock, red_smem, st>>>(P->vlptr.p, P->vlent.p, P->off.p, P->idx.p,
		                                       P->has_weights ? P->w.p : nullptr, P->patptr.p, P->patcol.p, T,
		                                       ch.d_tofs, P->scale.p, ch.s0, ch.s1, out_kind == kHaB200OutCSC ? 1 : 0,
		                                       smem_cap, d_vals); }
		HA_CUDA(cudaGetLastError());
	}
	P->last_chunk = (int)P->chunks.size() - 1;
	P->last_rowmajor = rowmajor;
	return kHaSuccess;
}

// Enqueue the searchlight ridge solve + reduction over all chunks (float64 throughout).
int run_ridge(HaB200Plan *P, const double *d_X, const double *d_Y, double alpha, int out_kind, double *d_vals,
              cudaStream_t st) {
	const int nt = P->nt, nv = P->nv;
	const int rowmajor = out_kind == kHaB200OutCSR ? 1 : 0;
	int rc;
	if (P->chunks.empty() && (rc = build_chunks(P)) != kHaSuccess) return rc;
	int64_t maxT = 1;
	for (auto &ch : P->chunks) maxT = std::max(maxT, ch.t_elems);
	if ((rc = P->scrT64.ensure((size_t)maxT)) != kHaSuccess) return rc;
	HA_CUDA(cudaMemsetAsync(P->counters.p, 0, 5 * sizeof(int32_t), st));
	const int smem_cap = std::min(P->max_row, 16384);
	const size_t red_smem = (size_t)smem_cap * 12;
	for (size_t c = 0; c < P->chunks.size(); c++) {
		Chunk &ch = P->chunks[c];
		const int nsl = ch.s1 - ch.s0;
		HA_CUDA(cudaMemsetAsync(P->stats.p, 0, (size_t)nsl * sizeof(SlStats), st));
		double *G = P->scrA.p, *R = P->scrV.p;
		if ((rc = g_fan.begin(st)) != kHaSuccess) return rc;
		for (size_t bi = 0; bi < ch.b64.size(); bi++) {
			const Bucket &b = ch.b64[bi];
			const cudaStream_t bs = g_fan.at((int)bi);
			const SlWork *wk = ch.d_w64 + b.first;
			{ HA_LAUNCH(kHaB200KXcov64, bs); k_xcov<double, 16><<<b.count, kBlock, 0, bs>>>(wk, P->idx.p, d_X, d_X, nt, nt, G, P->stats.p, 0); }
			{ HA_LAUNCH(kHaB200KXcov64, bs); k_xcov<double, 16><<<b.count, kBlock, 0, bs>>>(wk, P->idx.p, d_X, d_Y, nt, nt, R, P->stats.p, 0); }
			{ HA_LAUNCH(kHaB200KRidge, bs); k_ridge_chol<<<b.count, kBlock, 0, bs>>>(wk, G, R, P->scrT64.p, alpha, rowmajor, P->stats.p); }
		}
		if ((rc = g_fan.end(st)) != kHaSuccess) return rc;
		{ HA_LAUNCH(kHaB200KScale, st); k_scale<<<(nsl + 127) / 128, 128, 0, st>>>(ch.d_w64, nsl, P->idx.p, nullptr, P->stats.p, nt, 0, P->scale.p); }
		{ HA_LAUNCH(kHaB200KScale, st); k_count_flags<<<(nsl + 127) / 128, 128, 0, st>>>(P->stats.p, nsl, P->counters.p); }
		{ HA_LAUNCH(kHaB200KReduce, st); k_reduce<double><<<nv, kBlock, red_smem, st>>>(P->vlptr.p, P->vlent.p, P->off.p, P->idx.p,
		                                       P->has_weights ? P->w.p : nullptr, P->patptr.p, P->patcol.p, P->scrT64.p,
		                                       ch.d_tofs, P->scale.p, ch.s0, ch.s1, out_kind == kHaB200OutCSC ? 1 : 0,
		                                       smem_cap, d_vals); }
		HA_CUDA(cudaGetLastError());
	}
	P->last_chunk = (int)P->chunks.size() - 1;
	P->last_rowmajor = rowmajor;
	return kHaSuccess;
}

// ---- ridge grid search with cross-validated ensembles ----

// Host description of the grid and the CV models (validated), in the layout the grid kernels use.
struct GridSpec {
	std::vector<double> alphas;
	std::vector<int32_t> npcs;
	std::vector<GridModel> mdl;
	std::vector<int32_t> rows, tpos, urows, untested;
	std::vector<double> winv;
	int mte = 1, ntu = 0;
};

int grid_spec(int nt, const double *alphas, int n_alphas, const int32_t *npcs, int n_npcs,
              const int32_t *const *train_li, const int32_t *const *test_li, const int32_t *train_sizes,
              const int32_t *test_sizes, int n_models, GridSpec &gs) {
	if (!alphas || !npcs || !train_li || !test_li || !train_sizes || !test_sizes || n_alphas < 1 || n_npcs < 1 ||
	    n_models < 1)
		return kHaErrorArg;
	for (int a = 0; a < n_alphas; a++)
		if (!std::isfinite(alphas[a])) return kHaErrorArg;
	for (int p = 0; p < n_npcs; p++)
		if (npcs[p] < 0) {
			fprintf(stderr, "ha_b200 ridge grid: negative PC count %d\n", npcs[p]);
			return kHaErrorArg;
		}
	gs.alphas.assign(alphas, alphas + n_alphas);
	gs.npcs.assign(npcs, npcs + n_npcs);
	std::vector<int32_t> count((size_t)nt, 0);
	for (int m = 0; m < n_models; m++) {
		const int tr = train_sizes[m], te = test_sizes[m];
		if (tr < 1 || te < 0 || !train_li[m] || (te > 0 && !test_li[m])) return kHaErrorArg;
		for (int i = 0; i < tr; i++)
			if (train_li[m][i] < 0 || train_li[m][i] >= nt) return kHaErrorArg;
		for (int i = 0; i < te; i++) {
			const int t = test_li[m] ? test_li[m][i] : -1;
			if (t < 0 || t >= nt) return kHaErrorArg;
		}
	}
	std::vector<int32_t> seen((size_t)nt, -1);
	for (int m = 0; m < n_models; m++) {
		for (int i = 0; i < test_sizes[m]; i++) {
			const int t = test_li[m][i];
			if (seen[t] == m) {
				fprintf(stderr, "ha_b200 ridge grid: row %d repeats in the test list of model %d\n", t, m);
				return kHaErrorArg;
			}
			seen[t] = m;
			count[t]++;
		}
	}
	std::vector<int32_t> upos((size_t)nt, -1);
	gs.urows.clear();
	gs.untested.clear();
	gs.winv.clear();
	for (int t = 0; t < nt; t++) {
		if (count[t] > 0) {
			upos[t] = (int32_t)gs.urows.size();
			gs.urows.push_back(t);
			gs.winv.push_back(1.0 / count[t]);
		} else {
			gs.untested.push_back(t);
		}
	}
	gs.ntu = (int)gs.urows.size();
	gs.mdl.resize(n_models);
	gs.rows.clear();
	gs.tpos.clear();
	gs.mte = 1;
	for (int m = 0; m < n_models; m++) {
		GridModel md;
		md.tr_ofs = (int32_t)gs.rows.size();
		md.tr_n = train_sizes[m];
		gs.rows.insert(gs.rows.end(), train_li[m], train_li[m] + train_sizes[m]);
		gs.tpos.resize(gs.rows.size(), -1);
		md.te_ofs = (int32_t)gs.rows.size();
		md.te_n = test_sizes[m];
		for (int i = 0; i < test_sizes[m]; i++) {
			gs.rows.push_back(test_li[m][i]);
			gs.tpos.push_back(upos[test_li[m][i]]);
		}
		gs.mte = std::max(gs.mte, md.te_n);
		gs.mdl[m] = md;
	}
	return kHaSuccess;
}

template <typename T>
int upload_vec(DevArr<T> &d, const std::vector<T> &h, cudaStream_t st) {
	int rc = d.ensure(std::max<size_t>(h.size(), 1));
	if (rc != kHaSuccess) return rc;
	if (!h.empty()) HA_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
	return kHaSuccess;
}

// Grid scratch budget per sub-batch of searchlights (HA_B200_GRID_GB overrides the default 24 GB).
size_t grid_budget_bytes() {
	const char *e = getenv("HA_B200_GRID_GB");
	double gb = e ? atof(e) : 24.0;
	if (!(gb > 0.001)) gb = 24.0;
	return (size_t)(gb * 1073741824.0);
}

// ---- learned (alpha, PC count) proposal: perceptron training and inference ----

size_t mlp_smem(int C) {
	return ((size_t)kMlpSamples * kMlpIn + 4 * (size_t)kMlpSamples * kMlpHidden + (size_t)kMlpSamples * C) * 4;
}

int mlp_check(int C) {
	if (C < 1 || C > kMlpMaxClasses) {
		fprintf(stderr, "ha_b200 mlp: %d classes outside 1..%d\n", C, kMlpMaxClasses);
		return kHaErrorArg;
	}
	static bool attr = false;
	if (!attr) {
		const int m = (int)mlp_smem(kMlpMaxClasses);
		HA_CUDA(cudaFuncSetAttribute(k_mlp_fwdbwd, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
		HA_CUDA(cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
		attr = true;
	}
	return kHaSuccess;
}

int mlp_labels_ok(const int32_t *d_y, int n, int C) {
	std::vector<int32_t> h((size_t)n);
	HA_CUDA(cudaMemcpy(h.data(), d_y, (size_t)n * 4, cudaMemcpyDeviceToHost));
	for (int i = 0; i < n; i++)
		if (h[i] < 0 || h[i] >= C) {
			fprintf(stderr, "ha_b200 mlp: label %d of sample %d outside 0..%d\n", h[i], i, C - 1);
			return kHaErrorArg;
		}
	return kHaSuccess;
}

// SplitMix64 stream for the host-side initialisation and shuffles.
struct HostRng {
	uint64_t x;
	explicit HostRng(uint64_t s) : x(s) {}
	uint64_t next() {
		uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
		z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
		z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
		return z ^ (z >> 31);
	}
	double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct MlpBufs {
	DevArr<float> part, loss, m, v;
	DevArr<int32_t> idx;
	DevArr<__nv_bfloat16> pbf;
	void release() { part.release(); loss.release(); m.release(); v.release(); idx.release(); pbf.release(); }
} g_mlp;

// Upload the grid / CV description and fill the kernel parameters (active: none).
int grid_upload(HaB200Plan *P, const GridSpec &gs, cudaStream_t st, GridParams &gp) {
	int rc;
	if ((rc = upload_vec(P->galpha, gs.alphas, st)) != kHaSuccess) return rc;
	if ((rc = upload_vec(P->gnpcs, gs.npcs, st)) != kHaSuccess) return rc;
	if ((rc = upload_vec(P->gmdl, gs.mdl, st)) != kHaSuccess) return rc;
	if ((rc = upload_vec(P->grows, gs.rows, st)) != kHaSuccess) return rc;
	if ((rc = upload_vec(P->gtpos, gs.tpos, st)) != kHaSuccess) return rc;
	if ((rc = upload_vec(P->gwinv, gs.winv, st)) != kHaSuccess) return rc;
	if ((rc = upload_vec(P->gurows, gs.urows, st)) != kHaSuccess) return rc;
	if ((rc = upload_vec(P->guntested, gs.untested, st)) != kHaSuccess) return rc;
	if ((rc = P->gbase.ensure((size_t)P->max_slots)) != kHaSuccess) return rc;
	gp.models = (int)gs.mdl.size();
	gp.mte = gs.mte;
	gp.ntu = gs.ntu;
	gp.n_alphas = (int)gs.alphas.size();
	gp.n_npcs = (int)gs.npcs.size();
	gp.nt = P->nt;
	gp.n_untested = (int)gs.untested.size();
	gp.alphas = P->galpha.p;
	gp.npcs = P->gnpcs.p;
	gp.mdl = P->gmdl.p;
	gp.rows = P->grows.p;
	gp.tpos = P->gtpos.p;
	gp.winv = P->gwinv.p;
	gp.urows = P->gurows.p;
	gp.untested = P->guntested.p;
	gp.gbase = P->gbase.p;
	return kHaSuccess;
}

int grid_prepare(HaB200Plan *P) {
	if (P->max_n > kGridMaxN) {
		fprintf(stderr, "ha_b200 ridge grid: searchlight of %d vertices exceeds the grid limit of %d\n", P->max_n,
		        kGridMaxN);
		return kHaErrorArg;
	}
	int rc;
	if (P->chunks.empty() && (rc = build_chunks(P)) != kHaSuccess) return rc;
	int64_t maxT = 1;
	for (auto &ch : P->chunks) maxT = std::max(maxT, ch.t_elems);
	return P->scrT64.ensure((size_t)maxT);
}

size_t pchol_smem(int rpl, size_t esz = sizeof(double)) { return (size_t)kPcholNb * 32 * rpl * esz; }

JacobiParams eig_params(bool only_flagged) {
	JacobiParams jp;
	jp.max_sweeps = 40;
	jp.t_rowmajor = 0;
	jp.ill_ratio = 0.0;
	jp.weak = weak_factor();
	jp.eig = 1;
	jp.only_flagged = only_flagged ? 1 : 0;
	jp.keep_v = 0;
	jp.warm = 0;
	jp.stop_cos = fp64_stop_cos();
	return jp;
}

// Scale (1), flag counts and the deterministic reduction of one chunk's float64 betas.
int reduce_chunk64(HaB200Plan *P, Chunk &ch, int out_kind, double *d_vals, cudaStream_t st) {
	const int nsl = ch.s1 - ch.s0;
	const int smem_cap = std::min(P->max_row, 16384);
	const size_t red_smem = (size_t)smem_cap * 12;
	{ HA_LAUNCH(kHaB200KScale, st); k_scale<<<(nsl + 127) / 128, 128, 0, st>>>(ch.d_w64, nsl, P->idx.p, nullptr, P->stats.p, P->nt, 0, P->scale.p); }
	{ HA_LAUNCH(kHaB200KScale, st); k_count_flags<<<(nsl + 127) / 128, 128, 0, st>>>(P->stats.p, nsl, P->counters.p); }
	{ HA_LAUNCH(kHaB200KReduce, st); k_reduce<double><<<P->nv, kBlock, red_smem, st>>>(P->vlptr.p, P->vlent.p, P->off.p, P->idx.p,
	                                       P->has_weights ? P->w.p : nullptr, P->patptr.p, P->patcol.p, P->scrT64.p,
	                                       ch.d_tofs, P->scale.p, ch.s0, ch.s1, out_kind == kHaB200OutCSC ? 1 : 0,
	                                       smem_cap, d_vals); }
	HA_CUDA(cudaGetLastError());
	return kHaSuccess;
}

// The grid search of one chunk: per sub-batch of searchlights (bounded by the grid scratch budget)
// and CV model, the Gram and cross-covariance over the model's training rows, the pivoted Cholesky
// factor and its float64 Jacobi eigen decomposition, and the per-model products; then the grid
// evaluation, the winners (d_best) and their betas in the float64 T scratch.  The chunk's work list
// may be a subset of the plan chunk's (the learned form's fallback searchlights).
// Sub-batches of a chunk's grid search: searchlights [i0, i1) of the eigenvector-mode work list,
// as many as fit the grid scratch budget, and each one's per-slot scratch base offsets.
struct GridBatch {
	int i0, i1;
	int64_t total;  // elements of grid scratch (float64 or float32, by the search's arithmetic)
};

void grid_plan_chunk(const Chunk &ch, const GridParams &gp, bool fp32, std::vector<GridBatch> &bt,
                     std::vector<int64_t> &gbase_all) {
	const int nsl = ch.s1 - ch.s0;
	const int grid = gp.n_alphas * gp.n_npcs;
	const size_t budget = grid_budget_bytes();
	const std::vector<SlWork> &items = fp32 ? ch.weig32 : ch.weig;
	const size_t esz = fp32 ? 4 : 8;
	const int nitems = (int)items.size();
	bt.clear();
	int i0 = 0;
	while (i0 < nitems) {
		const size_t g0 = gbase_all.size();
		gbase_all.resize(g0 + (size_t)nsl, 0);
		int64_t total = 0;
		int i1 = i0;
		while (i1 < nitems) {
			const SlWork &wi = items[i1];
			const GridLayout Lg = GridLayout::make(wi.n, gp.models, gp.mte, gp.ntu, gp.n_alphas, grid);
			if (i1 > i0 && (size_t)(total + Lg.total) * esz > budget) break;
			gbase_all[g0 + wi.slot] = total;
			total += Lg.total;
			i1++;
		}
		bt.push_back({i0, i1, total});
		i0 = i1;
	}
}

// The launches of one chunk's grid search (no host copies or allocations: capturable); the
// sub-batches' base offsets are at d_gbase (nsl per sub-batch).  Real is the arithmetic type:
// double for the float64 grid search, float for the plain FP32 one (the float32 eigenvector-mode
// work list, the A / V / grid scratch read as float; the winners' betas still go to the float64
// T scratch for the reduction).
template <typename Real>
int grid_chunk_launch_t(HaB200Plan *P, Chunk &ch, const double *d_X, const double *d_Y, const GridSpec &gs,
                        GridParams gp, const std::vector<GridBatch> &bt, const int64_t *d_gbase, int rowmajor,
                        int32_t *d_best, double *d_cost, cudaStream_t st) {
	constexpr bool f32 = sizeof(Real) == 4;
	const int nt = P->nt;
	const int nsl = ch.s1 - ch.s0;
	const JacobiParams jp = eig_params(false);
	const std::vector<Bucket> &beig = f32 ? ch.beig32 : ch.beig;
	SlWork *d_work = f32 ? ch.d_weig32 : ch.d_weig;
	Real *A = reinterpret_cast<Real *>(P->scrA.p), *V = reinterpret_cast<Real *>(P->scrV.p);
	Real *G = reinterpret_cast<Real *>(P->gridscr.p);
	int rc;
	for (size_t bi_ = 0; bi_ < bt.size(); bi_++) {
		const int i0 = bt[bi_].i0, i1 = bt[bi_].i1;
		gp.gbase = d_gbase + bi_ * (size_t)nsl;
		for (int mo = 0; mo < gp.models; mo++) {
			const GridModel &md = gs.mdl[mo];
			const int32_t *tr = P->grows.p + md.tr_ofs;
			if ((rc = g_fan.begin(st)) != kHaSuccess) return rc;
			for (size_t bi = 0; bi < beig.size(); bi++) {
				const Bucket &b = beig[bi];
				const int x0 = std::max(i0, b.first), x1 = std::min(i1, b.first + b.count);
				if (x1 <= x0) continue;
				const cudaStream_t bs = g_fan.at((int)bi);
				const SlWork *wk = d_work + x0;
				// Gram into the V scratch, its pivoted Cholesky factor into the A scratch
				{ HA_LAUNCH(f32 ? kHaB200KXcov32 : kHaB200KXcov64, bs); k_xcov_rows<16, Real><<<x1 - x0, kBlock, 0, bs>>>(wk, P->idx.p, d_X, d_X, nt, tr, md.tr_n, V, G, gp, 0); }
				{ HA_LAUNCH(f32 ? kHaB200KXcov32 : kHaB200KXcov64, bs); k_xcov_rows<16, Real><<<x1 - x0, kBlock, 0, bs>>>(wk, P->idx.p, d_X, d_Y, nt, tr, md.tr_n, A, G, gp, 1); }
				{ HA_LAUNCH(kHaB200KRidge, bs); k_pchol<Real><<<x1 - x0, kBlock, pchol_smem(b.rpl, sizeof(Real)), bs>>>(wk, V, A, P->stats.p); }
				{
					HA_LAUNCH(f32 ? kHaB200KJacobi32 : kHaB200KJacobi64, bs);
					if ((rc = launch_jacobi<Real>(b.rpl, x1 - x0, b.threads, b.smem, bs, wk, A, V, P->scrT.p, P->stats.p, P->uv.p, jp)) != kHaSuccess)
						return rc;
				}
			}
			if ((rc = g_fan.end(st)) != kHaSuccess) return rc;
			{ HA_LAUNCH(kHaB200KGrid, st); k_grid_model<Real><<<i1 - i0, kBlock, 0, st>>>(d_work + i0, P->idx.p, d_X, d_Y, V, P->uv.p, mo, G, gp); }
		}
		{ HA_LAUNCH(kHaB200KGrid, st); k_grid_eval<Real><<<dim3(i1 - i0, gp.n_alphas), kBlock, 0, st>>>(d_work + i0, G, gp); }
		{ HA_LAUNCH(kHaB200KGrid, st); k_grid_final<Real><<<i1 - i0, kBlock, 0, st>>>(d_work + i0, P->idx.p, d_Y, G, gp, P->scrT64.p, rowmajor, d_best, d_cost); }
		HA_CUDA(cudaGetLastError());
	}
	return kHaSuccess;
}

int grid_chunk_launch(HaB200Plan *P, Chunk &ch, const double *d_X, const double *d_Y, const GridSpec &gs,
                      GridParams gp, bool fp32, const std::vector<GridBatch> &bt, const int64_t *d_gbase,
                      int rowmajor, int32_t *d_best, double *d_cost, cudaStream_t st) {
	return fp32 ? grid_chunk_launch_t<float>(P, ch, d_X, d_Y, gs, gp, bt, d_gbase, rowmajor, d_best, d_cost, st)
	            : grid_chunk_launch_t<double>(P, ch, d_X, d_Y, gs, gp, bt, d_gbase, rowmajor, d_best, d_cost, st);
}

// One chunk's grid search enqueued directly (sub-batch plan, scratch and offsets, launches).
int grid_chunk(HaB200Plan *P, Chunk &ch, const double *d_X, const double *d_Y, const GridSpec &gs,
               const GridParams &gp, bool fp32, int rowmajor, int32_t *d_best, double *d_cost, cudaStream_t st) {
	std::vector<GridBatch> bt;
	std::vector<int64_t> gbase;
	grid_plan_chunk(ch, gp, fp32, bt, gbase);
	int64_t mx = 1;
	for (const auto &b : bt) mx = std::max(mx, b.total);
	int rc;
	if ((rc = P->gridscr.ensure((size_t)mx)) != kHaSuccess) return rc;
	if ((rc = P->gbase.ensure(std::max<size_t>(gbase.size(), 1))) != kHaSuccess) return rc;
	HA_CUDA(cudaMemcpyAsync(P->gbase.p, gbase.data(), gbase.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
	HA_CUDA(cudaStreamSynchronize(st));  // the host vector goes out of scope
	return grid_chunk_launch(P, ch, d_X, d_Y, gs, gp, fp32, bt, P->gbase.p, rowmajor, d_best, d_cost, st);
}

int run_ridge_grid(HaB200Plan *P, const double *d_X, const double *d_Y, const GridSpec &gs, int out_kind,
                   double *d_vals, int32_t *d_best, double *d_cost, cudaStream_t st) {
	const int rowmajor = out_kind == kHaB200OutCSR ? 1 : 0;
	const bool fp32 = P->grid_bits == 32;
	int rc;
	if ((rc = grid_prepare(P)) != kHaSuccess) return rc;
	GridParams gp;
	if ((rc = grid_upload(P, gs, st, gp)) != kHaSuccess) return rc;
	// sub-batches of every chunk, their scratch offsets uploaded once, the scratch sized once: what
	// follows is launches only, captured into a CUDA graph (fold x alpha x PC grid of every
	// searchlight) and replayed while the inputs, outputs, grid shape and buffers are the same
	std::vector<std::vector<GridBatch>> bts(P->chunks.size());
	std::vector<size_t> gofs(P->chunks.size());
	std::vector<int64_t> gbase;
	int64_t mx = 1;
	for (size_t c = 0; c < P->chunks.size(); c++) {
		gofs[c] = gbase.size();
		grid_plan_chunk(P->chunks[c], gp, fp32, bts[c], gbase);
		for (const auto &b : bts[c]) mx = std::max(mx, b.total);
	}
	if ((rc = P->gridscr.ensure((size_t)mx)) != kHaSuccess) return rc;
	if ((rc = P->gbase.ensure(std::max<size_t>(gbase.size(), 1))) != kHaSuccess) return rc;
	HA_CUDA(cudaMemcpyAsync(P->gbase.p, gbase.data(), gbase.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
	HA_CUDA(cudaStreamSynchronize(st));
	auto enqueue = [&](cudaStream_t ls) -> int {
		HA_CUDA(cudaMemsetAsync(P->counters.p, 0, 5 * sizeof(int32_t), ls));
		for (size_t c = 0; c < P->chunks.size(); c++) {
			Chunk &ch = P->chunks[c];
			HA_CUDA(cudaMemsetAsync(P->stats.p, 0, (size_t)(ch.s1 - ch.s0) * sizeof(SlStats), ls));
			int r = grid_chunk_launch(P, ch, d_X, d_Y, gs, gp, fp32, bts[c], P->gbase.p + gofs[c], rowmajor, d_best, d_cost, ls);
			if (r != kHaSuccess) return r;
			if ((r = reduce_chunk64(P, ch, out_kind, d_vals, ls)) != kHaSuccess) return r;
		}
		return kHaSuccess;
	};
	if (!graphs_enabled() || g_timing) {
		if ((rc = enqueue(st)) != kHaSuccess) return rc;
	} else {
		const uint64_t key[] = {(uint64_t)(uintptr_t)d_X, (uint64_t)(uintptr_t)d_Y, (uint64_t)(uintptr_t)d_vals,
		                        (uint64_t)(uintptr_t)d_best, (uint64_t)(uintptr_t)d_cost, (uint64_t)out_kind,
		                        (uint64_t)gp.models, (uint64_t)gp.mte, (uint64_t)gp.ntu, (uint64_t)gp.n_alphas,
		                        (uint64_t)gp.n_npcs, (uint64_t)gp.n_untested, (uint64_t)(uintptr_t)gp.alphas,
		                        (uint64_t)(uintptr_t)gp.npcs, (uint64_t)(uintptr_t)gp.mdl, (uint64_t)(uintptr_t)gp.rows,
		                        (uint64_t)(uintptr_t)gp.tpos, (uint64_t)(uintptr_t)gp.winv, (uint64_t)(uintptr_t)gp.urows,
		                        (uint64_t)(uintptr_t)gp.untested, (uint64_t)(uintptr_t)P->gridscr.p,
		                        (uint64_t)(uintptr_t)P->gbase.p, fnv1a(gbase.data(), gbase.size() * 8, 1469598103934665603ULL),
		                        (uint64_t)P->grid_bits};
		std::vector<uint64_t> kv(key, key + sizeof(key) / sizeof(key[0]));
		for (const auto &m : gs.mdl) kv.push_back(((uint64_t)m.tr_ofs << 32) ^ (uint64_t)m.tr_n);
		if (!P->grid_graph || kv != P->grid_key) {
			if (P->grid_graph) cudaGraphExecDestroy(P->grid_graph);
			P->grid_graph = nullptr;
			if ((rc = g_fan.init()) != kHaSuccess) return rc;  // no stream creation inside the capture
			cudaStream_t cs = capture_stream();
			if (!cs) return kHaErrorInternal;
			int64_t n0[kHaB200NumKernelKinds];
			memcpy(n0, g_kernel_n, sizeof(n0));
			const int64_t l0 = g_launches;
			HA_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
			rc = enqueue(cs);
			cudaGraph_t gr = nullptr;
			const cudaError_t ce = cudaStreamEndCapture(cs, &gr);
			P->grid_graph_launches = g_launches - l0;
			g_launches = l0;
			memcpy(g_kernel_n, n0, sizeof(n0));
			if (rc != kHaSuccess || ce != cudaSuccess) {
				if (gr) cudaGraphDestroy(gr);
				fprintf(stderr, "ha_b200: capture of the grid search failed: %s\n", cudaGetErrorString(ce));
				return rc != kHaSuccess ? rc : kHaErrorInternal;
			}
			const cudaError_t ie = cudaGraphInstantiate(&P->grid_graph, gr, 0);
			cudaGraphDestroy(gr);
			if (ie != cudaSuccess) {
				P->grid_graph = nullptr;
				fprintf(stderr, "ha_b200: instantiating the grid-search graph failed: %s\n", cudaGetErrorString(ie));
				return kHaErrorInternal;
			}
			P->grid_key = kv;
		}
		HA_CUDA(cudaGraphLaunch(P->grid_graph, st));
		g_launches += P->grid_graph_launches;
	}
	P->last_chunk = (int)P->chunks.size() - 1;
	P->last_rowmajor = rowmajor;
	return kHaSuccess;
}

// Eigen decomposition of every searchlight's Gram over the given rows (device list, n_rows
// entries): the pivoted Cholesky factor and the eigenvector-mode Jacobi leave the eigenvectors in
// the V scratch and the eigenvalues in the u/v buffer; with d_Y, C = X^T Y over the same rows goes
// to the T scratch of the arithmetic type (float64 T scratch for double, float32 T scratch for
// float).  Then the features of the chunk's searchlights.
template <typename Real>
int eigen_chunk(HaB200Plan *P, Chunk &ch, const double *d_X, const double *d_Y, const int32_t *d_rows, int n_rows,
                float *d_feat, cudaStream_t st) {
	constexpr bool f32 = sizeof(Real) == 4;
	GridParams gp = {};
	const JacobiParams jp = eig_params(false);
	Real *A = reinterpret_cast<Real *>(P->scrA.p), *V = reinterpret_cast<Real *>(P->scrV.p);
	Real *Cout = f32 ? reinterpret_cast<Real *>(P->scrT.p) : reinterpret_cast<Real *>(P->scrT64.p);
	const std::vector<Bucket> &beig = f32 ? ch.beig32 : ch.beig;
	const std::vector<SlWork> &items = f32 ? ch.weig32 : ch.weig;
	SlWork *d_work = f32 ? ch.d_weig32 : ch.d_weig;
	int rc;
	if ((rc = g_fan.begin(st)) != kHaSuccess) return rc;
	for (size_t bi = 0; bi < beig.size(); bi++) {
		const Bucket &b = beig[bi];
		const cudaStream_t bs = g_fan.at((int)bi);
		const SlWork *wk = d_work + b.first;
		{ HA_LAUNCH(f32 ? kHaB200KXcov32 : kHaB200KXcov64, bs); k_xcov_rows<16, Real><<<b.count, kBlock, 0, bs>>>(wk, P->idx.p, d_X, d_X, P->nt, d_rows, n_rows, V, nullptr, gp, 0); }
		if (d_Y) { HA_LAUNCH(f32 ? kHaB200KXcov32 : kHaB200KXcov64, bs); k_xcov_rows<16, Real><<<b.count, kBlock, 0, bs>>>(wk, P->idx.p, d_X, d_Y, P->nt, d_rows, n_rows, Cout, nullptr, gp, 2); }
		{ HA_LAUNCH(kHaB200KRidge, bs); k_pchol<Real><<<b.count, kBlock, pchol_smem(b.rpl, sizeof(Real)), bs>>>(wk, V, A, P->stats.p); }
		{
			HA_LAUNCH(f32 ? kHaB200KJacobi32 : kHaB200KJacobi64, bs);
			if ((rc = launch_jacobi<Real>(b.rpl, b.count, b.threads, b.smem, bs, wk, A, V, P->scrT.p, P->stats.p, P->uv.p, jp)) != kHaSuccess)
				return rc;
		}
	}
	if ((rc = g_fan.end(st)) != kHaSuccess) return rc;
	{ HA_LAUNCH(kHaB200KGrid, st); k_features<<<(int)items.size(), kBlock, 0, st>>>(d_work, P->uv.p, d_feat); }
	HA_CUDA(cudaGetLastError());
	return kHaSuccess;
}

int eigen_chunk_any(HaB200Plan *P, Chunk &ch, const double *d_X, const double *d_Y, const int32_t *d_rows, int n_rows,
                    float *d_feat, cudaStream_t st) {
	return P->grid_bits == 32 ? eigen_chunk<float>(P, ch, d_X, d_Y, d_rows, n_rows, d_feat, st)
	                          : eigen_chunk<double>(P, ch, d_X, d_Y, d_rows, n_rows, d_feat, st);
}

int upload_rows(HaB200Plan *P, const int32_t *rows, int n_rows, cudaStream_t st) {
	if (!rows || n_rows < 1) return kHaErrorArg;
	for (int i = 0; i < n_rows; i++)
		if (rows[i] < 0 || rows[i] >= P->nt) return kHaErrorArg;
	int rc;
	if ((rc = P->gfit.ensure((size_t)n_rows)) != kHaSuccess) return rc;
	HA_CUDA(cudaMemcpyAsync(P->gfit.p, rows, (size_t)n_rows * 4, cudaMemcpyHostToDevice, st));
	HA_CUDA(cudaStreamSynchronize(st));
	return kHaSuccess;
}

// Features of every searchlight over the given rows (no fit).
int run_ridge_features(HaB200Plan *P, const double *d_X, const int32_t *rows, int n_rows, float *d_feat,
                       cudaStream_t st) {
	int rc;
	if ((rc = grid_prepare(P)) != kHaSuccess) return rc;
	if ((rc = upload_rows(P, rows, n_rows, st)) != kHaSuccess) return rc;
	for (size_t c = 0; c < P->chunks.size(); c++) {
		Chunk &ch = P->chunks[c];
		HA_CUDA(cudaMemsetAsync(P->stats.p, 0, (size_t)(ch.s1 - ch.s0) * sizeof(SlStats), st));
		if ((rc = eigen_chunk_any(P, ch, d_X, nullptr, P->gfit.p, n_rows, d_feat, st)) != kHaSuccess) return rc;
	}
	return kHaSuccess;
}

// The learned form: per chunk the eigen decomposition over the fit rows, the features, the
// perceptron's proposal, the single fit at the proposed grid point for searchlights whose proposal
// probability is at least min_prob, the full CV grid search for the others, and the reduction.
int run_ridge_learned(HaB200Plan *P, const double *d_X, const double *d_Y, const int32_t *rows, int n_rows,
                      const GridSpec &gs, const float *d_params, float min_prob, int out_kind, double *d_vals,
                      int32_t *d_choice, float *d_prob, cudaStream_t st) {
	const int rowmajor = out_kind == kHaB200OutCSR ? 1 : 0;
	const bool fp32 = P->grid_bits == 32;
	const int C = (int)(gs.alphas.size() * gs.npcs.size());
	int rc;
	if ((rc = mlp_check(C)) != kHaSuccess) return rc;
	if ((rc = grid_prepare(P)) != kHaSuccess) return rc;
	if ((rc = upload_rows(P, rows, n_rows, st)) != kHaSuccess) return rc;
	GridParams gp;
	if ((rc = grid_upload(P, gs, st, gp)) != kHaSuccess) return rc;
	if ((rc = P->gfeat.ensure((size_t)P->count * (kFeatSv + 1))) != kHaSuccess) return rc;
	HA_CUDA(cudaMemsetAsync(P->counters.p, 0, 5 * sizeof(int32_t), st));
	std::vector<float> hprob;
	for (size_t c = 0; c < P->chunks.size(); c++) {
		Chunk &ch = P->chunks[c];
		const int nsl = ch.s1 - ch.s0;
		HA_CUDA(cudaMemsetAsync(P->stats.p, 0, (size_t)nsl * sizeof(SlStats), st));
		if ((rc = eigen_chunk_any(P, ch, d_X, d_Y, P->gfit.p, n_rows, P->gfeat.p, st)) != kHaSuccess) return rc;
		if ((rc = ha_b200_mlp_infer(d_params, C, P->gfeat.p + (size_t)ch.s0 * (kFeatSv + 1), nsl, d_choice + ch.s0,
		                            d_prob + ch.s0, st)) != kHaSuccess)
			return rc;
		if (fp32) {
			HA_LAUNCH(kHaB200KGrid, st);
			k_proposed_fit<float><<<(int)ch.weig32.size(), kBlock, 0, st>>>(ch.d_weig32, reinterpret_cast<const float *>(P->scrV.p), P->uv.p, reinterpret_cast<float *>(P->scrA.p), P->scrT.p, P->scrT64.p, d_choice, d_prob, min_prob, gp.alphas, gp.npcs, gp.n_npcs, n_rows, rowmajor);
		} else {
			HA_LAUNCH(kHaB200KGrid, st);
			k_proposed_fit<double><<<(int)ch.weig.size(), kBlock, 0, st>>>(ch.d_weig, P->scrV.p, P->uv.p, P->scrA.p, P->scrT64.p, P->scrT64.p, d_choice, d_prob, min_prob, gp.alphas, gp.npcs, gp.n_npcs, n_rows, rowmajor);
		}
		HA_CUDA(cudaGetLastError());
		// searchlights below the threshold: the full grid search
		hprob.resize((size_t)nsl);
		HA_CUDA(cudaMemcpyAsync(hprob.data(), d_prob + ch.s0, (size_t)nsl * 4, cudaMemcpyDeviceToHost, st));
		HA_CUDA(cudaStreamSynchronize(st));
		// the fallback searchlights as a work list of their own (same buckets, same scratch slots)
		Chunk fb;
		fb.s0 = ch.s0;
		fb.s1 = ch.s1;
		const std::vector<Bucket> &cb = fp32 ? ch.beig32 : ch.beig;
		const std::vector<SlWork> &cw = fp32 ? ch.weig32 : ch.weig;
		std::vector<SlWork> &fw = fp32 ? fb.weig32 : fb.weig;
		std::vector<Bucket> &fbk = fp32 ? fb.beig32 : fb.beig;
		for (const Bucket &b : cb) {
			Bucket nb = b;
			nb.first = (int)fw.size();
			for (int i = b.first; i < b.first + b.count; i++)
				if (hprob[(size_t)(cw[i].s - ch.s0)] < min_prob) fw.push_back(cw[i]);
			nb.count = (int)fw.size() - nb.first;
			if (nb.count > 0) fbk.push_back(nb);
		}
		if (!fw.empty()) {
			if ((rc = P->gwork.ensure(fw.size())) != kHaSuccess) return rc;
			HA_CUDA(cudaMemcpyAsync(P->gwork.p, fw.data(), fw.size() * sizeof(SlWork), cudaMemcpyHostToDevice, st));
			(fp32 ? fb.d_weig32 : fb.d_weig) = P->gwork.p;
			if ((rc = grid_chunk(P, fb, d_X, d_Y, gs, gp, fp32, rowmajor, d_choice, nullptr, st)) != kHaSuccess) return rc;
		}
		if ((rc = reduce_chunk64(P, ch, out_kind, d_vals, st)) != kHaSuccess) return rc;
	}
	P->last_chunk = (int)P->chunks.size() - 1;
	P->last_rowmajor = rowmajor;
	return kHaSuccess;
}

// ---- CV split indices (csrc/ha_ensemble.c:12-249) ----

// xoshiro256** seeded through splitmix64, with modulo range reduction (csrc/ha_ensemble.c:12-46).
struct CvRng {
	uint64_t s[4];
	static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
	explicit CvRng(uint64_t seed) {
		for (int i = 0; i < 4; i++) {
			seed += 0x9e3779b97f4a7c15ULL;
			uint64_t z = seed;
			z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
			z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
			s[i] = z ^ (z >> 31);
		}
	}
	uint64_t next() {
		const uint64_t out = rotl(s[1] * 5, 7) * 9;
		const uint64_t t = s[1] << 17;
		s[2] ^= s[0];
		s[3] ^= s[1];
		s[1] ^= s[2];
		s[0] ^= s[3];
		s[2] ^= t;
		s[3] = rotl(s[3], 45);
		return out;
	}
	int32_t below(int32_t n) { return (int32_t)(next() % (uint64_t)n); }
};

// Temporally blocked CV splits with buffer zones: the blocks are shuffled and dealt to folds;
// training rows are a bootstrap of nt draws from the rows outside the test blocks' buffers;
// test rows are the rows outside the buffers of the drawn training rows.  The draws follow
// csrc/ha_ensemble.c:58-249 one for one, so the same seed gives the same splits.
int ensemble_indices(int32_t nt, int32_t n_perms, int32_t n_folds, int32_t blocksize, int32_t buffersize,
                     uint64_t seed, const bool *mask, int32_t *train_out, int32_t *test_out, int32_t *test_sizes) {
	if (nt < 1 || n_perms < 1 || n_folds < 1 || blocksize < 1 || buffersize < 0 || !train_out || !test_out ||
	    !test_sizes)
		return kHaErrorArg;
	CvRng rng(seed);
	const int32_t n_blocks = nt / blocksize, remainder = nt % blocksize;
	const int32_t padded = nt + 2 * buffersize;
	std::vector<int32_t> mapping, order((size_t)n_blocks), test_raw, valid;
	if (mask) {
		mapping.assign((size_t)nt, -1);
		int32_t cum = 0;
		for (int32_t i = 0; i < nt; i++)
			if (mask[i]) mapping[i] = cum++;
	}
	std::vector<char> trm((size_t)padded), tem((size_t)padded), used((size_t)nt);
	auto block_out = [&](std::vector<char> &mk, int32_t centre) {
		for (int32_t b = -buffersize; b <= buffersize; b++) {
			const int32_t pos = centre + buffersize + b;
			if (pos >= 0 && pos < padded) mk[pos] = 0;
		}
	};
	int split = 0;
	for (int32_t perm = 0; perm < n_perms; perm++) {
		const int32_t shift = rng.below(remainder + 1);
		for (int32_t i = 0; i < n_blocks; i++) order[i] = i;
		for (int32_t i = n_blocks - 1; i > 0; i--) std::swap(order[i], order[rng.below(i + 1)]);
		int32_t f0 = 0;
		for (int32_t fold = 0; fold < n_folds; fold++, split++) {
			const int32_t f1 = (int32_t)((int64_t)(fold + 1) * n_blocks / n_folds);
			test_raw.clear();
			for (int32_t b = f0; b < f1; b++)
				for (int32_t k = 0; k < blocksize; k++) {
					const int32_t t = order[b] * blocksize + k + shift;
					if (t < nt) test_raw.push_back(t);
				}
			std::fill(trm.begin(), trm.end(), 1);
			for (int32_t t : test_raw) block_out(trm, t);
			if (mask)
				for (int32_t i = 0; i < nt; i++)
					if (!mask[i]) trm[i + buffersize] = 0;
			valid.clear();
			for (int32_t i = 0; i < nt; i++)
				if (trm[i + buffersize]) valid.push_back(i);
			if (valid.empty()) {
				fprintf(stderr, "ha_ensemble_indices_b200: fold %d leaves no training rows\n", fold);
				return kHaErrorArg;
			}
			int32_t *train = train_out + (size_t)split * nt;
			for (int32_t i = 0; i < nt; i++) train[i] = valid[rng.below((int32_t)valid.size())];
			std::fill(tem.begin(), tem.end(), 1);
			std::fill(used.begin(), used.end(), 0);
			for (int32_t i = 0; i < nt; i++) used[train[i]] = 1;
			for (int32_t i = 0; i < nt; i++)
				if (used[i]) block_out(tem, i);
			if (mask)
				for (int32_t i = 0; i < nt; i++)
					if (!mask[i]) tem[i + buffersize] = 0;
			int32_t *test = test_out + (size_t)split * nt;
			int32_t nte = 0;
			for (int32_t i = 0; i < nt; i++)
				if (tem[i + buffersize]) test[nte++] = i;
			if (mask) {
				for (int32_t i = 0; i < nt; i++) train[i] = mapping[train[i]];
				for (int32_t i = 0; i < nte; i++) test[i] = mapping[test[i]];
			}
			test_sizes[split] = nte;
			f0 = f1;
		}
	}
	return kHaSuccess;
}

int host_threads() {
	int t = g_threads > 0 ? g_threads : omp_get_max_threads();
	return std::max(1, t);
}

// Cached plan for the host entry points (geometry + weights identify it). The hash only
// screens; a hit is confirmed against the full key, so a collision rebuilds instead of reusing.
HaB200Plan *g_cached_plan = nullptr;
int g_cached_dev = -1;  // device the cached plan and the host-call buffers live on
uint64_t g_cached_key = 0;
int g_cached_mode = 0;
double g_cached_radius = 0.0;
std::vector<double> g_cached_aux;  // the dists or weights the cached plan was built from

bool cached_plan_matches(int32_t nt, int32_t nv, const int32_t *idx, const int32_t *off, int32_t count,
                         double radius, int mode, const double *aux) {
	const HaB200Plan *P = g_cached_plan;
	if (P->nt != nt || P->nv != nv || P->count != count || g_cached_mode != mode) return false;
	if (std::memcmp(&g_cached_radius, &radius, sizeof(radius)) != 0) return false;
	if (std::memcmp(P->h_off.data(), off, ((size_t)count + 1) * 4) != 0) return false;
	if (std::memcmp(P->h_idx.data(), idx, (size_t)off[count] * 4) != 0) return false;
	if (aux && (g_cached_aux.size() != (size_t)off[count] ||
	            std::memcmp(g_cached_aux.data(), aux, (size_t)off[count] * 8) != 0))
		return false;
	return true;
}

int get_plan(int32_t nt, int32_t nv, const int32_t *idx, const int32_t *off, const double *dists, int32_t count,
             double radius, const double *weights, bool unweighted, HaB200Plan **out) {
	if (!idx || !off || count <= 0) return kHaErrorArg;
	if (off[count] < 0) return kHaErrorArg;
	uint64_t h = 1469598103934665603ULL;
	int32_t hdr[3] = {nt, nv, count};
	h = fnv1a(hdr, sizeof(hdr), h);
	h = fnv1a(&radius, sizeof(radius), h);
	h = fnv1a(off, ((size_t)count + 1) * 4, h);
	h = fnv1a(idx, (size_t)off[count] * 4, h);
	int mode = dists ? 1 : weights ? 2 : unweighted ? 3 : 0;
	h = fnv1a(&mode, sizeof(mode), h);
	if (dists) h = fnv1a(dists, (size_t)off[count] * 8, h);
	if (weights) h = fnv1a(weights, (size_t)off[count] * 8, h);
	const double *aux = weights ? weights : dists;  // weights override dists in plan_create_impl
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return kHaErrorInternal;
	if (g_cached_plan && g_cached_dev != dev) {
		// the caller switched devices: free the old device's plan and buffers on that device
		if (cudaSetDevice(g_cached_dev) == cudaSuccess) {
			ha_b200_plan_destroy(g_cached_plan);
			g_bufs.release();
			g_fan.release();  // the side streams belong to the old device too
		}
		g_cached_plan = nullptr;
		if (cudaSetDevice(dev) != cudaSuccess) return kHaErrorInternal;
	}
	if (g_cached_plan && g_cached_key == h &&
	    cached_plan_matches(nt, nv, idx, off, count, radius, mode, aux)) {
		*out = g_cached_plan;
		return kHaSuccess;
	}
	if (g_cached_plan) {
		ha_b200_plan_destroy(g_cached_plan);
		g_cached_plan = nullptr;
	}
	int rc = plan_create_impl(nt, nv, idx, off, dists, count, radius, weights, unweighted, out);
	if (rc != kHaSuccess) return rc;
	g_cached_plan = *out;
	g_cached_dev = dev;
	g_cached_key = h;
	g_cached_mode = mode;
	g_cached_radius = radius;
	if (aux) g_cached_aux.assign(aux, aux + off[count]);
	else g_cached_aux.clear();
	return kHaSuccess;
}

// Upload X, Y (float64, host) as column-major device arrays.
int upload_inputs(const double *X, const double *Y, int nt, int nv, bool col_major, const double **dX,
                  const double **dY, cudaStream_t st) {
	size_t n = (size_t)nt * nv;
	int rc;
	if ((rc = g_bufs.X64.ensure(n)) != kHaSuccess) return rc;
	if ((rc = g_bufs.Y64.ensure(n)) != kHaSuccess) return rc;
	if (col_major) {
		HA_CUDA(cudaMemcpyAsync(g_bufs.X64.p, X, n * 8, cudaMemcpyHostToDevice, st));
		HA_CUDA(cudaMemcpyAsync(g_bufs.Y64.p, Y, n * 8, cudaMemcpyHostToDevice, st));
	} else {
		if ((rc = g_bufs.Xtmp.ensure(n)) != kHaSuccess) return rc;
		dim3 grid((nv + 31) / 32, (nt + 31) / 32), block(32, 8);
		HA_CUDA(cudaMemcpyAsync(g_bufs.Xtmp.p, X, n * 8, cudaMemcpyHostToDevice, st));
		{ HA_LAUNCH(kHaB200KConvert, st); k_transpose_f64<<<grid, block, 0, st>>>(g_bufs.Xtmp.p, nt, nv, g_bufs.X64.p); }
		HA_CUDA(cudaMemcpyAsync(g_bufs.Xtmp.p, Y, n * 8, cudaMemcpyHostToDevice, st));
		{ HA_LAUNCH(kHaB200KConvert, st); k_transpose_f64<<<grid, block, 0, st>>>(g_bufs.Xtmp.p, nt, nv, g_bufs.Y64.p); }
		HA_CUDA(cudaGetLastError());
	}
	*dX = g_bufs.X64.p;
	*dY = g_bufs.Y64.p;
	return kHaSuccess;
}

int dense_impl(const double *X, const double *Y, int32_t nt, int32_t nv, const int32_t *idx, const int32_t *off,
               const double *dists, int32_t count, double radius, double *T_out, bool refl, bool scal,
               bool col_major) {
	if (!X || !Y || !idx || !off || !T_out || nt <= 0 || nv <= 0 || count <= 0) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	HaB200Plan *P = nullptr;
	if ((rc = get_plan(nt, nv, idx, off, dists, count, radius, nullptr, false, &P)) != kHaSuccess) return rc;
	cudaStream_t st = 0;
	const double *dX, *dY;
	if ((rc = upload_inputs(X, Y, nt, nv, col_major, &dX, &dY, st)) != kHaSuccess) return rc;
	if ((rc = g_bufs.vals.ensure((size_t)P->nnz)) != kHaSuccess) return rc;
	HA_CUDA(cudaMemsetAsync(g_bufs.vals.p, 0, (size_t)P->nnz * 8, st));
	if ((rc = run_procrustes(P, dX, dY, refl, scal, kHaB200SolverTC, kHaB200OutCSR, g_bufs.vals.p, st)) != kHaSuccess)
		return rc;
	g_bufs.h_vals.resize((size_t)P->nnz);
	HA_CUDA(cudaMemcpyAsync(g_bufs.h_vals.data(), g_bufs.vals.p, (size_t)P->nnz * 8, cudaMemcpyDeviceToHost, st));
	HA_CUDA(cudaStreamSynchronize(st));
	if (P->h_patcol.empty()) {
		P->h_patcol.resize((size_t)P->nnz);
		HA_CUDA(cudaMemcpy(P->h_patcol.data(), P->patcol.p, (size_t)P->nnz * 4, cudaMemcpyDeviceToHost));
	}
	const int64_t *pp = P->h_patptr.data();
	const int32_t *pc = P->h_patcol.data();
	const double *vals = g_bufs.h_vals.data();
#pragma omp parallel for schedule(dynamic, 64) num_threads(host_threads())
	for (int r = 0; r < nv; r++) {
		double *row = T_out + (size_t)r * nv;
		for (int64_t k = pp[r]; k < pp[r + 1]; k++) row[pc[k]] += vals[k];
	}
	return kHaSuccess;
}

// Map the plan's (symmetric) pattern onto a caller CSC pattern: pos[k] = position in the caller's
// arrays of the plan's entry k (column-ordered), or -1 if the caller lacks it (skipped, as
// csrc/ha_sparse.c:137-139 does).
int map_pattern(HaB200Plan *P, const int32_t *indptr, const int32_t *indices, int64_t nnz, std::vector<int64_t> &pos) {
	if (P->h_patcol.empty()) {
		P->h_patcol.resize((size_t)P->nnz);
		HA_CUDA(cudaMemcpy(P->h_patcol.data(), P->patcol.p, (size_t)P->nnz * 4, cudaMemcpyDeviceToHost));
	}
	if (indptr[0] != 0 || indptr[P->nv] != nnz) return kHaErrorArg;
	pos.assign((size_t)P->nnz, -1);
	const int nv = P->nv;
	for (int c = 0; c < nv; c++) {
		int64_t a = P->h_patptr[c], ae = P->h_patptr[c + 1];
		int64_t b = indptr[c], be = indptr[c + 1];
		while (a < ae && b < be) {
			int32_t ra = P->h_patcol[a], rb = indices[b];
			if (ra == rb) { pos[a] = b; a++; b++; }
			else if (ra < rb) a++;
			else b++;
		}
	}
	return kHaSuccess;
}

int csc_impl(const double *X, const double *Y, int32_t nt, int32_t nv, const int32_t *idx, const int32_t *off,
             int32_t count, const double *weights, const int32_t *indptr, const int32_t *indices, int64_t nnz,
             double *data, bool refl, bool scal, bool col_major, bool ridge, double alpha) {
	if (!X || !Y || !idx || !off || !indptr || !indices || !data || nt <= 0 || nv <= 0 || count <= 0 || nnz < 0)
		return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	HaB200Plan *P = nullptr;
	if ((rc = get_plan(nt, nv, idx, off, nullptr, count, 0.0, weights, weights == nullptr, &P)) != kHaSuccess) return rc;
	std::vector<int64_t> pos;
	if ((rc = map_pattern(P, indptr, indices, nnz, pos)) != kHaSuccess) return rc;
	cudaStream_t st = 0;
	const double *dX, *dY;
	if ((rc = upload_inputs(X, Y, nt, nv, col_major, &dX, &dY, st)) != kHaSuccess) return rc;
	if ((rc = g_bufs.vals.ensure((size_t)P->nnz)) != kHaSuccess) return rc;
	HA_CUDA(cudaMemsetAsync(g_bufs.vals.p, 0, (size_t)P->nnz * 8, st));
	if (ridge)
		rc = ha_b200_plan_ridge_device(P, dX, dY, alpha, kHaB200OutCSC, g_bufs.vals.p, st);
	else
		rc = run_procrustes(P, dX, dY, refl, scal, kHaB200SolverTC, kHaB200OutCSC, g_bufs.vals.p, st);
	if (rc != kHaSuccess) return rc;
	g_bufs.h_vals.resize((size_t)P->nnz);
	HA_CUDA(cudaMemcpyAsync(g_bufs.h_vals.data(), g_bufs.vals.p, (size_t)P->nnz * 8, cudaMemcpyDeviceToHost, st));
	HA_CUDA(cudaStreamSynchronize(st));
	const double *vals = g_bufs.h_vals.data();
	const int64_t tot = P->nnz;
#pragma omp parallel for schedule(static) num_threads(host_threads())
	for (int64_t k = 0; k < tot; k++)
		if (pos[k] >= 0) data[pos[k]] += vals[k];
	return kHaSuccess;
}

int grid_csc_impl(const double *X, const double *Y, int32_t nt, int32_t nv, const int32_t *idx, const int32_t *off,
                  int32_t count, const double *weights, const int32_t *indptr, const int32_t *indices, int64_t nnz,
                  double *data, const GridSpec &gs, int32_t *best_out, double *cost_out, bool col_major) {
	if (!X || !Y || !idx || !off || !indptr || !indices || !data || !best_out || nt <= 0 || nv <= 0 || count <= 0 ||
	    nnz < 0)
		return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	HaB200Plan *P = nullptr;
	if ((rc = get_plan(nt, nv, idx, off, nullptr, count, 0.0, weights, weights == nullptr, &P)) != kHaSuccess) return rc;
	std::vector<int64_t> pos;
	if ((rc = map_pattern(P, indptr, indices, nnz, pos)) != kHaSuccess) return rc;
	cudaStream_t st = 0;
	const double *dX, *dY;
	if ((rc = upload_inputs(X, Y, nt, nv, col_major, &dX, &dY, st)) != kHaSuccess) return rc;
	const int grid = (int)(gs.alphas.size() * gs.npcs.size());
	DevArr<int32_t> dbest;
	DevArr<double> dcost;
	auto done = [&](int code) {
		dbest.release();
		dcost.release();
		return code;
	};
	if ((rc = g_bufs.vals.ensure((size_t)P->nnz)) != kHaSuccess) return done(rc);
	if ((rc = dbest.ensure((size_t)count)) != kHaSuccess) return done(rc);
	if (cost_out && (rc = dcost.ensure((size_t)count * grid)) != kHaSuccess) return done(rc);
	if (cudaMemsetAsync(g_bufs.vals.p, 0, (size_t)P->nnz * 8, st) != cudaSuccess) return done(kHaErrorInternal);
	if ((rc = run_ridge_grid(P, dX, dY, gs, kHaB200OutCSC, g_bufs.vals.p, dbest.p, cost_out ? dcost.p : nullptr, st)) !=
	    kHaSuccess)
		return done(rc);
	g_bufs.h_vals.resize((size_t)P->nnz);
	if (cudaMemcpyAsync(g_bufs.h_vals.data(), g_bufs.vals.p, (size_t)P->nnz * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
	    cudaMemcpyAsync(best_out, dbest.p, (size_t)count * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
	    (cost_out && cudaMemcpyAsync(cost_out, dcost.p, (size_t)count * grid * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
	    cudaStreamSynchronize(st) != cudaSuccess) {
		fprintf(stderr, "ha_searchlight_ridge_grid_b200: CUDA failure: %s\n", cudaGetErrorString(cudaGetLastError()));
		return done(kHaErrorInternal);
	}
	const double *vals = g_bufs.h_vals.data();
	const int64_t tot = P->nnz;
#pragma omp parallel for schedule(static) num_threads(host_threads())
	for (int64_t k = 0; k < tot; k++)
		if (pos[k] >= 0) data[pos[k]] += vals[k];
	return done(kHaSuccess);
}

}  // namespace

// Searchlight template loop on the device (csrc/ha_template.c:14-114 with searchlight solves).
int template_impl(const double *dms, int ns, int nt, int nv, const int32_t *idx, const int32_t *off,
                  const double *dists, int count, double radius, bool refl, bool scal, bool zs, int level2,
                  double *tpl_out) {
	if (!dms || !tpl_out || ns < 2 || nt <= 0 || nv <= 0 || count <= 0 || level2 < 0) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	HaB200Plan *P = nullptr;
	if ((rc = get_plan(nt, nv, idx, off, dists, count, radius, nullptr, false, &P)) != kHaSuccess) return rc;
	const size_t m = (size_t)nt * nv;
	DevArr<double> D, A, common, ref, vals;
	auto done = [&](int code) {
		D.release(); A.release(); common.release(); ref.release(); vals.release();
		return code;
	};
	if ((rc = D.ensure(m * ns)) != kHaSuccess) return done(rc);
	if ((rc = A.ensure(m * ns)) != kHaSuccess) return done(rc);
	if ((rc = common.ensure(m)) != kHaSuccess) return done(rc);
	if ((rc = ref.ensure(m)) != kHaSuccess) return done(rc);
	if ((rc = vals.ensure((size_t)P->nnz)) != kHaSuccess) return done(rc);
	cudaStream_t st = 0;
	if (cudaMemcpyAsync(D.p, dms, m * ns * 8, cudaMemcpyHostToDevice, st) != cudaSuccess) return done(kHaErrorInternal);
	const int eg = 148 * 8;
	const int zg = (nv + 127) / 128;
	// aligned_s = X_s @ SL(X_s -> target)
	auto align = [&](int s, const double *target) -> int {
		if (cudaMemsetAsync(vals.p, 0, (size_t)P->nnz * 8, st) != cudaSuccess) return kHaErrorInternal;
		int r = run_procrustes(P, D.p + m * s, target, refl, scal, kHaB200SolverTC, kHaB200OutCSC, vals.p, st);
		if (r != kHaSuccess) return r;
		k_spmm_csc<<<nv, 128, 0, st>>>(D.p + m * s, nt, nv, P->patptr.p, P->patcol.p, vals.p, A.p + m * s);
		return cudaGetLastError() == cudaSuccess ? kHaSuccess : kHaErrorInternal;
	};
	if (cudaMemcpyAsync(common.p, D.p, m * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
	    cudaMemcpyAsync(A.p, D.p, m * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
		return done(kHaErrorInternal);
	for (int s = 1; s < ns; s++) {
		if ((rc = align(s, common.p)) != kHaSuccess) return done(rc);
		if (zs) k_zscore_cols<<<zg, 128, 0, st>>>(A.p + m * s, nt, nv);
		k_axpbz<<<eg, 256, 0, st>>>(common.p, common.p, A.p + m * s, 0.5, 1.0, (int64_t)m);
		if (zs) k_zscore_cols<<<zg, 128, 0, st>>>(common.p, nt, nv);
	}
	for (int it = 0; it < level2; it++) {
		// common = sum over subjects (in subject order)
		k_axpbz<<<eg, 256, 0, st>>>(common.p, A.p, nullptr, 1.0, 0.0, (int64_t)m);
		for (int s = 1; s < ns; s++) k_axpbz<<<eg, 256, 0, st>>>(common.p, common.p, A.p + m * s, 1.0, 1.0, (int64_t)m);
		for (int s = 0; s < ns; s++) {
			k_axpbz<<<eg, 256, 0, st>>>(ref.p, common.p, A.p + m * s, 1.0 / (ns - 1), -1.0, (int64_t)m);
			if (zs) k_zscore_cols<<<zg, 128, 0, st>>>(ref.p, nt, nv);
			if ((rc = align(s, ref.p)) != kHaSuccess) return done(rc);
		}
	}
	k_axpbz<<<eg, 256, 0, st>>>(common.p, A.p, nullptr, 1.0, 0.0, (int64_t)m);
	for (int s = 1; s < ns; s++) k_axpbz<<<eg, 256, 0, st>>>(common.p, common.p, A.p + m * s, 1.0, 1.0, (int64_t)m);
	if (zs)
		k_zscore_cols<<<zg, 128, 0, st>>>(common.p, nt, nv);
	else
		k_axpbz<<<eg, 256, 0, st>>>(common.p, common.p, nullptr, 1.0 / ns, 0.0, (int64_t)m);
	if (cudaGetLastError() != cudaSuccess ||
	    cudaMemcpyAsync(tpl_out, common.p, m * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
	    cudaStreamSynchronize(st) != cudaSuccess) {
		fprintf(stderr, "ha_searchlight_template_b200: CUDA failure: %s\n", cudaGetErrorString(cudaGetLastError()));
		return done(kHaErrorInternal);
	}
	return done(kHaSuccess);
}

// Searchlight PCA template (src/hyperalignment/searchlight.py:215-236, tpl_kind="pca"), float64
// throughout.  Consecutive searchlights form batches sized to the scratch budget; per batch: the
// Gram of the smaller side (k_pca_gram), its pivoted Cholesky factor and eigenvector-mode Jacobi,
// the template and B = tmpl^T M (k_pca_tmpl), the float64 Jacobi polar of B, C = tmpl R
// (k_pca_contrib) and the weighted per-vertex reduction into the template (k_pca_reduce).
int pca_template_impl(const double *dms, int ns, int nt, int nv, const int32_t *idx, const int32_t *off,
                      const double *dists, int count, double radius, double *tpl_out) {
	if (!dms || !tpl_out || ns < 1 || nt <= 0 || nv <= 0 || count <= 0) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	HaB200Plan *P = nullptr;
	if ((rc = get_plan(nt, nv, idx, off, dists, count, radius, nullptr, false, &P)) != kHaSuccess) return rc;
	// per searchlight: Gram order, scratch region of the eigen / polar solves, template scratch
	std::vector<int> mg(count), nn(count);
	std::vector<int64_t> region(count), ptot(count);
	std::vector<size_t> bytes(count);
	for (int s = 0; s < count; s++) {
		const int n = P->h_off[s + 1] - P->h_off[s];
		const int64_t vn = (int64_t)ns * n;
		const int m = vn < nt ? (int)vn : nt;
		if (n > nt || m > kPcaMaxM) {
			fprintf(stderr,
			        "ha_searchlight_pca_template_b200: searchlight %d has %d vertices; the GPU template needs n <= nt (%d) "
			        "and min(nt, n_subj * n) <= %d\n", s, n, nt, kPcaMaxM);
			return kHaErrorArg;
		}
		nn[s] = n;
		mg[s] = n > 0 ? m : nt;
		if (n == 0) { region[s] = ptot[s] = 0; bytes[s] = 0; continue; }
		int be, ke, bp, kp;
		size_t me, mp;
		jacobi_layout(m, true, be, ke, me, kSmemMax, false);
		jacobi_layout(n, true, bp, kp, mp);
		int64_t r = std::max<int64_t>((int64_t)m * std::max(m, be * ke), (int64_t)n * kp * bp);
		region[s] = (r + 31) & ~(int64_t)31;
		ptot[s] = PcaLayout::make(nt, n, m, m != nt).total;
		bytes[s] = (size_t)(2 * region[s] + ptot[s] + m + 2 * n) * 8 + (size_t)n * n * 4 + 2 * sizeof(SlStats);
	}
	// batches of consecutive searchlights
	const size_t budget = scratch_budget_bytes();
	std::vector<int> bstart{0};
	{
		size_t acc = 0;
		for (int s = 0; s < count; s++) {
			if (s > bstart.back() && acc + bytes[s] > budget) {
				bstart.push_back(s);
				acc = 0;
			}
			acc += bytes[s];
		}
		bstart.push_back(count);
	}
	int64_t maxR = 1, maxP = 1, maxT = 1, maxUV = 1;
	int maxS = 1;
	for (size_t b = 0; b + 1 < bstart.size(); b++) {
		int64_t R = 0, Pt = 0, Tt = 0, U = 0;
		for (int s = bstart[b]; s < bstart[b + 1]; s++) {
			R += region[s];
			Pt += ptot[s];
			Tt += (int64_t)nn[s] * nn[s];
			U += nn[s] > 0 ? mg[s] + 2 * nn[s] : 0;
		}
		maxR = std::max(maxR, R);
		maxP = std::max(maxP, Pt);
		maxT = std::max(maxT, Tt);
		maxUV = std::max(maxUV, U);
		maxS = std::max(maxS, bstart[b + 1] - bstart[b]);
	}
	const size_t m1 = (size_t)nt * nv;
	DevArr<double> D, eA, eV, Pw, uvb, tpl;
	DevArr<float> T;
	DevArr<SlStats> stE, stP;
	DevArr<SlWork> dwe, dwp, dwes, dwps;
	DevArr<int64_t> dpofs;
	DevArr<int32_t> dmg;
	auto done = [&](int code) {
		D.release(); eA.release(); eV.release(); Pw.release(); uvb.release(); tpl.release(); T.release();
		stE.release(); stP.release(); dwe.release(); dwp.release(); dwes.release(); dwps.release();
		dpofs.release(); dmg.release();
		return code;
	};
	if ((rc = D.ensure(m1 * ns)) != kHaSuccess || (rc = tpl.ensure(m1)) != kHaSuccess ||
	    (rc = eA.ensure((size_t)maxR)) != kHaSuccess || (rc = eV.ensure((size_t)maxR)) != kHaSuccess ||
	    (rc = Pw.ensure((size_t)maxP)) != kHaSuccess || (rc = uvb.ensure((size_t)maxUV)) != kHaSuccess ||
	    (rc = T.ensure((size_t)maxT)) != kHaSuccess || (rc = stE.ensure((size_t)maxS)) != kHaSuccess ||
	    (rc = stP.ensure((size_t)maxS)) != kHaSuccess || (rc = dwe.ensure((size_t)maxS)) != kHaSuccess ||
	    (rc = dwp.ensure((size_t)maxS)) != kHaSuccess || (rc = dwes.ensure((size_t)maxS)) != kHaSuccess ||
	    (rc = dwps.ensure((size_t)maxS)) != kHaSuccess || (rc = dpofs.ensure((size_t)maxS)) != kHaSuccess ||
	    (rc = dmg.ensure((size_t)maxS)) != kHaSuccess)
		return done(rc);
	cudaStream_t st = 0;
	if (cudaMemcpyAsync(D.p, dms, m1 * ns * 8, cudaMemcpyHostToDevice, st) != cudaSuccess ||
	    cudaMemsetAsync(tpl.p, 0, m1 * 8, st) != cudaSuccess)
		return done(kHaErrorInternal);
	const JacobiParams jpe = eig_params(false);
	JacobiParams jpp;
	jpp.max_sweeps = 40;
	jpp.t_rowmajor = 0;
	jpp.ill_ratio = 0.0;
	jpp.weak = weak_factor();
	jpp.eig = 0;
	jpp.only_flagged = 0;
	jpp.keep_v = 0;
	jpp.warm = 0;
	jpp.stop_cos = fp64_stop_cos();
	for (size_t b = 0; b + 1 < bstart.size(); b++) {
		const int s_lo = bstart[b], s_hi = bstart[b + 1];
		std::vector<SlWork> we, wp;
		std::vector<int64_t> pofs(s_hi - s_lo, 0);
		std::vector<int32_t> mgb(s_hi - s_lo);
		int64_t ro = 0, po = 0, to = 0, uo = 0;
		for (int s = s_lo; s < s_hi; s++) {
			const int q = s - s_lo, n = nn[s], m = mg[s];
			mgb[q] = m;
			if (n == 0) continue;
			SlWork e, p;
			e.s = p.s = s;
			e.slot = p.slot = q;
			e.sofs = p.sofs = P->h_off[s];
			e.aofs = p.aofs = ro;
			e.tofs = p.tofs = to;
			e.n = m;
			p.n = n;
			{
				int bb, kk;
				size_t mm;
				jacobi_layout(m, true, bb, kk, mm, kSmemMax, false);
				e.bsz = bb; e.nblk = kk;
				jacobi_layout(n, true, bb, kk, mm);
				p.bsz = bb; p.nblk = kk;
			}
			e.uvofs = uo;
			p.uvofs = uo + m;
			we.push_back(e);
			wp.push_back(p);
			pofs[q] = po;
			ro += region[s];
			po += ptot[s];
			to += (int64_t)n * n;
			uo += m + 2 * n;
		}
		const int nb = (int)we.size();
		if (nb == 0) continue;
		std::vector<SlWork> wes = we, wps = wp;
		const std::vector<Bucket> be = bucketize(wes, 2), bp = bucketize(wps, 1);
		if (cudaMemcpyAsync(dwe.p, we.data(), nb * sizeof(SlWork), cudaMemcpyHostToDevice, st) != cudaSuccess ||
		    cudaMemcpyAsync(dwp.p, wp.data(), nb * sizeof(SlWork), cudaMemcpyHostToDevice, st) != cudaSuccess ||
		    cudaMemcpyAsync(dwes.p, wes.data(), nb * sizeof(SlWork), cudaMemcpyHostToDevice, st) != cudaSuccess ||
		    cudaMemcpyAsync(dwps.p, wps.data(), nb * sizeof(SlWork), cudaMemcpyHostToDevice, st) != cudaSuccess ||
		    cudaMemcpyAsync(dpofs.p, pofs.data(), pofs.size() * 8, cudaMemcpyHostToDevice, st) != cudaSuccess ||
		    cudaMemcpyAsync(dmg.p, mgb.data(), mgb.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
		    cudaMemsetAsync(stE.p, 0, (size_t)(s_hi - s_lo) * sizeof(SlStats), st) != cudaSuccess ||
		    cudaMemsetAsync(stP.p, 0, (size_t)(s_hi - s_lo) * sizeof(SlStats), st) != cudaSuccess)
			return done(kHaErrorInternal);
		{ HA_LAUNCH(kHaB200KPca, st); k_pca_gram<16><<<nb, kBlock, 0, st>>>(dwe.p, P->idx.p, P->off.p, D.p, ns, nt, nv, eV.p); }
		for (const Bucket &k : be) {
			const SlWork *wk = dwes.p + k.first;
			{ HA_LAUNCH(kHaB200KRidge, st); k_pchol<double><<<k.count, kBlock, pchol_smem(k.rpl), st>>>(wk, eV.p, eA.p, stE.p); }
			HA_LAUNCH(kHaB200KJacobi64, st);
			if ((rc = launch_jacobi<double>(k.rpl, k.count, k.threads, k.smem, st, wk, eA.p, eV.p, T.p, stE.p, uvb.p, jpe)) != kHaSuccess)
				return done(rc);
		}
		{ HA_LAUNCH(kHaB200KPca, st); k_pca_tmpl<<<nb, kBlock, 0, st>>>(dwe.p, dwp.p, P->idx.p, D.p, ns, nt, nv, eV.p, uvb.p, dpofs.p, Pw.p, eA.p); }
		for (const Bucket &k : bp) {
			const SlWork *wk = dwps.p + k.first;
			{
				HA_LAUNCH(kHaB200KJacobi64, st);
				if ((rc = launch_jacobi<double>(k.rpl, k.count, k.threads, k.smem, st, wk, eA.p, eV.p, T.p, stP.p, uvb.p, jpp)) != kHaSuccess)
					return done(rc);
			}
			if (k.blocked) { HA_LAUNCH(kHaB200KFormT64, st); k_form_t_global<double><<<k.count, kBlock, 0, st>>>(wk, eA.p, eV.p, T.p, stP.p, 0, 0); }
		}
		{ HA_LAUNCH(kHaB200KPca, st); k_pca_contrib<<<nb, kBlock, 0, st>>>(dwe.p, dwp.p, T.p, nt, dpofs.p, Pw.p); }
		{ HA_LAUNCH(kHaB200KPca, st); k_pca_reduce<<<nv, kBlock, 0, st>>>(P->vlptr.p, P->vlent.p, P->off.p, P->has_weights ? P->w.p : nullptr,
		                                                              dpofs.p, dmg.p, Pw.p, nt, s_lo, s_hi, tpl.p); }
		// the host work lists are rebuilt for the next batch
		if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
			fprintf(stderr, "ha_searchlight_pca_template_b200: CUDA failure: %s\n", cudaGetErrorString(cudaGetLastError()));
			return done(kHaErrorInternal);
		}
	}
	if (cudaMemcpyAsync(tpl_out, tpl.p, m1 * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
	    cudaStreamSynchronize(st) != cudaSuccess) {
		fprintf(stderr, "ha_searchlight_pca_template_b200: CUDA failure: %s\n", cudaGetErrorString(cudaGetLastError()));
		return done(kHaErrorInternal);
	}
	return done(kHaSuccess);
}

// =============================================================================================
// C ABI
// =============================================================================================

extern "C" {

int ha_b200_init(void) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (g_inited) return kHaSuccess;
	int ndev = 0;
	cudaError_t e = cudaGetDeviceCount(&ndev);
	if (e != cudaSuccess || ndev == 0) {
		cudaGetLastError();
		fprintf(stderr, "ha_b200: no CUDA device available (%s)\n", cudaGetErrorString(e));
		return kHaErrorInternal;
	}
	int dev = 0;
	cudaGetDevice(&dev);
	cudaDeviceProp prop;
	if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return kHaErrorInternal;
	if (prop.major != 10) {
		fprintf(stderr, "ha_b200: device %d is sm_%d%d; this library is built for sm_100a only\n", dev, prop.major,
		        prop.minor);
		return kHaErrorInternal;
	}
	if (cudaFree(0) != cudaSuccess) return kHaErrorInternal;
	g_num_sms = prop.multiProcessorCount;
	g_inited = true;
	return kHaSuccess;
}

void ha_b200_cleanup(void) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (g_cached_plan) {
		ha_b200_plan_destroy(g_cached_plan);
		g_cached_plan = nullptr;
	}
	std::vector<double>().swap(g_cached_aux);
	g_bufs.release();
	g_fan.release();
	g_mlp.release();
	g_inited = false;
}

bool ha_b200_available(void) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	return g_inited;
}

void ha_set_num_threads(int n) { g_threads = n; }
int ha_get_num_threads(void) { return host_threads(); }

int ha_searchlight_procrustes_b200(const double *X_data, const double *Y_data, int32_t nt, int32_t nv,
                                   const int32_t *sl_indices, const int32_t *sl_offsets, const double *sl_dists,
                                   int32_t count, double radius, double *T_out, bool isReflection, bool isScaling,
                                   bool col_major) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	return dense_impl(X_data, Y_data, nt, nv, sl_indices, sl_offsets, sl_dists, count, radius, T_out, isReflection,
	                  isScaling, col_major);
}

int ha_searchlight_procrustes_dense(const double *X_data, const double *Y_data, int32_t nt, int32_t nv,
                                    const int32_t *sl_indices, const int32_t *sl_offsets, const double *sl_dists,
                                    int32_t count, double radius, double *T_out, bool isReflection, bool isScaling,
                                    THaBackend backend, bool col_major) {
	if ((int)backend != 4) {
		fprintf(stderr, "ha_searchlight_procrustes_dense: this library implements only backend 4 (B200); got %d\n",
		        (int)backend);
		return kHaErrorArg;
	}
	return ha_searchlight_procrustes_b200(X_data, Y_data, nt, nv, sl_indices, sl_offsets, sl_dists, count, radius,
	                                      T_out, isReflection, isScaling, col_major);
}

int ha_searchlight_template_b200(const double *dms, int32_t n_subj, int32_t nt, int32_t nv,
                                 const int32_t *sl_indices, const int32_t *sl_offsets, const double *sl_dists,
                                 int32_t count, double radius, bool isReflection, bool isScaling,
                                 bool isZscoreCommon, int32_t level2_iter, double *tpl_out) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	return template_impl(dms, n_subj, nt, nv, sl_indices, sl_offsets, sl_dists, count, radius, isReflection,
	                     isScaling, isZscoreCommon, level2_iter, tpl_out);
}

int ha_searchlight_pca_template_b200(const double *dms, int32_t n_subj, int32_t nt, int32_t nv,
                                     const int32_t *sl_indices, const int32_t *sl_offsets, const double *sl_dists,
                                     int32_t count, double radius, double *tpl_out) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	return pca_template_impl(dms, n_subj, nt, nv, sl_indices, sl_offsets, sl_dists, count, radius, tpl_out);
}

int ha_sparse_pattern_b200(const int32_t *sl_indices, const int32_t *sl_offsets, int32_t count, int32_t nv,
                           int32_t *indptr, int32_t *indices, int64_t capacity, int64_t *nnz) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!indptr || !nnz) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	HaB200Plan *P = nullptr;
	if ((rc = get_plan(1, nv, sl_indices, sl_offsets, nullptr, count, 0.0, nullptr, true, &P)) != kHaSuccess) return rc;
	*nnz = P->nnz;
	if (P->nnz > INT32_MAX) {
		fprintf(stderr, "ha_sparse_pattern_b200: nnz %lld does not fit int32 indptr\n", (long long)P->nnz);
		return kHaErrorArg;
	}
	for (int v = 0; v <= nv; v++) indptr[v] = (int32_t)P->h_patptr[v];
	if (indices) {
		if (capacity < P->nnz) return kHaErrorArg;
		HA_CUDA(cudaMemcpy(indices, P->patcol.p, (size_t)P->nnz * 4, cudaMemcpyDeviceToHost));
	}
	return kHaSuccess;
}

int ha_searchlight_weights_b200(const int32_t *sl_indices, const int32_t *sl_offsets, const double *sl_dists,
                                int32_t count, double radius, int32_t nv, double *weights_out) {
	if (!weights_out) return kHaErrorArg;
	int rc = validate_searchlights(sl_indices, sl_offsets, count, nv);
	if (rc != kHaSuccess) return rc;
	compute_weights(sl_indices, sl_offsets, sl_dists, count, radius, nv, weights_out);
	return kHaSuccess;
}

int ha_searchlight_procrustes_csc_b200(const double *X_data, const double *Y_data, int32_t nt, int32_t nv,
                                       const int32_t *sl_indices, const int32_t *sl_offsets, int32_t count,
                                       const double *weights, const int32_t *indptr, const int32_t *indices,
                                       int64_t nnz, double *data, bool isReflection, bool isScaling,
                                       bool col_major) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	return csc_impl(X_data, Y_data, nt, nv, sl_indices, sl_offsets, count, weights, indptr, indices, nnz, data,
	                isReflection, isScaling, col_major, false, 0.0);
}

int ha_searchlight_ridge_grid_b200(const double *X_data, const double *Y_data, int32_t nt, int32_t nv,
                                   const int32_t *sl_indices, const int32_t *sl_offsets, int32_t count,
                                   const double *weights, const int32_t *indptr, const int32_t *indices, int64_t nnz,
                                   double *data, const double *alphas, int32_t n_alphas, const int32_t *npcs,
                                   int32_t n_npcs, const int32_t *const *train_idx_li,
                                   const int32_t *const *test_idx_li, const int32_t *train_sizes,
                                   const int32_t *test_sizes, int32_t n_models, int32_t *best_out, double *cost_out,
                                   bool col_major) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (nt <= 0) return kHaErrorArg;
	GridSpec gs;
	int rc = grid_spec(nt, alphas, n_alphas, npcs, n_npcs, train_idx_li, test_idx_li, train_sizes, test_sizes,
	                   n_models, gs);
	if (rc != kHaSuccess) return rc;
	return grid_csc_impl(X_data, Y_data, nt, nv, sl_indices, sl_offsets, count, weights, indptr, indices, nnz, data,
	                     gs, best_out, cost_out, col_major);
}

int ha_ensemble_indices_b200(int32_t nt, int32_t n_perms, int32_t n_folds, int32_t blocksize, int32_t buffersize,
                             uint64_t seed, const bool *mask, int32_t *train_out, int32_t *test_out,
                             int32_t *test_sizes) {
	return ensemble_indices(nt, n_perms, n_folds, blocksize, buffersize, seed, mask, train_out, test_out, test_sizes);
}

int ha_searchlight_ridge_csc_b200(const double *X_data, const double *Y_data, int32_t nt, int32_t nv,
                                  const int32_t *sl_indices, const int32_t *sl_offsets, int32_t count,
                                  const double *weights, const int32_t *indptr, const int32_t *indices, int64_t nnz,
                                  double *data, double alpha, bool col_major) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	return csc_impl(X_data, Y_data, nt, nv, sl_indices, sl_offsets, count, weights, indptr, indices, nnz, data,
	                true, false, col_major, true, alpha);
}

int ha_b200_plan_create(int32_t nt, int32_t nv, const int32_t *sl_indices, const int32_t *sl_offsets,
                        const double *sl_dists, int32_t count, double radius, const double *weights,
                        HaB200Plan **plan_out) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!plan_out) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	return plan_create_impl(nt, nv, sl_indices, sl_offsets, sl_dists, count, radius, weights, false, plan_out);
}

void ha_b200_plan_destroy(HaB200Plan *P) {
	if (!P) return;
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (P == g_cached_plan) g_cached_plan = nullptr;
	for (auto &ch : P->chunks) {
		if (ch.d_w32) cudaFree(ch.d_w32);
		if (ch.d_w64) cudaFree(ch.d_w64);
		if (ch.d_weig) cudaFree(ch.d_weig);
		if (ch.d_weig32) cudaFree(ch.d_weig32);
		if (ch.d_tofs) cudaFree(ch.d_tofs);
		if (ch.d_tcw) cudaFree(ch.d_tcw);
		if (ch.tc_graph) cudaGraphExecDestroy(ch.tc_graph);
		for (int c = 0; c < 2; c++) {
			if (ch.d_tct[c]) cudaFree(ch.d_tct[c]);
			if (ch.d_tco[c]) cudaFree(ch.d_tco[c]);
		}
	}
	P->idx.release(); P->off.release(); P->lo.release(); P->hi.release(); P->w.release();
	P->vlptr.release(); P->vlent.release(); P->patptr.release(); P->patcol.release();
	P->scrA.release(); P->scrV.release(); P->scrT.release(); P->scrT64.release(); P->uv.release(); P->scale.release();
	P->stats.release(); P->X32.release(); P->Y32.release(); P->var.release(); P->counters.release();
	P->gridscr.release(); P->galpha.release(); P->gwinv.release(); P->gbase.release(); P->gnpcs.release();
	P->grows.release(); P->gtpos.release(); P->gurows.release(); P->guntested.release(); P->gmdl.release();
	P->gfit.release(); P->gfeat.release(); P->gwork.release();
	P->tcXb.release(); P->tcYb.release(); P->tcXp.release(); P->tcXq.release(); P->tcPp.release(); P->tcA.release(); P->tcRes.release();
	P->tcSt.release(); P->tcSched.release(); P->tcPlain.release(); P->tcQueue.release();
	if (P->grid_graph) cudaGraphExecDestroy(P->grid_graph);
	delete P;
}

int64_t ha_b200_plan_nnz(const HaB200Plan *P) { return P ? P->nnz : -1; }

int ha_b200_plan_pattern(const HaB200Plan *P, int64_t *indptr, int32_t *indices) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || !indptr) return kHaErrorArg;
	memcpy(indptr, P->h_patptr.data(), ((size_t)P->nv + 1) * 8);
	if (indices) HA_CUDA(cudaMemcpy(indices, P->patcol.p, (size_t)P->nnz * 4, cudaMemcpyDeviceToHost));
	return kHaSuccess;
}

int ha_b200_plan_device_pattern(const HaB200Plan *P, const int64_t **d_indptr, const int32_t **d_indices) {
	if (!P || !d_indptr || !d_indices) return kHaErrorArg;
	*d_indptr = P->patptr.p;
	*d_indices = P->patcol.p;
	return kHaSuccess;
}

int ha_b200_plan_stats(const HaB200Plan *P, int32_t *n_fp64, int32_t *n_unconverged) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P) return kHaErrorArg;
	int32_t h[4] = {0, 0, 0, 0};
	HA_CUDA(cudaMemcpy(h, P->counters.p, sizeof(h), cudaMemcpyDeviceToHost));
	if (n_fp64) *n_fp64 = h[0];
	if (n_unconverged) *n_unconverged = h[1];
	return kHaSuccess;
}

int ha_b200_plan_sweep_stats(const HaB200Plan *P, int64_t *sweeps_sum, int32_t *sweeps_max) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P) return kHaErrorArg;
	int32_t h[4] = {0, 0, 0, 0};
	HA_CUDA(cudaMemcpy(h, P->counters.p, sizeof(h), cudaMemcpyDeviceToHost));
	if (sweeps_sum) *sweeps_sum = h[2];
	if (sweeps_max) *sweeps_max = h[3];
	return kHaSuccess;
}

int ha_b200_plan_searchlight_stats(const HaB200Plan *P, int32_t first, int32_t n, double *s_min, double *s_max,
                                   int32_t *flags, int32_t *sweeps) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || P->last_chunk < 0 || n <= 0) return kHaErrorArg;
	const Chunk &ch = P->chunks[(size_t)P->last_chunk];
	if (first < ch.s0 || first + n > ch.s1) return kHaErrorArg;
	std::vector<SlStats> st((size_t)n);
	HA_CUDA(cudaDeviceSynchronize());
	HA_CUDA(cudaMemcpy(st.data(), P->stats.p + (first - ch.s0), (size_t)n * sizeof(SlStats), cudaMemcpyDeviceToHost));
	for (int q = 0; q < n; q++) {
		if (s_min) s_min[q] = st[q].s_min;
		if (s_max) s_max[q] = st[q].s_max;
		if (flags) flags[q] = st[q].flags;
		if (sweeps) sweeps[q] = st[q].sweeps;
	}
	return kHaSuccess;
}

int ha_b200_plan_procrustes_device(HaB200Plan *P, const double *d_X, const double *d_Y, bool isReflection,
                                   bool isScaling, int solver, int out_kind, double *d_values, void *stream) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || !d_X || !d_Y || !d_values) return kHaErrorArg;
	if (solver < 0 || solver > 3 || out_kind < 0 || out_kind > 1) return kHaErrorArg;
	return run_procrustes(P, d_X, d_Y, isReflection, isScaling, solver, out_kind, d_values, (cudaStream_t)stream);
}

int ha_b200_plan_ridge_device(HaB200Plan *P, const double *d_X, const double *d_Y, double alpha, int out_kind,
                              double *d_values, void *stream) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || !d_X || !d_Y || !d_values || out_kind < 0 || out_kind > 1) return kHaErrorArg;
	if (!(alpha >= 0.0)) {
		fprintf(stderr, "ha_b200: ridge alpha must be >= 0\n");
		return kHaErrorArg;
	}
	return run_ridge(P, d_X, d_Y, alpha, out_kind, d_values, (cudaStream_t)stream);
}

int ha_b200_aligned_correlation_device(const double *d_X, const double *d_Y, int32_t nt, int32_t nv,
                                       const int64_t *d_indptr, const int32_t *d_indices, const double *d_values,
                                       int64_t nnz, double *d_r, double *d_aligned, void *stream) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!d_X || !d_Y || !d_r || nt < 1 || nv < 1) return kHaErrorArg;
	if (d_values && (!d_indptr || !d_indices || nnz < 0)) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	cudaStream_t st = (cudaStream_t)stream;
	constexpr int kWarps = 8;  // columns per CTA, one warp each
	const unsigned blocks = (unsigned)(((int64_t)nv + kWarps - 1) / kWarps);
	{
		HA_LAUNCH(kHaB200KEval, st);
		k_aligned_corr<<<blocks, kWarps * 32, 0, st>>>(d_X, d_Y, nt, nv, d_indptr, d_indices, d_values, nnz, d_r,
		                                                d_aligned);
	}
	if (cudaGetLastError() != cudaSuccess) {
		fprintf(stderr, "ha_b200_aligned_correlation_device: launch failed\n");
		return kHaErrorInternal;
	}
	return kHaSuccess;
}

void ha_b200_set_kernel_timing(bool on) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	g_timing = on;
	if (on && (g_time_base || cudaEventCreate(&g_time_base) == cudaSuccess)) cudaEventRecord(g_time_base, 0);
}

int ha_b200_plan_ridge_grid_device(HaB200Plan *P, const double *d_X, const double *d_Y, const double *alphas,
                                   int32_t n_alphas, const int32_t *npcs, int32_t n_npcs,
                                   const int32_t *const *train_idx_li, const int32_t *const *test_idx_li,
                                   const int32_t *train_sizes, const int32_t *test_sizes, int32_t n_models,
                                   int out_kind, double *d_values, int32_t *d_best, double *d_cost, void *stream) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || !d_X || !d_Y || !d_values || !d_best) return kHaErrorArg;
	if (out_kind != kHaB200OutCSR && out_kind != kHaB200OutCSC) return kHaErrorArg;
	GridSpec gs;
	int rc = grid_spec(P->nt, alphas, n_alphas, npcs, n_npcs, train_idx_li, test_idx_li, train_sizes, test_sizes,
	                   n_models, gs);
	if (rc != kHaSuccess) return rc;
	return run_ridge_grid(P, d_X, d_Y, gs, out_kind, d_values, d_best, d_cost, (cudaStream_t)stream);
}

int ha_b200_plan_ridge_features_device(HaB200Plan *P, const double *d_X, const int32_t *rows, int32_t n_rows,
                                       float *d_features, void *stream) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || !d_X || !d_features) return kHaErrorArg;
	return run_ridge_features(P, d_X, rows, n_rows, d_features, (cudaStream_t)stream);
}

int ha_b200_plan_ridge_learned_device(HaB200Plan *P, const double *d_X, const double *d_Y, const int32_t *rows,
                                      int32_t n_rows, const double *alphas, int32_t n_alphas, const int32_t *npcs,
                                      int32_t n_npcs, const float *d_params, float min_prob,
                                      const int32_t *const *train_idx_li, const int32_t *const *test_idx_li,
                                      const int32_t *train_sizes, const int32_t *test_sizes, int32_t n_models,
                                      int out_kind, double *d_values, int32_t *d_choice, float *d_prob, void *stream) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || !d_X || !d_Y || !d_params || !d_values || !d_choice || !d_prob) return kHaErrorArg;
	if (out_kind != kHaB200OutCSR && out_kind != kHaB200OutCSC) return kHaErrorArg;
	GridSpec gs;
	int rc = grid_spec(P->nt, alphas, n_alphas, npcs, n_npcs, train_idx_li, test_idx_li, train_sizes, test_sizes,
	                   n_models, gs);
	if (rc != kHaSuccess) return rc;
	return run_ridge_learned(P, d_X, d_Y, rows, n_rows, gs, d_params, min_prob, out_kind, d_values, d_choice, d_prob,
	                         (cudaStream_t)stream);
}

int64_t ha_b200_mlp_param_count(int32_t n_classes) {
	if (n_classes < 1 || n_classes > kMlpMaxClasses) return -1;
	return MlpLayout::make(n_classes).total;
}

int ha_b200_mlp_init(float *d_params, int32_t n_classes, uint64_t seed) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!d_params) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	if ((rc = mlp_check(n_classes)) != kHaSuccess) return rc;
	const MlpLayout L = MlpLayout::make(n_classes);
	std::vector<float> h((size_t)L.total, 0.0f);
	HostRng g(seed);
	auto fill = [&](int64_t ofs, int fan_in, int64_t count) {
		const double a = 1.0 / std::sqrt((double)fan_in);
		for (int64_t k = 0; k < count; k++) h[(size_t)(ofs + k)] = (float)((2.0 * g.uniform() - 1.0) * a);
	};
	fill(L.W1, kMlpIn, (int64_t)kMlpIn * kMlpHidden);
	fill(L.b1, kMlpIn, kMlpHidden);
	fill(L.W2, kMlpHidden, (int64_t)kMlpHidden * kMlpHidden);
	fill(L.b2, kMlpHidden, kMlpHidden);
	fill(L.W3, kMlpHidden, (int64_t)kMlpHidden * n_classes);
	fill(L.b3, kMlpHidden, n_classes);
	HA_CUDA(cudaMemcpy(d_params, h.data(), (size_t)L.total * 4, cudaMemcpyHostToDevice));
	return kHaSuccess;
}

int ha_b200_mlp_grad(const float *d_params, int32_t n_classes, const float *d_x, const int32_t *d_y, int32_t n,
                     float *d_grad, float *loss_out) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!d_params || !d_x || !d_y || !d_grad || n < 1) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	if ((rc = mlp_check(n_classes)) != kHaSuccess) return rc;
	if ((rc = mlp_labels_ok(d_y, n, n_classes)) != kHaSuccess) return rc;
	const MlpLayout L = MlpLayout::make(n_classes);
	const int nb = (n + kMlpSamples - 1) / kMlpSamples;
	if ((rc = g_mlp.part.ensure((size_t)nb * L.total)) != kHaSuccess) return rc;
	if ((rc = g_mlp.loss.ensure((size_t)nb)) != kHaSuccess) return rc;
	{ HA_LAUNCH(kHaB200KMlp, 0); k_mlp_fwdbwd<<<nb, kBlock, mlp_smem(n_classes)>>>(d_params, n_classes, d_x, d_y, nullptr, n, 1.0f / n, g_mlp.part.p, g_mlp.loss.p); }
	{ HA_LAUNCH(kHaB200KMlp, 0); k_mlp_adam<<<(unsigned)((L.total + 255) / 256), 256>>>(nullptr, g_mlp.part.p, nb, L.total, nullptr, nullptr, 0.f, 0.f, 0.f, 0.f, 1.f, 1.f, d_grad); }
	HA_CUDA(cudaGetLastError());
	if (loss_out) {
		std::vector<float> lp((size_t)nb);
		HA_CUDA(cudaMemcpy(lp.data(), g_mlp.loss.p, (size_t)nb * 4, cudaMemcpyDeviceToHost));
		double a = 0.0;
		for (float x : lp) a += x;
		*loss_out = (float)(a / n);
	}
	HA_CUDA(cudaDeviceSynchronize());
	return kHaSuccess;
}

int ha_b200_mlp_train(float *d_params, int32_t n_classes, const float *d_x, const int32_t *d_y, int32_t n,
                      int32_t epochs, int32_t batch, float lr, uint64_t seed, float *final_loss) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!d_params || !d_x || !d_y || n < 1 || epochs < 0 || batch < 1 || !(lr > 0.0f)) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	if ((rc = mlp_check(n_classes)) != kHaSuccess) return rc;
	if ((rc = mlp_labels_ok(d_y, n, n_classes)) != kHaSuccess) return rc;
	const MlpLayout L = MlpLayout::make(n_classes);
	batch = std::min(batch, n);
	const int nbmax = (batch + kMlpSamples - 1) / kMlpSamples;
	if ((rc = g_mlp.part.ensure((size_t)nbmax * L.total)) != kHaSuccess) return rc;
	if ((rc = g_mlp.loss.ensure((size_t)nbmax)) != kHaSuccess) return rc;
	if ((rc = g_mlp.m.ensure((size_t)L.total)) != kHaSuccess) return rc;
	if ((rc = g_mlp.v.ensure((size_t)L.total)) != kHaSuccess) return rc;
	if ((rc = g_mlp.idx.ensure((size_t)n)) != kHaSuccess) return rc;
	HA_CUDA(cudaMemset(g_mlp.m.p, 0, (size_t)L.total * 4));
	HA_CUDA(cudaMemset(g_mlp.v.p, 0, (size_t)L.total * 4));
	const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
	HostRng g(seed);
	std::vector<int32_t> perm((size_t)n);
	int64_t step = 0;
	const unsigned pg = (unsigned)((L.total + 255) / 256);
	for (int ep = 0; ep < epochs; ep++) {
		for (int i = 0; i < n; i++) perm[i] = i;
		for (int i = n - 1; i > 0; i--) std::swap(perm[i], perm[(int)(g.next() % (uint64_t)(i + 1))]);
		HA_CUDA(cudaMemcpy(g_mlp.idx.p, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice));
		for (int b0 = 0; b0 < n; b0 += batch) {
			const int nbt = std::min(batch, n - b0);
			const int nb = (nbt + kMlpSamples - 1) / kMlpSamples;
			step++;
			const float bc1 = 1.0f - (float)std::pow((double)b1, (double)step);
			const float bc2 = 1.0f - (float)std::pow((double)b2, (double)step);
			{ HA_LAUNCH(kHaB200KMlp, 0); k_mlp_fwdbwd<<<nb, kBlock, mlp_smem(n_classes)>>>(d_params, n_classes, d_x, d_y, g_mlp.idx.p + b0, nbt, 1.0f / nbt, g_mlp.part.p, g_mlp.loss.p); }
			{ HA_LAUNCH(kHaB200KMlp, 0); k_mlp_adam<<<pg, 256>>>(d_params, g_mlp.part.p, nb, L.total, g_mlp.m.p, g_mlp.v.p, lr, b1, b2, eps, bc1, bc2, nullptr); }
		}
		HA_CUDA(cudaGetLastError());
	}
	HA_CUDA(cudaDeviceSynchronize());
	if (final_loss) {
		DevArr<float> gr;
		if ((rc = gr.ensure((size_t)L.total)) != kHaSuccess) return rc;
		rc = ha_b200_mlp_grad(d_params, n_classes, d_x, d_y, n, gr.p, final_loss);
		gr.release();
		return rc;
	}
	return kHaSuccess;
}

int ha_b200_mlp_infer(const float *d_params, int32_t n_classes, const float *d_x, int32_t n, int32_t *d_class,
                      float *d_prob, void *stream) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!d_params || !d_x || !d_class || !d_prob || n < 0) return kHaErrorArg;
	if (n == 0) return kHaSuccess;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	if ((rc = mlp_check(n_classes)) != kHaSuccess) return rc;
	const cudaStream_t st = (cudaStream_t)stream;
	const MlpLayout L = MlpLayout::make(n_classes);
	if ((rc = g_mlp.pbf.ensure((size_t)L.total)) != kHaSuccess) return rc;
	{ HA_LAUNCH(kHaB200KMlp, st); k_f32_to_bf16<<<(unsigned)((L.total + 255) / 256), 256, 0, st>>>(d_params, g_mlp.pbf.p, L.total); }
	{ HA_LAUNCH(kHaB200KMlp, st); k_mlp_infer<<<(n + kMlpSamples - 1) / kMlpSamples, kBlock, mlp_smem(n_classes), st>>>(g_mlp.pbf.p, n_classes, d_x, n, d_class, d_prob); }
	HA_CUDA(cudaGetLastError());
	return kHaSuccess;
}

int ha_b200_kernel_times(double *ms, int64_t *launches) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	// per kind: the union of the launch intervals (launches of one kind on different side streams
	// overlap; for serial launches the union is the sum of the durations)
	std::vector<std::vector<std::pair<float, float>>> iv(kHaB200NumKernelKinds);
	for (auto &t : g_timed) {
		float a = 0.0f, b = 0.0f;
		if (cudaEventSynchronize(t.b) == cudaSuccess) {
			if (g_time_base && cudaEventElapsedTime(&a, g_time_base, t.a) == cudaSuccess &&
			    cudaEventElapsedTime(&b, g_time_base, t.b) == cudaSuccess)
				iv[t.kind].push_back({a, b});
			else if (cudaEventElapsedTime(&b, t.a, t.b) == cudaSuccess)
				g_kernel_ms[t.kind] += b;
		}
		cudaEventDestroy(t.a);
		cudaEventDestroy(t.b);
	}
	g_timed.clear();
	for (int k = 0; k < kHaB200NumKernelKinds; k++) {
		auto &v = iv[k];
		std::sort(v.begin(), v.end());
		double lo = 0.0, hi = -1.0;
		for (auto &x : v) {
			if (x.first > hi) {
				if (hi > lo) g_kernel_ms[k] += hi - lo;
				lo = x.first;
				hi = x.second;
			} else if (x.second > hi) {
				hi = x.second;
			}
		}
		if (hi > lo) g_kernel_ms[k] += hi - lo;
	}
	if (g_time_base) cudaEventRecord(g_time_base, 0);
	for (int k = 0; k < kHaB200NumKernelKinds; k++) {
		if (ms) ms[k] = g_kernel_ms[k];
		if (launches) launches[k] = g_kernel_n[k];
		g_kernel_ms[k] = 0.0;
		g_kernel_n[k] = 0;
	}
	cudaGetLastError();
	return kHaSuccess;
}

int64_t ha_b200_launch_count(void) { return g_launches; }

void ha_b200_set_graphs(bool on) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	g_graphs = on ? 1 : 0;
}

int ha_b200_plan_set_grid_precision(HaB200Plan *P, int32_t bits) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || (bits != 32 && bits != 64)) return kHaErrorArg;
	P->grid_bits = bits;
	return kHaSuccess;
}

int ha_b200_plan_tc_layout(const HaB200Plan *P, int32_t *smem_kb, int32_t *tuned, double *cand_ms) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P) return kHaErrorArg;
	for (int c = 0; c < 2; c++) {
		if (smem_kb) smem_kb[c] = P->tc_smem[c] / 1024;
		if (cand_ms)
			for (int i = 0; i < 3; i++) cand_ms[3 * c + i] = P->tc_tune_ms[c][i];
	}
	if (tuned) *tuned = P->tc_tuned ? 1 : 0;
	return kHaSuccess;
}

int ha_b200_plan_set_tc_layout(HaB200Plan *P, const int32_t *smem_kb) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || !smem_kb) return kHaErrorArg;
	for (int c = 0; c < 2; c++) {
		bool ok = false;
		for (int i = 0; i < 3; i++) ok = ok || (kTcCand[c][i] && smem_kb[c] * 1024 == kTcCand[c][i]);
		if (!ok) {
			fprintf(stderr, "ha_b200_plan_set_tc_layout: %d KB is not a layout of size class %d\n", smem_kb[c], c);
			return kHaErrorArg;
		}
	}
	for (int c = 0; c < 2; c++) P->tc_smem[c] = smem_kb[c] * 1024;
	P->tc_tuned = true;
	return kHaSuccess;
}

int ha_b200_tc_selftest(int32_t which, int32_t n, int32_t nt, const float *h_a, const float *h_b, float *h_out) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!h_a || !h_out || n <= 0 || n > kTcMaxNp || which < 0 || which > 2) return kHaErrorArg;
	if (which != 0 && !h_b) return kHaErrorArg;
	if (which == 2 && nt <= 0) return kHaErrorArg;
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	if ((rc = set_tc_attrs()) != kHaSuccess) return rc;
	const int np = (n + 15) & ~15;
	const int ntp = (nt + 15) & ~15;
	const int64_t pe3 = 3 * (int64_t)np * np;
	DevArr<__nv_bfloat16> Xp, Pp, Xb, Yb;
	DevArr<float> A32, T, R, in0, in1;
	DevArr<double> d0, d1;
	DevArr<TcWork> dw;
	DevArr<TcTile> dt;
	DevArr<TcState> dst;
	DevArr<int32_t> sl, err;
	auto release_all = [&]() {
		Xp.release(); Pp.release(); Xb.release(); Yb.release(); A32.release(); T.release(); R.release();
		in0.release(); in1.release(); d0.release(); d1.release(); dw.release(); dt.release(); dst.release();
		sl.release(); err.release();
	};
	if (Xp.ensure(pe3) || Pp.ensure(pe3) || A32.ensure((size_t)np * np) || T.ensure((size_t)n * n) ||
	    R.ensure(kTcResSlots) || dw.ensure(1) || dt.ensure(2 * kTcMaxNp / 128) || dst.ensure(2) || sl.ensure(n) ||
	    err.ensure(1)) {
		release_all();
		return kHaErrorAlloc;
	}
	TcWork w = {};
	w.n = n;
	w.np = np;
	std::vector<TcTile> tiles;
	const int h0 = np > 256 ? ((np / 2 + 15) & ~15) : np;
	for (int t = 0; t * 128 < np; t++) {
		tiles.push_back({0, t, 0, h0});
		if (h0 < np) tiles.push_back({0, t, h0, np - h0});
	}
	std::vector<int32_t> hs((size_t)n);
	for (int i = 0; i < n; i++) hs[i] = i;
	cudaStream_t st = 0;
	rc = kHaSuccess;
	do {
		if (cudaMemcpy(dw.p, &w, sizeof(w), cudaMemcpyHostToDevice) != cudaSuccess ||
		    cudaMemcpy(dt.p, tiles.data(), tiles.size() * sizeof(TcTile), cudaMemcpyHostToDevice) != cudaSuccess ||
		    cudaMemcpy(sl.p, hs.data(), (size_t)n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
		    cudaMemset(dst.p, 0, 2 * sizeof(TcState)) != cudaSuccess ||
		    cudaMemset(R.p, 0, kTcResSlots * sizeof(float)) != cudaSuccess ||
		    cudaMemset(err.p, 0, sizeof(int32_t)) != cudaSuccess) {
			rc = kHaErrorInternal;
			break;
		}
		TcArgs a = {};
		a.work = dw.p;
		a.tiles = dt.p;
		a.Xp = Xp.p;
		a.Xw = Xp.p;
		a.Pp = Pp.p;
		a.A32 = A32.p;
		a.T = T.p;
		a.t_rowmajor = 1;
		a.st_in = dst.p;
		a.st_out = dst.p + 1;
		a.res_part = R.p;
		a.smem_bytes = kTcSmemSmall;
		a.err = err.p;
		const int grid = (int)tiles.size();
		if (which == 2) {
			const int64_t vplane = (int64_t)n * ntp;
			if (Xb.ensure(3 * vplane) || Yb.ensure(3 * vplane) || d0.ensure((size_t)n * nt) || d1.ensure((size_t)n * nt)) {
				rc = kHaErrorAlloc;
				break;
			}
			std::vector<double> hx((size_t)n * nt), hy((size_t)n * nt);
			for (size_t i = 0; i < hx.size(); i++) { hx[i] = h_a[i]; hy[i] = h_b[i]; }
			if (cudaMemcpy(d0.p, hx.data(), hx.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
			    cudaMemcpy(d1.p, hy.data(), hy.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
				rc = kHaErrorInternal;
				break;
			}
			k_split3_vertex_major<<<64, kBlock, 0, st>>>(d0.p, nt, n, ntp, Xb.p);
			k_split3_vertex_major<<<64, kBlock, 0, st>>>(d1.p, nt, n, ntp, Yb.p);
			a.Xb = Xb.p; a.Yb = Yb.p; a.vplane = vplane; a.ntp = ntp; a.sl_idx = sl.p;
			{ HA_LAUNCH(kHaB200KTcXcov, st); k_tc_gemm<kTcPhaseXcov><<<grid, kTcThreads, a.smem_bytes, st>>>(a); }
			std::vector<float> full((size_t)np * np);
			if (cudaGetLastError() != cudaSuccess ||
			    cudaMemcpy(full.data(), A32.p, full.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
				rc = kHaErrorInternal;
				break;
			}
			for (int r = 0; r < n; r++)
				for (int c = 0; c < n; c++) h_out[(size_t)r * n + c] = full[(size_t)r * np + c];
		} else {
			if (in0.ensure((size_t)n * n) || in1.ensure((size_t)n * n)) {
				rc = kHaErrorAlloc;
				break;
			}
			if (cudaMemcpy(in0.p, h_a, (size_t)n * n * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
				rc = kHaErrorInternal;
				break;
			}
			k_tc_pack<<<64, kBlock, 0, st>>>(in0.p, n, np, Xp.p);
			if (which == 0) {
				a.c1 = 0.f;
				a.c3 = 1.f;  // P = X^T X
				{ HA_LAUNCH(kHaB200KTcNs, st); launch_tc_tiles<kTcPhaseGram>(grid, a, st, 256, tc_iter_from() == 0); }
				k_tc_unpack<<<64, kBlock, 0, st>>>(Pp.p, n, np, T.p);
			} else {
				if (cudaMemcpy(in1.p, h_b, (size_t)n * n * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
					rc = kHaErrorInternal;
					break;
				}
				k_tc_pack<<<64, kBlock, 0, st>>>(in1.p, n, np, Pp.p);
				a.plain = 1;
				a.tol_stop = 1e30f;  // residual 0 < tol: the update is final and writes T = X P
				{ HA_LAUNCH(kHaB200KTcNs, st); launch_tc_tiles<kTcPhaseUpdate>(grid, a, st, 256, tc_iter_from() == 0); }
			}
			if (cudaGetLastError() != cudaSuccess ||
			    cudaMemcpy(h_out, T.p, (size_t)n * n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
				rc = kHaErrorInternal;
				break;
			}
		}
		int32_t e = 0;
		if (cudaMemcpy(&e, err.p, 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
			rc = kHaErrorInternal;
			break;
		}
		if (e) {
			fprintf(stderr, "ha_b200: tensor-core self-test: a pipeline wait timed out\n");
			rc = kHaErrorInternal;
		}
	} while (false);
	if (rc == kHaErrorInternal) fprintf(stderr, "ha_b200: tensor-core self-test failed: %s\n", cudaGetErrorString(cudaGetLastError()));
	release_all();
	return rc;
}


int ha_b200_plan_local_transforms(const HaB200Plan *P, int32_t first, int32_t n, float *out) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!P || !out || P->last_chunk < 0) return kHaErrorArg;
	const Chunk &ch = P->chunks[(size_t)P->last_chunk];
	if (first < ch.s0 || first + n > ch.s1 || n <= 0) return kHaErrorArg;
	int64_t a = ch.tofs[(size_t)(first - ch.s0)];
	int64_t e = (first + n < ch.s1) ? ch.tofs[(size_t)(first + n - ch.s0)] : ch.t_elems;
	HA_CUDA(cudaDeviceSynchronize());
	HA_CUDA(cudaMemcpy(out, P->scrT.p + a, (size_t)(e - a) * 4, cudaMemcpyDeviceToHost));
	return kHaSuccess;
}

}  // extern "C"

// =============================================================================================
// Local Procrustes without allocation
// =============================================================================================
//
// Some callers cannot call cudaMalloc: applications whose own pool allocator has already
// reserved the GPU's memory and hands out nothing else, plugins whose host program forbids
// them to create device allocations, and loops where the device-wide synchronisation of
// cudaMalloc/cudaFree is not acceptable.  For them this entry point computes the local
// transforms of searchlights of up to kNoAllocMaxN vertices from buffers the caller already
// owns, using as scratch only the file-scope device array below.  That array is part of the
// library image: every GPU that loads the library holds it until the process exits.

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)64 << 20;  // 64 MiB
constexpr int kNoAllocMaxN = 160;                          // largest searchlight (resident FP32 Jacobi)
constexpr int kNoAllocMaxBatch = 2048;                     // searchlights per launch
constexpr int kNoAllocMaxDevices = 64;

// Scratch of every call: [status word | work items | solve records | u/v pairs | A matrices].
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr size_t kNaStatusOfs = 0;
constexpr size_t kNaWorkOfs = 256;
constexpr size_t kNaStatsOfs = kNaWorkOfs + (((size_t)kNoAllocMaxBatch * sizeof(SlWork) + 255) & ~(size_t)255);
constexpr size_t kNaUvOfs = kNaStatsOfs + (((size_t)kNoAllocMaxBatch * sizeof(SlStats) + 255) & ~(size_t)255);
constexpr size_t kNaAOfs = kNaUvOfs + (((size_t)kNoAllocMaxBatch * 2 * kNoAllocMaxN * sizeof(double) + 255) & ~(size_t)255);
constexpr size_t kNaAFloats = (kNoAllocScratchBytes - kNaAOfs) / sizeof(float);
static_assert(kNaAOfs < kNoAllocScratchBytes, "no-alloc scratch layout");

// Device address of g_noalloc_scratch per device (host code may not use the symbol itself).
unsigned char *g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};
SlWork g_noalloc_items[kNoAllocMaxBatch];  // host staging of one batch's work items
int32_t g_noalloc_status_host = 0;

// Cross-covariance from float64 vertex-major inputs, rounded to float32 on load (the same
// tiling and summation order as k_xcov<float>).  Indices outside [0, nv) are read as zero
// columns and reported through *status.
template <int KT>
__global__ void __launch_bounds__(256) k_xcov_f64in(const SlWork *__restrict__ work, const int32_t *__restrict__ sl_idx,
                                                    const double *__restrict__ X, const double *__restrict__ Y, int nt,
                                                    int nv, float *__restrict__ Ascr, int32_t *__restrict__ status) {
	const SlWork w = work[blockIdx.x];
	const int n = w.n;
	const int ncol = w.nblk * w.bsz;
	const int32_t *sl = sl_idx + w.sofs;
	float *A = Ascr + w.aofs;
	__shared__ float xs[KT][64 + 1];
	__shared__ float ys[KT][64 + 1];
	__shared__ int32_t vi[64], vj[64];
	const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
	for (int i0 = 0; i0 < n; i0 += 64) {
		for (int j0 = 0; j0 < n; j0 += 64) {
			__syncthreads();
			if (threadIdx.x < 128) {
				const int r = threadIdx.x & 63;
				const int idx = (threadIdx.x < 64 ? i0 : j0) + r;
				int v = -1;
				if (idx < n) {
					v = sl[idx];
					if (v < 0 || v >= nv) {
						atomicOr(status, 1);
						v = -1;
					}
				}
				if (threadIdx.x < 64) vi[r] = v; else vj[r] = v;
			}
			float acc[4][4];
#pragma unroll
			for (int a = 0; a < 4; a++)
#pragma unroll
				for (int b = 0; b < 4; b++) acc[a][b] = 0.0f;
			for (int t0 = 0; t0 < nt; t0 += KT) {
				__syncthreads();
				for (int e = threadIdx.x; e < 64 * KT; e += 256) {
					const int r = e / KT, t = e - r * KT;
					const int tt = t0 + t;
					const int v = vi[r], u = vj[r];
					xs[t][r] = (v >= 0 && tt < nt) ? (float)X[(int64_t)v * nt + tt] : 0.0f;
					ys[t][r] = (u >= 0 && tt < nt) ? (float)Y[(int64_t)u * nt + tt] : 0.0f;
				}
				__syncthreads();
#pragma unroll 4
				for (int t = 0; t < KT; t++) {
					float a[4], b[4];
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
	for (int64_t e = (int64_t)n * n + threadIdx.x; e < (int64_t)n * ncol; e += 256) A[e] = 0.0f;
}

// Once per device, with that device current: find the scratch array's device address and
// raise the shared-memory limit of the kernels used below.
int noalloc_setup(int dev, unsigned char **out) {
	if (dev < 0 || dev >= kNoAllocMaxDevices) {
		fprintf(stderr, "ha_b200_local_procrustes_noalloc: device %d out of range\n", dev);
		return kHaErrorInternal;
	}
	if (!g_noalloc_ptr[dev]) {
		void *p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || !p) {
			fprintf(stderr, "ha_b200_local_procrustes_noalloc: cudaGetSymbolAddress failed: %s\n",
			        cudaGetErrorString(e));
			cudaGetLastError();
			return kHaErrorInternal;
		}
		if (set_jacobi_attrs<float>() != kHaSuccess) {
			fprintf(stderr, "ha_b200_local_procrustes_noalloc: cudaFuncSetAttribute failed\n");
			return kHaErrorInternal;
		}
		g_noalloc_ptr[dev] = (unsigned char *)p;
	}
	*out = g_noalloc_ptr[dev];
	return kHaSuccess;
}

}  // namespace

extern "C" int ha_b200_local_procrustes_noalloc(const double *d_X, const double *d_Y, int32_t nt, int32_t nv,
                                                const int32_t *d_sl_indices, const int32_t *sl_offsets,
                                                int32_t count, float *d_T_out, void *stream) {
	std::lock_guard<std::recursive_mutex> lk(g_mu);
	if (!d_X || !d_Y || !d_sl_indices || !sl_offsets || !d_T_out || nt <= 0 || nv <= 0 || count <= 0)
		return kHaErrorArg;
	if (sl_offsets[0] != 0) {
		fprintf(stderr, "ha_b200_local_procrustes_noalloc: sl_offsets[0] must be 0\n");
		return kHaErrorArg;
	}
	for (int32_t s = 0; s < count; s++) {
		const int32_t n = sl_offsets[s + 1] - sl_offsets[s];
		if (n < 1 || n > kNoAllocMaxN) {
			fprintf(stderr,
			        "ha_b200_local_procrustes_noalloc: searchlight %d has %d vertices; this entry point "
			        "supports 1 to %d (use ha_b200_plan_procrustes_device for larger ones)\n",
			        s, n, kNoAllocMaxN);
			return kHaErrorArg;
		}
	}
	int rc = check_cuda_ready();
	if (rc != kHaSuccess) return rc;
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return kHaErrorInternal;
	unsigned char *base = nullptr;
	if ((rc = noalloc_setup(dev, &base)) != kHaSuccess) return rc;
	cudaStream_t st = (cudaStream_t)stream;
	int32_t *d_status = reinterpret_cast<int32_t *>(base + kNaStatusOfs);
	SlWork *d_work = reinterpret_cast<SlWork *>(base + kNaWorkOfs);
	SlStats *d_stats = reinterpret_cast<SlStats *>(base + kNaStatsOfs);
	double *d_uv = reinterpret_cast<double *>(base + kNaUvOfs);
	float *d_A = reinterpret_cast<float *>(base + kNaAOfs);
	// the array keeps the previous call's contents: clear the status word and the solve records
	HA_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int32_t), st));

	JacobiParams jp;
	jp.max_sweeps = 40;
	jp.t_rowmajor = 1;
	jp.ill_ratio = 0.0;
	jp.weak = 1000.0;
	jp.eig = 0;
	jp.only_flagged = 0;
	jp.keep_v = 0;
	jp.warm = 0;
	jp.stop_cos = 0.0;
	int64_t tofs = 0;  // packed output offset of the current searchlight
	int32_t s = 0;
	// an error after work was queued: wait for that work before returning, so no later call finds
	// the shared array still in use
	auto fail_after_enqueue = [&](int code, const char *what) {
		fprintf(stderr, "ha_b200_local_procrustes_noalloc: %s failed: %s\n", what, cudaGetErrorString(cudaGetLastError()));
		cudaStreamSynchronize(st);
		cudaGetLastError();
		return code;
	};
	while (s < count) {
		// one batch: as many searchlights as fit the work-item and A areas
		int nb = 0;
		int64_t a_used = 0, uv_used = 0;
		while (s + nb < count && nb < kNoAllocMaxBatch) {
			const int32_t n = sl_offsets[s + nb + 1] - sl_offsets[s + nb];
			int bsz, nblk;
			size_t smem;
			jacobi_layout(n, false, bsz, nblk, smem);
			const int64_t need = ((int64_t)n * nblk * bsz + 63) & ~(int64_t)63;
			if (a_used + need > (int64_t)kNaAFloats) break;
			SlWork &w = g_noalloc_items[nb];
			w.s = s + nb;
			w.n = n;
			w.bsz = bsz;
			w.nblk = nblk;
			w.aofs = a_used;
			w.tofs = tofs;
			w.sofs = sl_offsets[s + nb];
			w.slot = nb;
			w.uvofs = uv_used;
			a_used += need;
			uv_used += 2 * (int64_t)n;
			tofs += (int64_t)n * n;
			nb++;
		}
		if (cudaMemcpyAsync(d_work, g_noalloc_items, (size_t)nb * sizeof(SlWork), cudaMemcpyHostToDevice, st) != cudaSuccess ||
		    cudaMemsetAsync(d_stats, 0, (size_t)nb * sizeof(SlStats), st) != cudaSuccess)
			return fail_after_enqueue(kHaErrorInternal, "staging a batch");
		// one launch per rows-per-lane group (items of a batch are in searchlight order)
		k_xcov_f64in<32><<<nb, kBlock, 0, st>>>(d_work, d_sl_indices, d_X, d_Y, nt, nv, d_A, d_status);
		if (cudaGetLastError() != cudaSuccess) return fail_after_enqueue(kHaErrorInternal, "the cross-covariance launch");
		int q = 0;
		while (q < nb) {
			const int rpl = rpl_for(g_noalloc_items[q].n);
			int e = q, maxb = 0;
			size_t smem = 0;
			while (e < nb && rpl_for(g_noalloc_items[e].n) == rpl) {
				int bsz, nblk;
				size_t sm;
				jacobi_layout(g_noalloc_items[e].n, false, bsz, nblk, sm);
				smem = std::max(smem, sm);
				maxb = std::max(maxb, bsz);
				e++;
			}
			if ((rc = launch_jacobi<float>(rpl, e - q, jacobi_threads(maxb, false), smem, st, d_work + q, d_A, d_A,
			                               d_T_out, d_stats, d_uv, jp)) != kHaSuccess)
				return fail_after_enqueue(rc, "the Jacobi launch");
			if (cudaGetLastError() != cudaSuccess) return fail_after_enqueue(kHaErrorInternal, "the Jacobi launch");
			q = e;
		}
		// the next batch reuses the scratch: finish this one before its items are overwritten
		if (cudaStreamSynchronize(st) != cudaSuccess) return fail_after_enqueue(kHaErrorInternal, "a batch");
		s += nb;
	}
	HA_CUDA(cudaMemcpyAsync(&g_noalloc_status_host, d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
	HA_CUDA(cudaStreamSynchronize(st));
	if (g_noalloc_status_host != 0) {
		fprintf(stderr, "ha_b200_local_procrustes_noalloc: a searchlight index is outside [0, %d)\n", nv);
		return kHaErrorArg;
	}
	return kHaSuccess;
}
