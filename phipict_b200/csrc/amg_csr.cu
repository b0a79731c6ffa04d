// AMG-preconditioned CG on CSR matrices: the backend function AMGPCGSolve of phiPICT
// (bindings.cpp:764-776, solvers/krylov/krylov.cu:1248-1612), for callers that bring their own
// algebraic hierarchy (phiPICT's solvers/amg.py builds one with pyamg). The PISO step itself
// does not use it: its pressure and potential solves run the structured multigrid of
// phb_amg.cuh.
//
// The method follows the reference: on each level a damped Jacobi sweep from zero
// (x = w D^-1 b) and pre-1 more sweeps, the residual restricted with R, the coarsest level
// solved with a dense (pseudo-)inverse (one shared or one per environment), the correction
// prolongated with P and post sweeps of the smoother; with projectConstant the right-hand side
// and the preconditioned residual are kept mean-free per environment (singular systems). CG
// stops per environment on ||r||_2 (/ sqrt(n) when normalized) below its tolerance.
// Environments share the sparsity pattern; the system and level operators may carry one set
// of values per environment. Dot products are block partial sums reduced in a fixed order, so
// a solve is deterministic. The host drives the iteration and reads the scalars of every
// iteration: these solves are not on the step's hot path, which runs the persistent solvers.
#include <cmath>
#include <vector>
#include <algorithm>
#include "phb_device.cuh"
#include "phb_launch.cuh"

namespace phb {
namespace csrpcg {

constexpr int BLK = 256;

template <typename V>
struct Csr {
	const int32_t *row, *col;
	const V *val;
	int64_t valStride; // values per environment (0: shared)
	int n;             // rows
};

template <typename V, typename X>
__device__ __forceinline__ double rowDot(const Csr<V> &A, int env, int i, const X *x) {
	const V *v = A.val + env * A.valStride;
	double s = 0;
	for (int k = A.row[i]; k < A.row[i + 1]; ++k) s += double(v[k]) * double(x[A.col[k]]);
	return s;
}

// x = w D^-1 (b - shift)
template <typename H, typename TB>
__global__ void kPre(int n, int64_t dStride, const H *dinv, const TB *b, const double *shift, H *x, double w, const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	const H *dv = dinv + e * dStride;
	const double sh = shift ? shift[e] : 0.0;
	for (int i = blockIdx.x * BLK + threadIdx.x; i < n; i += gridDim.x * BLK)
		x[(int64_t)e * n + i] = H(w * double(dv[i]) * (double(b[(int64_t)e * n + i]) - sh));
}
// res = b - shift - A x
template <typename H, typename TB>
__global__ void kRes(Csr<H> A, const TB *b, const double *shift, const H *x, H *res, const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	const int n = A.n;
	const double sh = shift ? shift[e] : 0.0;
	for (int i = blockIdx.x * BLK + threadIdx.x; i < n; i += gridDim.x * BLK)
		res[(int64_t)e * n + i] = H(double(b[(int64_t)e * n + i]) - sh - rowDot(A, e, i, x + (int64_t)e * n));
}
// out = x + w D^-1 (b - shift - A x)
template <typename H, typename TB, typename TO>
__global__ void kJac(Csr<H> A, int64_t dStride, const H *dinv, const TB *b, const double *shift, const H *x, TO *out, double w,
		const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	const int n = A.n;
	const H *dv = dinv + e * dStride;
	const double sh = shift ? shift[e] : 0.0;
	for (int i = blockIdx.x * BLK + threadIdx.x; i < n; i += gridDim.x * BLK) {
		const int64_t o = (int64_t)e * n + i;
		out[o] = TO(double(x[o]) + w * double(dv[i]) * (double(b[o]) - sh - rowDot(A, e, i, x + (int64_t)e * n)));
	}
}
// out (+)= M in, M rectangular with shared values (M.n rows, nIn columns)
template <typename H>
__global__ void kRect(Csr<H> M, const H *in, int nIn, H *out, int acc, const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	for (int i = blockIdx.x * BLK + threadIdx.x; i < M.n; i += gridDim.x * BLK) {
		const double s = rowDot(M, 0, i, in + (int64_t)e * nIn);
		const int64_t o = (int64_t)e * M.n + i;
		out[o] = acc ? H(double(out[o]) + s) : H(s);
	}
}
// x = pinv b on the coarsest level
template <typename H>
__global__ void kCoarse(const H *pinv, int nc, int batched, const H *b, H *x, const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	const H *pe = pinv + (batched ? (int64_t)e * nc * nc : 0);
	for (int i = blockIdx.x * BLK + threadIdx.x; i < nc; i += gridDim.x * BLK) {
		double s = 0;
		for (int j = 0; j < nc; ++j) s += double(pe[(int64_t)i * nc + j]) * double(b[(int64_t)e * nc + j]);
		x[(int64_t)e * nc + i] = H(s);
	}
}
// block partial sums of a.b and c.d (c may be null) per environment: partial[e][blk][2]
template <typename T>
__global__ void kDots(int n, const T *a, const T *b, const T *c, const T *d, double *partial, const int *active) {
	const int e = blockIdx.y;
	__shared__ double s0[BLK], s1[BLK];
	double v0 = 0, v1 = 0;
	if (active[e]) {
		for (int i = blockIdx.x * BLK + threadIdx.x; i < n; i += gridDim.x * BLK) {
			const int64_t o = (int64_t)e * n + i;
			v0 += double(a[o]) * (b ? double(b[o]) : 1.0);
			if (c) v1 += double(c[o]) * double(d[o]);
		}
	}
	s0[threadIdx.x] = v0;
	s1[threadIdx.x] = v1;
	__syncthreads();
	for (int h = BLK / 2; h > 0; h >>= 1) {
		if ((int)threadIdx.x < h) { s0[threadIdx.x] += s0[threadIdx.x + h]; s1[threadIdx.x] += s1[threadIdx.x + h]; }
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		partial[((int64_t)e * gridDim.x + blockIdx.x) * 2] = s0[0];
		partial[((int64_t)e * gridDim.x + blockIdx.x) * 2 + 1] = s1[0];
	}
}
// fixed-order sums of the block partials: out[e][2]; with `mean`, out[e][0] /= n as well
__global__ void kSum(const double *partial, int nblk, int B, double *out, int n, int mean) {
	const int e = blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= B) return;
	double a = 0, b = 0;
	for (int k = 0; k < nblk; ++k) { a += partial[((int64_t)e * nblk + k) * 2]; b += partial[((int64_t)e * nblk + k) * 2 + 1]; }
	out[e * 2] = mean ? a / double(n) : a;
	out[e * 2 + 1] = b;
}
template <typename T>
__global__ void kSubMean(int n, T *v, const double *sums, const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	const double m = sums[e * 2];
	for (int i = blockIdx.x * BLK + threadIdx.x; i < n; i += gridDim.x * BLK) v[(int64_t)e * n + i] = T(double(v[(int64_t)e * n + i]) - m);
}
template <typename T>
__global__ void kSpmv(Csr<T> A, const T *p, T *q, const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	for (int i = blockIdx.x * BLK + threadIdx.x; i < A.n; i += gridDim.x * BLK)
		q[(int64_t)e * A.n + i] = T(rowDot(A, e, i, p + (int64_t)e * A.n));
}
template <typename T>
__global__ void kResid(Csr<T> A, const T *b, const T *x, T *r, const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	for (int i = blockIdx.x * BLK + threadIdx.x; i < A.n; i += gridDim.x * BLK) {
		const int64_t o = (int64_t)e * A.n + i;
		r[o] = T(double(b[o]) - rowDot(A, e, i, x + (int64_t)e * A.n));
	}
}
// p = z + beta p (beta per environment: coef[e][0])
template <typename T>
__global__ void kDir(int n, const T *z, T *p, const double *coef, const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	const double bt = coef[e * 2];
	for (int i = blockIdx.x * BLK + threadIdx.x; i < n; i += gridDim.x * BLK) {
		const int64_t o = (int64_t)e * n + i;
		p[o] = T(double(z[o]) + bt * double(p[o]));
	}
}
// x += alpha p, r -= alpha q (alpha per environment: coef[e][1])
template <typename T>
__global__ void kUpd(int n, T *x, T *r, const T *p, const T *q, const double *coef, const int *active) {
	const int e = blockIdx.y;
	if (!active[e]) return;
	const double a = coef[e * 2 + 1];
	for (int i = blockIdx.x * BLK + threadIdx.x; i < n; i += gridDim.x * BLK) {
		const int64_t o = (int64_t)e * n + i;
		x[o] = T(double(x[o]) + a * double(p[o]));
		r[o] = T(double(r[o]) - a * double(q[o]));
	}
}

} // namespace csrpcg
} // namespace phb

using namespace phb::csrpcg;

namespace {

// outcomes, as phb_solve_result::status
enum { CONV = 1, NONFIN = 2, MAXITS = 3, RISE = 4 };
constexpr int RISING_LIMIT = 100; // successive non-decreasing residuals that end a best-result solve

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// the workspace carve-up; with base == nullptr only the total is computed
template <typename T, typename H>
struct Work {
	std::vector<H *> lx, ly, lres, lb;
	H *cx = nullptr;
	T *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *bw = nullptr, *xbest = nullptr;
	double *partial = nullptr, *sums = nullptr, *coef = nullptr;
	int *active = nullptr;
	size_t total = 0;
	Work(const phb_csr_pcg *a, int G, char *base) {
		const int L = a->nlevels, B = a->nenv;
		auto take = [&](size_t bytes) { void *p = base ? base + total : nullptr; total += align256(bytes); return p; };
		lx.resize(L); ly.resize(L); lres.resize(L); lb.resize(L + 1);
		for (int l = 0; l < L; ++l) {
			const size_t m = (size_t)a->levels[l].n * B * sizeof(H);
			lx[l] = (H *)take(m); ly[l] = (H *)take(m); lres[l] = (H *)take(m); lb[l] = (H *)take(m);
		}
		lb[L] = (H *)take((size_t)a->coarse_n * B * sizeof(H));
		cx = (H *)take((size_t)a->coarse_n * B * sizeof(H));
		const size_t vm = (size_t)a->n * B * sizeof(T);
		r = (T *)take(vm); z = (T *)take(vm); p = (T *)take(vm); q = (T *)take(vm); bw = (T *)take(vm);
		xbest = (T *)take(vm);
		partial = (double *)take((size_t)B * G * 2 * sizeof(double));
		sums = (double *)take((size_t)B * 2 * sizeof(double));
		coef = (double *)take((size_t)B * 2 * sizeof(double));
		active = (int *)take((size_t)B * sizeof(int));
	}
};

int gridFor(const phb_csr_pcg *a) {
	return std::max(1, std::min(4 * 148 / std::max(1, a->nenv) + 1, (a->n + BLK - 1) / BLK));
}

#define CSR_CUDA(x) PHB_CUDA(x)

template <typename T, typename H>
int runPcg(const phb_csr_pcg *a, phb_solve_result *out, cudaStream_t s) {
	const int n = a->n, B = a->nenv, L = a->nlevels, nc = a->coarse_n;
	const int G = gridFor(a);
	Work<T, H> W(a, G, (char *)a->work);
	auto grid = [&](int rows) { return dim3(std::max(1, std::min(G, (rows + BLK - 1) / BLK)), B); };
	const Csr<T> A{a->row, a->col, (const T *)a->val, a->val_stride, n};
	std::vector<Csr<H>> lA(L), lR(L), lP(L);
	std::vector<const H *> dinv(L);
	std::vector<int64_t> dStride(L);
	for (int l = 0; l < L; ++l) {
		const phb_csr_level &v = a->levels[l];
		lA[l] = Csr<H>{v.a_row, v.a_col, (const H *)v.a_val, v.a_val_stride, v.n};
		lR[l] = Csr<H>{v.r_row, v.r_col, (const H *)v.r_val, 0, l + 1 < L ? a->levels[l + 1].n : nc};
		lP[l] = Csr<H>{v.p_row, v.p_col, (const H *)v.p_val, 0, v.n};
		dinv[l] = (const H *)v.dinv;
		dStride[l] = v.a_val_stride ? v.n : 0;
	}
	T *x = (T *)a->x;
	const T *b = (const T *)a->b;
	const double ns = a->normalized ? 1.0 / std::sqrt(double(n)) : 1.0;
	const double w = a->omega;
	const int pre = std::max(1, a->pre_sweeps), post = std::max(1, a->post_sweeps);
	const bool project = a->project_constant != 0;
	std::vector<int> act(B, 1);
	std::vector<double> hs(2 * B), tol(B), best(B, INFINITY), crit(B, 0.0), rzOld(B, 0.0);
	std::vector<int> used(B, 0), bestIt(B, -1), state(B, 0);
	for (int e = 0; e < B; ++e) tol[e] = a->tolerances ? a->tolerances[e] : a->tol;
	auto upload = [&]() -> int {
		CSR_CUDA(cudaMemcpyAsync(W.active, act.data(), B * sizeof(int), cudaMemcpyHostToDevice, s));
		return 0;
	};
	// sums[e] = (u . v, u2 . v2) of the active environments, also to the host; `mean`: u . 1 / n
	auto dots = [&](const T *u, const T *v, const T *u2, const T *v2, bool mean) -> int {
		kDots<T><<<dim3(G, B), BLK, 0, s>>>(n, u, v, u2, v2, W.partial, W.active);
		kSum<<<(B + 127) / 128, 128, 0, s>>>(W.partial, G, B, W.sums, n, mean ? 1 : 0);
		CSR_CUDA(cudaMemcpyAsync(hs.data(), W.sums, 2 * B * sizeof(double), cudaMemcpyDeviceToHost, s));
		CSR_CUDA(cudaStreamSynchronize(s));
		return 0;
	};
	// z = M r: one V-cycle
	auto vcycle = [&]() -> int {
		const double *shift = nullptr;
		if (project) {
			kDots<T><<<dim3(G, B), BLK, 0, s>>>(n, W.r, nullptr, nullptr, nullptr, W.partial, W.active);
			kSum<<<(B + 127) / 128, 128, 0, s>>>(W.partial, G, B, W.sums, n, 1);
			shift = W.sums; // mean of r in sums[e][0]
		}
		std::vector<H *> cur(L), oth(L);
		for (int l = 0; l < L; ++l) {
			cur[l] = W.lx[l];
			oth[l] = W.ly[l];
			const int nl = lA[l].n;
			const dim3 g = grid(nl);
			if (l == 0) kPre<H, T><<<g, BLK, 0, s>>>(nl, dStride[l], dinv[l], W.r, shift, cur[l], w, W.active);
			else kPre<H, H><<<g, BLK, 0, s>>>(nl, dStride[l], dinv[l], W.lb[l], nullptr, cur[l], w, W.active);
			for (int k = 1; k < pre; ++k) {
				if (l == 0) kJac<H, T, H><<<g, BLK, 0, s>>>(lA[l], dStride[l], dinv[l], W.r, shift, cur[l], oth[l], w, W.active);
				else kJac<H, H, H><<<g, BLK, 0, s>>>(lA[l], dStride[l], dinv[l], W.lb[l], nullptr, cur[l], oth[l], w, W.active);
				std::swap(cur[l], oth[l]);
			}
			if (l == 0) kRes<H, T><<<g, BLK, 0, s>>>(lA[l], W.r, shift, cur[l], W.lres[l], W.active);
			else kRes<H, H><<<g, BLK, 0, s>>>(lA[l], W.lb[l], nullptr, cur[l], W.lres[l], W.active);
			kRect<H><<<grid(lR[l].n), BLK, 0, s>>>(lR[l], W.lres[l], nl, W.lb[l + 1], 0, W.active);
		}
		kCoarse<H><<<grid(nc), BLK, 0, s>>>((const H *)a->coarse_pinv, nc, a->coarse_batched, W.lb[L], W.cx, W.active);
		for (int l = L - 1; l >= 0; --l) {
			const int nl = lA[l].n;
			const dim3 g = grid(nl);
			const H *xc = l + 1 < L ? cur[l + 1] : W.cx;
			const int ncoarse = l + 1 < L ? lA[l + 1].n : nc;
			kRect<H><<<grid(lP[l].n), BLK, 0, s>>>(lP[l], xc, ncoarse, cur[l], 1, W.active);
			for (int k = 0; k < post; ++k) {
				if (l == 0 && k == post - 1) {
					kJac<H, T, T><<<g, BLK, 0, s>>>(lA[l], dStride[l], dinv[l], W.r, shift, cur[l], W.z, w, W.active);
				} else {
					if (l == 0) kJac<H, T, H><<<g, BLK, 0, s>>>(lA[l], dStride[l], dinv[l], W.r, shift, cur[l], oth[l], w, W.active);
					else kJac<H, H, H><<<g, BLK, 0, s>>>(lA[l], dStride[l], dinv[l], W.lb[l], nullptr, cur[l], oth[l], w, W.active);
					std::swap(cur[l], oth[l]);
				}
			}
		}
		if (project) {
			kDots<T><<<dim3(G, B), BLK, 0, s>>>(n, W.z, nullptr, nullptr, nullptr, W.partial, W.active);
			kSum<<<(B + 127) / 128, 128, 0, s>>>(W.partial, G, B, W.sums, n, 1);
			kSubMean<T><<<dim3(G, B), BLK, 0, s>>>(n, W.z, W.sums, W.active);
		}
		CSR_CUDA(cudaGetLastError());
		return 0;
	};
	int rc;
	if ((rc = upload())) return rc;
	CSR_CUDA(cudaMemsetAsync(W.p, 0, (size_t)n * B * sizeof(T), s)); // the first direction is z + 0 p
	CSR_CUDA(cudaMemcpyAsync(W.bw, b, (size_t)n * B * sizeof(T), cudaMemcpyDeviceToDevice, s));
	if (project) { // a compatible right-hand side: mean-free per environment
		if ((rc = dots(W.bw, nullptr, nullptr, nullptr, true))) return rc;
		kSubMean<T><<<dim3(G, B), BLK, 0, s>>>(n, W.bw, W.sums, W.active);
	}
	kResid<T><<<dim3(G, B), BLK, 0, s>>>(A, W.bw, x, W.r, W.active);
	if ((rc = dots(W.r, W.r, nullptr, nullptr, false))) return rc;
	// CG takes at least one iteration: only a non-finite or an exactly zero start residual
	// ends it here (krylov.cu:345-357)
	for (int e = 0; e < B; ++e) {
		crit[e] = std::sqrt(hs[2 * e]) * ns;
		if (!std::isfinite(crit[e])) state[e] = NONFIN;
		else if (crit[e] == 0.0) state[e] = CONV;
		if (state[e]) act[e] = 0;
	}
	auto anyRunning = [&]() { return std::any_of(act.begin(), act.end(), [](int v) { return v != 0; }); };
	std::vector<double> coef(2 * B, 0.0), last(B, 0.0);
	std::vector<int> its(B, 0), rising(B, 0), saveBest(B, 0), restart(B, 1);
	while (anyRunning()) {
		if ((rc = upload())) return rc;
		if ((rc = vcycle())) return rc;
		if ((rc = dots(W.r, W.z, nullptr, nullptr, false))) return rc;
		for (int e = 0; e < B; ++e) { // beta = (r, z) / (r, z)_old; the first direction is z
			if (!act[e]) continue;
			const double rz = hs[2 * e];
			coef[2 * e] = restart[e] ? 0.0 : rz / rzOld[e];
			restart[e] = 0;
			rzOld[e] = rz;
			if (!std::isfinite(rz) || !std::isfinite(coef[2 * e])) { state[e] = NONFIN; used[e] = its[e]; act[e] = 0; }
		}
		if (!anyRunning()) break;
		if ((rc = upload())) return rc;
		CSR_CUDA(cudaMemcpyAsync(W.coef, coef.data(), 2 * B * sizeof(double), cudaMemcpyHostToDevice, s));
		kDir<T><<<dim3(G, B), BLK, 0, s>>>(n, W.z, W.p, W.coef, W.active);
		kSpmv<T><<<dim3(G, B), BLK, 0, s>>>(A, W.p, W.q, W.active);
		if ((rc = dots(W.p, W.q, nullptr, nullptr, false))) return rc;
		for (int e = 0; e < B; ++e) {
			if (!act[e]) continue;
			coef[2 * e + 1] = rzOld[e] / hs[2 * e];
			if (!std::isfinite(coef[2 * e + 1])) { state[e] = NONFIN; used[e] = its[e]; act[e] = 0; }
		}
		if (!anyRunning()) break;
		if ((rc = upload())) return rc;
		CSR_CUDA(cudaMemcpyAsync(W.coef, coef.data(), 2 * B * sizeof(double), cudaMemcpyHostToDevice, s));
		for (int e = 0; e < B; ++e) // the iterate of the best residual so far, before it moves on
			if (act[e] && saveBest[e])
				CSR_CUDA(cudaMemcpyAsync(W.xbest + (size_t)e * n, x + (size_t)e * n, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, s));
		kUpd<T><<<dim3(G, B), BLK, 0, s>>>(n, x, W.r, W.p, W.q, W.coef, W.active);
		if ((rc = dots(W.r, W.r, nullptr, nullptr, false))) return rc;
		// stop tests of kCgUpdate (krylov.cu:536-561)
		for (int e = 0; e < B; ++e) {
			if (!act[e]) continue;
			crit[e] = std::sqrt(hs[2 * e]) * ns;
			++its[e];
			used[e] = its[e] - 1;
			saveBest[e] = 0;
			if (!std::isfinite(crit[e])) { state[e] = NONFIN; act[e] = 0; continue; }
			if (a->return_best) {
				if (crit[e] < best[e]) { best[e] = crit[e]; bestIt[e] = its[e] - 1; saveBest[e] = 1; }
				if (its[e] > 1 && crit[e] >= last[e]) ++rising[e];
				else rising[e] = 0;
				last[e] = crit[e];
			}
			if (crit[e] < tol[e]) state[e] = CONV;
			else if (its[e] >= a->maxit) state[e] = MAXITS;
			else if (a->return_best && rising[e] >= RISING_LIMIT) state[e] = RISE;
			if (state[e]) act[e] = 0;
		}
	}
	for (int e = 0; e < B; ++e) {
		phb_solve_result &o = out[e];
		o.final_residual = crit[e];
		o.used_iterations = used[e];
		o.converged = state[e] == CONV;
		o.finite = std::isfinite(crit[e]) ? 1 : 0;
		o.status = state[e];
		o.inner_iterations = 0;
		o.pad = 0;
		if (a->return_best && (state[e] == MAXITS || state[e] == RISE) && bestIt[e] >= 0 && best[e] < crit[e]) {
			CSR_CUDA(cudaMemcpyAsync(x + (size_t)e * n, W.xbest + (size_t)e * n, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, s));
			o.final_residual = best[e];
			o.used_iterations = bestIt[e];
		}
	}
	CSR_CUDA(cudaStreamSynchronize(s));
	return PHB_OK;
}

int checkArgs(const phb_csr_pcg *a) {
	if (!a || !a->row || !a->col || !a->val || !a->b || !a->x || !a->coarse_pinv || a->n <= 0 || a->nenv <= 0 ||
			a->nlevels < 1 || !a->levels || a->coarse_n <= 0)
		return ::phb::setError(PHB_ERR_ARG, "phb_csr_pcg: bad argument");
	if ((a->dtype != PHB_F32 && a->dtype != PHB_F64) || (a->hdtype != PHB_F32 && a->hdtype != PHB_F64))
		return ::phb::setError(PHB_ERR_ARG, "phb_csr_pcg: dtype");
	if (a->levels[0].n != a->n) return ::phb::setError(PHB_ERR_ARG, "phb_csr_pcg: the finest level does not match the system matrix");
	for (int l = 0; l < a->nlevels; ++l) {
		const phb_csr_level &v = a->levels[l];
		if (!v.a_row || !v.a_col || !v.a_val || !v.dinv || !v.r_row || !v.r_col || !v.r_val || !v.p_row || !v.p_col || !v.p_val || v.n <= 0)
			return ::phb::setError(PHB_ERR_ARG, "phb_csr_pcg: incomplete level");
	}
	return PHB_OK;
}

} // namespace

extern "C" int64_t phb_csr_pcg_work_bytes(const phb_csr_pcg *a) {
	if (checkArgs(a) != PHB_OK) return -1;
	const int G = gridFor(a);
	if (a->dtype == PHB_F64) {
		if (a->hdtype == PHB_F64) return (int64_t)Work<double, double>(a, G, nullptr).total;
		return (int64_t)Work<double, float>(a, G, nullptr).total;
	}
	if (a->hdtype == PHB_F64) return (int64_t)Work<float, double>(a, G, nullptr).total;
	return (int64_t)Work<float, float>(a, G, nullptr).total;
}

extern "C" int phb_csr_pcg_solve(const phb_csr_pcg *a, phb_solve_result *out, phb_stream stream) {
	int rc = checkArgs(a);
	if (rc) return rc;
	if (!a->work || !out) return ::phb::setError(PHB_ERR_ARG, "phb_csr_pcg_solve: work and out are required");
	cudaStream_t s = (cudaStream_t)stream;
	if (a->dtype == PHB_F64) return a->hdtype == PHB_F64 ? runPcg<double, double>(a, out, s) : runPcg<double, float>(a, out, s);
	return a->hdtype == PHB_F64 ? runPcg<float, double>(a, out, s) : runPcg<float, float>(a, out, s);
}
