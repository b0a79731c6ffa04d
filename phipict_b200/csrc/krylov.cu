// Fused, batched Krylov solvers on stencil matrices: CG and BiCGStab for many systems at
// once (instances x right-hand sides), plus FP64 iterative refinement around FP32 inner
// solves.
//
// Algorithm and stop rule follow phiPICT's fused solvers (solvers/krylov/krylov.cu):
// classic CG in two fused phases per iteration (:428-568), van der Vorst BiCGStab with a
// half-step convergence check (:599-824), the criterion ||r||_2/sqrt(n) < tol per system,
// FP64 accumulation of every inner product and a deterministic fixed-order reduction in
// the last CTA to finish (:157-202). The B200 design differs where the hardware rewards it:
//   - the SpMV reads a stencil (2d+1 values per row, no column indices, neighbours by
//     index arithmetic), one CTA per 256-cell tile of one block, so every CTA belongs to
//     one instance and per-instance reductions are contiguous CTA ranges;
//   - the search direction update is folded into the SpMV of the next phase (p is evaluated
//     on the fly at the stencil points), which also removes BiCGStab's separate p kernel;
//   - the iteration loop is a conditional WHILE node of a CUDA graph whose condition the
//     last CTA sets, so a solve is one graph launch with no host round trip, and when the
//     caller is capturing a stream (a whole PISO step as one graph) the loop is spliced
//     into that capture instead.
#include <map>
#include <vector>
#include <mutex>
#include <string>
#include <cstring>
#include <cmath>
#include <functional>
#include <type_traits>
#include "phb_device.cuh"
#include "phb_amg.cuh"
#include "phb_launch.cuh"

int phbCheckAmg(const phb_amg *amg); // amg.cu

namespace phb {

constexpr int NWARPS = PHB_TILE / 32;
enum Done : int { RUNNING = 0, CONVERGED = 1, NONFINITE = 2, MAXIT = 3, RISING = 4 };
constexpr int RISING_CUTOFF = 100;

struct SysState {
	double tol, rho, alpha, beta, omega, crit, best, last, halfCrit, innerTol;
	int it, maxit, bestIt, rising, done, restart, saveBest, halfDone, usedIt, innerIts;
	int launched, pad2;
};
static_assert(sizeof(SysState) == 128, "SysState layout");

struct Control {
	unsigned int counter;
	int allDone;
	int loops;
	int maxLoops;
	unsigned int barCount; // grid barrier of the persistent solvers: arrival counter
	int barErr;            // set when a barrier wait ran out (the kernel then returns)
	int pad[2];
};
static_assert(sizeof(Control) == 32, "Control layout");

// device helpers -----------------------------------------------------------------------
__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// Block-reduce NV values, write this CTA's partials, and return whether this CTA is the
// last of the grid to finish (the ticket pattern of krylov.cu:157-182).
template <int NV>
__device__ __forceinline__ bool storePartials(double (&v)[NV], double *partial, unsigned int *counter) {
	__shared__ double sm[NV][NWARPS];
	__shared__ bool isLast;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int q = 0; q < NV; ++q) {
		const double s = warpSum(v[q]);
		if (lane == 0) sm[q][warp] = s;
	}
	__syncthreads();
	if (threadIdx.x < NV) {
		double s = 0;
#pragma unroll
		for (int w = 0; w < NWARPS; ++w) s += sm[threadIdx.x][w];
		partial[(size_t)blockIdx.x * NV + threadIdx.x] = s;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		__threadfence();
		const unsigned int ticket = atomicAdd(counter, 1u);
		isLast = ticket == gridDim.x - 1;
	}
	__syncthreads();
	return isLast;
}

// In the last CTA: the warps are split into groups of G (a power of two, as many as fit
// NWARPS/nsys); each group sums the CTA partials of one system's instance in a fixed order
// (lanes strided over the tiles, two accumulators in flight, then warp and group sums) and
// its leader calls fn(state, inst, sums, instSum). allDone is updated and the ticket
// counter reset for the next kernel. With INSTQ >= 0 the group also sums quantity INSTQ over
// all K systems of the instance (instSum), e.g. the whole right-hand side norm.
template <int K, int NQ, int INSTQ = -1, typename Fn>
__device__ __forceinline__ void finalizeSystems(const int32_t *insts, int ninst, const double *partial, SysState *st, Control *ctrl, Fn fn) {
	constexpr int NV = NQ + 1;
	__shared__ int running;
	__shared__ double gsm[NWARPS][NV];
	if (threadIdx.x == 0) running = 0;
	__threadfence();
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int nsys = ninst * K;
	int G = NWARPS;
	while (G > 1 && G * nsys > NWARPS) G >>= 1;
	const int NG = NWARPS / G;
	const int group = warp / G, wg = warp - group * G;
	for (int base = 0; base < nsys; base += NG) {
		const int s = base + group;
		const bool act = s < nsys && st[s].done == RUNNING;
		double a0[NV], a1[NV];
#pragma unroll
		for (int q = 0; q < NV; ++q) { a0[q] = 0; a1[q] = 0; }
		if (act) {
			const int inst = s / K, k = s - inst * K;
			const int t0 = insts[inst * PHB_IREC + I_TILESTART], tc = insts[inst * PHB_IREC + I_TILECOUNT];
			const int stride = G * 32;
			auto load = [&](int t, double *a) {
				const double *pp = partial + (size_t)(t0 + t) * K * NQ;
#pragma unroll
				for (int q = 0; q < NQ; ++q) a[q] += __ldcg(pp + k * NQ + q);
				if (INSTQ >= 0) {
#pragma unroll
					for (int kk = 0; kk < K; ++kk) a[NQ] += __ldcg(pp + kk * NQ + (INSTQ < 0 ? 0 : INSTQ));
				}
			};
			int t = wg * 32 + lane;
			for (; t + stride < tc; t += 2 * stride) { load(t, a0); load(t + stride, a1); }
			if (t < tc) load(t, a0);
		}
#pragma unroll
		for (int q = 0; q < NV; ++q) {
			const double v = warpSum(a0[q] + a1[q]);
			if (lane == 0) gsm[warp][q] = v;
		}
		__syncthreads();
		if (act && wg == 0 && lane == 0) {
			double red[NV];
#pragma unroll
			for (int q = 0; q < NV; ++q) {
				double v = 0;
				for (int w = 0; w < G; ++w) v += gsm[group * G + w][q];
				red[q] = v;
			}
			fn(st[s], s / K, red, red[NQ]);
		}
		if (wg == 0 && lane == 0 && s < nsys && st[s].done == RUNNING) atomicAdd(&running, 1);
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		ctrl->allDone = running == 0;
		ctrl->counter = 0;
	}
}

__device__ __forceinline__ bool fin(double v) { return isfinite(v); }
__device__ __forceinline__ double normScale(const int32_t *insts, int inst) { return 1.0 / sqrt(double(insts[inst * PHB_IREC + I_NCELLS])); }

template <int K>
__device__ __forceinline__ int64_t vk(const int32_t *B, int64_t g, int k) {
	return g + (int64_t)(K - 1) * B[B_INSTOFF] + (int64_t)k * B[B_INSTN];
}

template <int D>
__device__ __forceinline__ void stencilNeighbors(const Dom<double, D> &dom, const Cell &c, int64_t *nb) {
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) nb[f] = neighborIndex<double, D>(dom, c, f);
}

// Krylov tile bodies on quads ------------------------------------------------------------
// Fields evaluated at the stencil points: at(o) one value, at4(o) four consecutive values.
// Every multiply-add is an explicit fma, so that the persistent kernel and the per-phase
// kernels round identically whatever contraction the compiler would choose in each.
template <typename T>
struct FX { // a stored vector
	const T *x;
	__device__ __forceinline__ T at(int64_t o) const { return x[o]; }
	__device__ __forceinline__ void at4(int64_t o, int n, bool al, T (&v)[4]) const { ld4(x + o, n, al, v); }
};
template <typename T>
struct FDir { // CG direction p' = z + beta p (z after a restart)
	const T *z, *p;
	T beta;
	bool rs;
	__device__ __forceinline__ T at(int64_t o) const { return rs ? z[o] : fma(beta, p[o], z[o]); }
	__device__ __forceinline__ void at4(int64_t o, int n, bool al, T (&v)[4]) const {
		ld4(z + o, n, al, v);
		if (rs) return;
		T b[4];
		ld4(p + o, n, al, b);
#pragma unroll
		for (int i = 0; i < 4; ++i) v[i] = fma(beta, b[i], v[i]);
	}
};
template <typename T>
struct FBicgP { // BiCGStab direction p = r + beta (p - omega v) (r after a restart)
	const T *r, *p, *v;
	T beta, omega;
	bool rs;
	__device__ __forceinline__ T at(int64_t o) const { return rs ? r[o] : fma(beta, fma(-omega, v[o], p[o]), r[o]); }
	__device__ __forceinline__ void at4(int64_t o, int n, bool al, T (&w)[4]) const {
		ld4(r + o, n, al, w);
		if (rs) return;
		T a[4], b[4];
		ld4(p + o, n, al, a);
		ld4(v + o, n, al, b);
#pragma unroll
		for (int i = 0; i < 4; ++i) w[i] = fma(beta, fma(-omega, b[i], a[i]), w[i]);
	}
};
template <typename T>
struct FBicgS { // BiCGStab half step s = r - alpha v
	const T *r, *v;
	T alpha;
	__device__ __forceinline__ T at(int64_t o) const { return fma(-alpha, v[o], r[o]); }
	__device__ __forceinline__ void at4(int64_t o, int n, bool al, T (&w)[4]) const {
		T b[4];
		ld4(r + o, n, al, w);
		ld4(v + o, n, al, b);
#pragma unroll
		for (int i = 0; i < 4; ++i) w[i] = fma(-alpha, b[i], w[i]);
	}
};

// y = A f and f itself at the quad's cells for every active right-hand side (zeros for the
// others and past q.n). On the fast path (a quad inside one row whose y and z neighbours are
// in the block or absent behind a prescribed face) the four cells' stencil rows and neighbour
// groups are loaded at once, slot by slot; elsewhere every cell resolves its neighbours
// across faces. The products are summed in the same order on both paths (centre, then faces
// -x +x -y +y -z +z, a face without neighbour skipped).
template <typename T, int D, int K, typename F>
__device__ __forceinline__ void quadApply(const Dom<double, D> &dom, const T *__restrict__ A, const Quad &q, const bool (&act)[K],
		const F (&fld)[K], T (&y)[K][4], T (&f)[K][4]) {
	const int64_t N = dom.ncells;
	if (q.fastW) {
		// x neighbours of the row ends: across the block's x face when the quad touches it
		int64_t gW = q.g - 1, gE = q.g + 4;
		if (q.p[0] == 0 || q.p[0] + 3 == q.B[B_NX] - 1) {
			Cell c;
			c.B = q.B;
			c.p[1] = q.p[1];
			c.p[2] = q.p[2];
			if (q.p[0] == 0) {
				c.p[0] = 0;
				c.g = (int)q.g;
				gW = neighborIndex<double, D>(dom, c, 0);
			}
			if (q.p[0] + 3 == q.B[B_NX] - 1) {
				c.p[0] = q.p[0] + 3;
				c.g = (int)(q.g + 3);
				gE = neighborIndex<double, D>(dom, c, 1);
			}
		}
		int64_t o[K];
#pragma unroll
		for (int k = 0; k < K; ++k) o[k] = vk<K>(q.B, q.g, k);
		T a[4];
		ld4(A + q.g, 4, q.al, a);
#pragma unroll
		for (int k = 0; k < K; ++k) {
			if (!act[k]) {
#pragma unroll
				for (int i = 0; i < 4; ++i) f[k][i] = 0;
			} else {
				fld[k].at4(o[k], 4, q.al, f[k]);
			}
#pragma unroll
			for (int i = 0; i < 4; ++i) y[k][i] = a[i] * f[k][i];
		}
		ld4(A + N + q.g, 4, q.al, a);
#pragma unroll
		for (int k = 0; k < K; ++k) {
			if (!act[k]) continue;
			if (gW >= 0) y[k][0] = fma(a[0], fld[k].at(vk<K>(q.B, gW, k)), y[k][0]);
#pragma unroll
			for (int i = 1; i < 4; ++i) y[k][i] = fma(a[i], f[k][i - 1], y[k][i]);
		}
		ld4(A + 2 * N + q.g, 4, q.al, a);
#pragma unroll
		for (int k = 0; k < K; ++k) {
			if (!act[k]) continue;
#pragma unroll
			for (int i = 0; i < 3; ++i) y[k][i] = fma(a[i], f[k][i + 1], y[k][i]);
			if (gE >= 0) y[k][3] = fma(a[3], fld[k].at(vk<K>(q.B, gE, k)), y[k][3]);
		}
#pragma unroll
		for (int sl = 3; sl < 2 * D + 1; ++sl) {
			if ((q.miss >> (sl - 3)) & 1) continue; // behind a prescribed face: no neighbour
			const int64_t off = sl == 3 ? -(int64_t)q.sy : sl == 4 ? (int64_t)q.sy : sl == 5 ? -(int64_t)q.sz : (int64_t)q.sz;
			const bool al = sl < 5 ? q.alY : q.alZ;
			ld4(A + sl * N + q.g, 4, q.al, a);
#pragma unroll
			for (int k = 0; k < K; ++k) {
				if (!act[k]) continue;
				T v[4];
				fld[k].at4(o[k] + off, 4, al, v);
#pragma unroll
				for (int i = 0; i < 4; ++i) y[k][i] = fma(a[i], v[i], y[k][i]);
			}
		}
		return;
	}
#pragma unroll
	for (int i = 0; i < 4; ++i) {
#pragma unroll
		for (int k = 0; k < K; ++k) { y[k][i] = 0; f[k][i] = 0; }
		if (i >= q.n) continue;
		Cell c;
		quadCell<D>(q, i, c);
		int64_t nb[2 * D];
		stencilNeighbors<D>(dom, c, nb);
		const T a0 = A[c.g];
		T af[2 * D];
#pragma unroll
		for (int fc = 0; fc < 2 * D; ++fc) af[fc] = A[(fc + 1) * N + c.g];
#pragma unroll
		for (int k = 0; k < K; ++k) {
			if (!act[k]) continue;
			const T ci = fld[k].at(vk<K>(c.B, c.g, k));
			T s = a0 * ci;
#pragma unroll
			for (int fc = 0; fc < 2 * D; ++fc)
				if (nb[fc] >= 0) s = fma(af[fc], fld[k].at(vk<K>(c.B, nb[fc], k)), s);
			y[k][i] = s;
			f[k][i] = ci;
		}
	}
}

// r = b - A x per right-hand side, (r, r) and (b, b) into acc[2k], acc[2k+1]; emit(k, o, q,
// r[4]) stores r.
template <typename T, int D, int K, typename Emit>
__device__ __forceinline__ void tileResidual(const Dom<double, D> &dom, const int32_t *sB, int l0, int nc, const T *__restrict__ A,
		const T *__restrict__ b, const T *__restrict__ x, const bool (&act)[K], double (&acc)[2 * K], Emit emit) {
	Quad q;
	quadAt<D, K>(dom.vec4, sB, l0, nc, q);
	FX<T> fx[K];
#pragma unroll
	for (int k = 0; k < K; ++k) fx[k].x = x;
	T y[K][4], f[K][4];
	quadApply<T, D, K>(dom, A, q, act, fx, y, f);
#pragma unroll
	for (int k = 0; k < K; ++k) {
		if (!act[k]) continue;
		const int64_t o = vk<K>(q.B, q.g, k);
		T bv[4], rv[4];
		ld4(b + o, q.n, q.al, bv);
#pragma unroll
		for (int i = 0; i < 4; ++i) {
			rv[i] = bv[i] - y[k][i];
			acc[2 * k] = fma(double(rv[i]), double(rv[i]), acc[2 * k]);
			acc[2 * k + 1] = fma(double(bv[i]), double(bv[i]), acc[2 * k + 1]);
		}
		emit(k, o, q, rv);
	}
}

// CG phase 1 on a tile: p' = z + beta p, q = A p', (p', q)
template <typename T, int D, int K>
__device__ __forceinline__ void tileCgDirection(const Dom<double, D> &dom, const int32_t *sB, int l0, int nc, const T *__restrict__ A,
		const T *z, const T *pIn, T *pOut, T *qv, const bool (&act)[K], const bool (&rs)[K], const T (&beta)[K], double (&acc)[K]) {
	Quad q;
	quadAt<D, K>(dom.vec4, sB, l0, nc, q);
	FDir<T> fd[K];
#pragma unroll
	for (int k = 0; k < K; ++k) fd[k] = FDir<T>{z, pIn, beta[k], rs[k]};
	T y[K][4], f[K][4];
	quadApply<T, D, K>(dom, A, q, act, fd, y, f);
#pragma unroll
	for (int k = 0; k < K; ++k) {
		if (!act[k]) continue;
		const int64_t o = vk<K>(q.B, q.g, k);
		st4(pOut + o, q.n, q.al, f[k]);
		st4(qv + o, q.n, q.al, y[k]);
#pragma unroll
		for (int i = 0; i < 4; ++i) acc[k] = fma(double(f[k][i]), double(y[k][i]), acc[k]);
	}
}

// CG phase 2 on a tile: x += alpha p, r -= alpha q, (r, r) (xbest = x before, when asked)
template <typename T, int D, int K>
__device__ __forceinline__ void tileCgUpdate(const Dom<double, D> &dom, const int32_t *sB, int l0, int nc, T *r, const T *p,
		const T *qv, T *x, T *xbest, const SysState *sst, double (&acc)[K]) {
	Quad q;
	quadAt<D, K>(dom.vec4, sB, l0, nc, q);
	const int inst = sB[B_INST];
#pragma unroll
	for (int k = 0; k < K; ++k) {
		const SysState &s = sst[inst * K + k];
		if (s.done != RUNNING) continue;
		const T alpha = T(s.alpha);
		const int64_t o = vk<K>(q.B, q.g, k);
		T xv[4], pv[4], rv[4], qq[4];
		ld4(x + o, q.n, q.al, xv);
		ld4(p + o, q.n, q.al, pv);
		ld4(r + o, q.n, q.al, rv);
		ld4(qv + o, q.n, q.al, qq);
		if (s.saveBest && xbest) st4(xbest + o, q.n, q.al, xv);
#pragma unroll
		for (int i = 0; i < 4; ++i) {
			xv[i] = fma(alpha, pv[i], xv[i]);
			rv[i] = fma(-alpha, qq[i], rv[i]);
			acc[k] = fma(double(rv[i]), double(rv[i]), acc[k]);
		}
		st4(x + o, q.n, q.al, xv);
		st4(r + o, q.n, q.al, rv);
	}
}

// BiCGStab phase 1 on a tile: p = r + beta (p - omega v), v = A p, (r0, v)
template <typename T, int D, int K>
__device__ __forceinline__ void tileBicgV(const Dom<double, D> &dom, const int32_t *sB, int l0, int nc, const T *__restrict__ A,
		const T *r, const T *pIn, const T *vIn, T *pOut, T *vOut, const T *r0, const bool (&act)[K], const bool (&rs)[K],
		const T (&beta)[K], const T (&omega)[K], double (&acc)[K]) {
	Quad q;
	quadAt<D, K>(dom.vec4, sB, l0, nc, q);
	FBicgP<T> fp[K];
#pragma unroll
	for (int k = 0; k < K; ++k) fp[k] = FBicgP<T>{r, pIn, vIn, beta[k], omega[k], rs[k]};
	T y[K][4], f[K][4];
	quadApply<T, D, K>(dom, A, q, act, fp, y, f);
#pragma unroll
	for (int k = 0; k < K; ++k) {
		if (!act[k]) continue;
		const int64_t o = vk<K>(q.B, q.g, k);
		st4(pOut + o, q.n, q.al, f[k]);
		st4(vOut + o, q.n, q.al, y[k]);
		T r0v[4];
		ld4(r0 + o, q.n, q.al, r0v);
#pragma unroll
		for (int i = 0; i < 4; ++i) acc[k] = fma(double(r0v[i]), double(y[k][i]), acc[k]);
	}
}

// BiCGStab phase 2 on a tile: s = r - alpha v, t = A s, (t, s), (t, t), (s, s)
template <typename T, int D, int K>
__device__ __forceinline__ void tileBicgT(const Dom<double, D> &dom, const int32_t *sB, int l0, int nc, const T *__restrict__ A,
		const T *r, const T *v, T *t, const bool (&act)[K], const T (&alpha)[K], double (&acc)[3 * K]) {
	Quad q;
	quadAt<D, K>(dom.vec4, sB, l0, nc, q);
	FBicgS<T> fs[K];
#pragma unroll
	for (int k = 0; k < K; ++k) fs[k] = FBicgS<T>{r, v, alpha[k]};
	T y[K][4], f[K][4];
	quadApply<T, D, K>(dom, A, q, act, fs, y, f);
#pragma unroll
	for (int k = 0; k < K; ++k) {
		if (!act[k]) continue;
		const int64_t o = vk<K>(q.B, q.g, k);
		st4(t + o, q.n, q.al, y[k]);
#pragma unroll
		for (int i = 0; i < 4; ++i) {
			acc[3 * k + 0] = fma(double(y[k][i]), double(f[k][i]), acc[3 * k + 0]);
			acc[3 * k + 1] = fma(double(y[k][i]), double(y[k][i]), acc[3 * k + 1]);
			acc[3 * k + 2] = fma(double(f[k][i]), double(f[k][i]), acc[3 * k + 2]);
		}
	}
}

// BiCGStab phase 3 on a tile: x += alpha p + omega s, r = s - omega t, (r0, r), (r, r); after
// a converged half step x += alpha p, r = s
template <typename T, int D, int K>
__device__ __forceinline__ void tileBicgUpdate(const Dom<double, D> &dom, const int32_t *sB, int l0, int nc, T *r, const T *r0,
		const T *p, const T *v, const T *t, T *x, const SysState *sst, double (&acc)[2 * K]) {
	Quad q;
	quadAt<D, K>(dom.vec4, sB, l0, nc, q);
	const int inst = sB[B_INST];
#pragma unroll
	for (int k = 0; k < K; ++k) {
		const SysState &s = sst[inst * K + k];
		if (s.done != RUNNING) continue;
		const T alpha = T(s.alpha), omega = T(s.omega);
		const int64_t o = vk<K>(q.B, q.g, k);
		T rv[4], vv[4], pv[4], xv[4];
		ld4(r + o, q.n, q.al, rv);
		ld4(v + o, q.n, q.al, vv);
		ld4(p + o, q.n, q.al, pv);
		ld4(x + o, q.n, q.al, xv);
		if (s.halfDone) {
#pragma unroll
			for (int i = 0; i < 4; ++i) {
				xv[i] = fma(alpha, pv[i], xv[i]);
				rv[i] = fma(-alpha, vv[i], rv[i]);
			}
		} else {
			T tv[4], r0v[4];
			ld4(t + o, q.n, q.al, tv);
			ld4(r0 + o, q.n, q.al, r0v);
#pragma unroll
			for (int i = 0; i < 4; ++i) {
				const T si = fma(-alpha, vv[i], rv[i]);
				xv[i] = fma(omega, si, fma(alpha, pv[i], xv[i]));
				rv[i] = fma(-omega, tv[i], si);
				acc[2 * k + 0] = fma(double(r0v[i]), double(rv[i]), acc[2 * k + 0]);
				acc[2 * k + 1] = fma(double(rv[i]), double(rv[i]), acc[2 * k + 1]);
			}
		}
		st4(x + o, q.n, q.al, xv);
		st4(r + o, q.n, q.al, rv);
	}
}

struct LoopCond {
	cudaGraphConditionalHandle handle;
	int active; // this kernel sets the loop condition
};
__device__ __forceinline__ void setLoop(const LoopCond lc, Control *ctrl) {
	if (!lc.active) return;
	const int loops = ++ctrl->loops; // one count per pass of the loop body
	const bool cont = !ctrl->allDone && loops < ctrl->maxLoops;
	cudaGraphSetConditional(lc.handle, cont ? 1u : 0u);
}

// kernels ------------------------------------------------------------------------------
// SolverTolerance._resolve_scale (solvers/tolerance.py:241-257)
__device__ __forceinline__ double resolveTol(const phb_tolerance &t, double scale) {
	double tol = 0.0;
	if (t.rtol > 0) tol = t.rtol * scale;
	if (t.atol > 0) tol = fmax(tol, t.atol);
	tol = fmax(tol, t.floor_eps * scale);
	if (!(tol > 0.0)) tol = t.fallback;
	return tol;
}

// Initial state of every system. fromInner: the tolerance was written into
// SysState::innerTol by the refinement residual (mode ignored).
__global__ void kInit(SysState *st, int nsys, phb_tolerance tol, int fromInner, int maxit, Control *ctrl, int maxLoops) {
	for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
		double t;
		if (fromInner) t = st[s].innerTol;
		else if (tol.mode == 0) t = tol.atol;
		else if (tol.mode == 2) t = tol.values[s];
		else t = NAN; // resolved from the right-hand side by kResidual
		SysState z;
		memset(&z, 0, sizeof(z));
		z.tol = t;
		z.innerTol = t;
		z.maxit = maxit;
		z.best = INFINITY;
		z.restart = 1;
		z.bestIt = -1;
		st[s] = z;
	}
	if (threadIdx.x == 0) {
		ctrl->counter = 0; ctrl->allDone = 0; ctrl->loops = 0; ctrl->maxLoops = maxLoops;
		ctrl->barCount = 0; ctrl->barErr = 0;
	}
}

// r = b - A x (and r0 = r for BiCGStab); rho = (r, r); the relative tolerance from (b, b);
// initial convergence check (krylov.cu:292-366). The reference CG stops on an exactly zero
// residual only, BiCGStab (and, here, every inner solve of the refinement: STOPSTART) on
// crit < tol.
template <typename T, int D, int K, bool BICG, bool STOPSTART>
__global__ void __launch_bounds__(PHB_TILE) kResidual(Dom<double, D> dom, const T *__restrict__ A, const T *__restrict__ b,
		const T *__restrict__ x, T *__restrict__ r, T *__restrict__ r0, SysState *st, double *partial, Control *ctrl, phb_tolerance tol,
		LoopCond arm) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	const int inst = sB[B_INST];
	bool act[K];
#pragma unroll
	for (int k = 0; k < K; ++k) act[k] = st[inst * K + k].done == RUNNING;
	double acc[2 * K];
#pragma unroll
	for (int k = 0; k < 2 * K; ++k) acc[k] = 0;
	tileResidual<T, D, K>(dom, sB, l0_, nc_, A, b, x, act, acc, [&](int, int64_t o, const Quad &q, const T (&rv)[4]) {
		st4(r + o, q.n, q.al, rv);
		if (BICG) st4(r0 + o, q.n, q.al, rv);
	});
	if (storePartials<2 * K>(acc, partial, &ctrl->counter)) {
		const bool relative = tol.mode == 1;
		finalizeSystems<K, 2, 1>(dom.insts, dom.ninst, partial, st, ctrl, [&](SysState &s, int in, const double *red, double bb) {
			const double ns = normScale(dom.insts, in);
			// the rhs scale of the whole instance: all K right-hand sides together
			if (relative) s.tol = resolveTol(tol, sqrt(bb / double(K)) * ns);
			const double crit = sqrt(red[0]) * ns;
			s.rho = red[0];
			s.restart = 1;
			s.crit = crit;
			if (!fin(crit)) { s.done = NONFINITE; s.usedIt = 0; }
			else if ((BICG || STOPSTART) ? crit < s.tol : crit == 0.0) { s.done = CONVERGED; s.usedIt = BICG ? -1 : 0; }
		});
		// arm the WHILE loop that follows: run its body only if a system is still running
		if (threadIdx.x == 0 && arm.active) cudaGraphSetConditional(arm.handle, ctrl->allDone ? 0u : 1u);
	}
}

// CG phase 1 (kCgDirection, krylov.cu:428-498): p' = r + beta p (p' = r on restart,
// evaluated at the stencil points), q = A p', (p', q); last CTA: alpha = rho / (p', q)
template <typename T, int D, int K>
__global__ void __launch_bounds__(PHB_TILE) kCgDirection(Dom<double, D> dom, const T *__restrict__ A, const T *__restrict__ r,
		const T *__restrict__ pIn, T *__restrict__ pOut, T *__restrict__ q, SysState *st, double *partial, Control *ctrl) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	const int inst = sB[B_INST];
	bool act[K], rs[K];
	T beta[K];
#pragma unroll
	for (int k = 0; k < K; ++k) {
		const SysState &s = st[inst * K + k];
		act[k] = s.done == RUNNING;
		rs[k] = s.restart;
		beta[k] = T(s.beta);
	}
	double acc[K];
#pragma unroll
	for (int k = 0; k < K; ++k) acc[k] = 0;
	tileCgDirection<T, D, K>(dom, sB, l0_, nc_, A, r, pIn, pOut, q, act, rs, beta, acc);
	if (storePartials<K>(acc, partial, &ctrl->counter)) {
		finalizeSystems<K, 1>(dom.insts, dom.ninst, partial, st, ctrl, [&](SysState &s, int, const double *red, double) {
			const double alpha = s.rho / red[0];
			s.restart = 0;
			if (!fin(alpha)) { s.done = NONFINITE; s.usedIt = s.it; }
			else s.alpha = alpha;
		});
	}
}

// CG phase 2 (kCgUpdate, krylov.cu:502-568): x += alpha p, r -= alpha q, (r, r); last CTA:
// convergence, beta = (r, r)_new / (r, r)_old, optional best-iterate tracking. Preconditioned
// (PC): beta comes from (r, z) after the next V-cycle instead (kPcgPrecond).
template <typename T, int D, int K, bool PC = false>
__global__ void __launch_bounds__(PHB_TILE) kCgUpdate(Dom<double, D> dom, T *__restrict__ r, const T *__restrict__ p,
		const T *__restrict__ q, T *__restrict__ x, T *__restrict__ xbest, SysState *st, double *partial, Control *ctrl,
		int returnBest, LoopCond lc) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	double acc[K];
#pragma unroll
	for (int k = 0; k < K; ++k) acc[k] = 0;
	tileCgUpdate<T, D, K>(dom, sB, l0_, nc_, r, p, q, x, xbest, st, acc);
	if (storePartials<K>(acc, partial, &ctrl->counter)) {
		finalizeSystems<K, 1>(dom.insts, dom.ninst, partial, st, ctrl, [&](SysState &s, int in, const double *red, double) {
			const double crit = sqrt(red[0]) * normScale(dom.insts, in);
			++s.it;
			s.crit = crit;
			s.saveBest = 0;
			s.usedIt = s.it - 1;
			if (!fin(crit)) { s.done = NONFINITE; return; }
			if (returnBest) {
				if (crit < s.best) { s.best = crit; s.bestIt = s.it - 1; s.saveBest = 1; }
				if (s.it > 1 && crit >= s.last) ++s.rising; else s.rising = 0;
				s.last = crit;
			}
			if (crit < s.tol) s.done = CONVERGED;
			else if (s.it >= s.maxit) s.done = MAXIT;
			else if (returnBest && s.rising >= RISING_CUTOFF) s.done = RISING;
			else if (!PC) {
				s.beta = red[0] / s.rho;
				s.rho = red[0];
				if (!fin(s.beta)) s.done = NONFINITE;
			}
		});
		if (threadIdx.x == 0) setLoop(lc, ctrl);
	}
}

// rho/beta of a running system from the new (r, z) (the preconditioned CG of
// amg_pcg_solve, solvers/amg.py:1544): the first iteration after a restart takes rho only.
__device__ __forceinline__ void pcgRho(SysState &s, double rz) {
	if (s.restart) s.rho = rz;
	else {
		s.beta = rz / s.rho;
		s.rho = rz;
		if (!fin(s.beta)) s.done = NONFINITE;
	}
	if (!fin(rz)) s.done = NONFINITE;
}

// Last step of the V-cycle on level 0 (prolongation and post-smoothing, z written to the
// hierarchy's level-0 x) fused with (r, z); last CTA: rho and beta (pcgRho).
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kPcgPrecond(Dom<double, D> dom, AmgView<D> mg, SysState *st, double *partial, Control *ctrl) {
	__shared__ int32_t sB[PHB_BREC];
	double acc[1] = {amgProlongQuad<D>(mg, 0, blockIdx.x, sB, mg.x[0])};
	if (storePartials<1>(acc, partial, &ctrl->counter)) {
		finalizeSystems<1, 1>(dom.insts, dom.ninst, partial, st, ctrl, [&](SysState &s, int, const double *red, double) { pcgRho(s, red[0]); });
	}
}

// BiCGStab phase 1 (kBicgP + kBicgV, krylov.cu:599-676): p = r + beta (p - omega v) (p = r
// on restart) evaluated at the stencil points, v = A p, (r0, v); last CTA: alpha
template <typename T, int D, int K>
__global__ void __launch_bounds__(PHB_TILE) kBicgV(Dom<double, D> dom, const T *__restrict__ A, const T *__restrict__ r,
		const T *__restrict__ pIn, const T *__restrict__ vIn, T *__restrict__ pOut, T *__restrict__ vOut, const T *__restrict__ r0,
		SysState *st, double *partial, Control *ctrl) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	const int inst = sB[B_INST];
	bool act[K], rs[K];
	T beta[K], omega[K];
#pragma unroll
	for (int k = 0; k < K; ++k) {
		const SysState &s = st[inst * K + k];
		act[k] = s.done == RUNNING;
		rs[k] = s.restart;
		beta[k] = T(s.beta);
		omega[k] = T(s.omega);
	}
	double acc[K];
#pragma unroll
	for (int k = 0; k < K; ++k) acc[k] = 0;
	tileBicgV<T, D, K>(dom, sB, l0_, nc_, A, r, pIn, vIn, pOut, vOut, r0, act, rs, beta, omega, acc);
	if (storePartials<K>(acc, partial, &ctrl->counter)) {
		finalizeSystems<K, 1>(dom.insts, dom.ninst, partial, st, ctrl, [&](SysState &s, int, const double *red, double) {
			const double alpha = s.rho / red[0];
			s.restart = 0;
			if (!fin(alpha)) { s.done = NONFINITE; s.usedIt = s.it; }
			else s.alpha = alpha;
		});
	}
}

// BiCGStab phase 2 (kBicgT, krylov.cu:680-750): s = r - alpha v on the fly, t = A s,
// (t,s), (t,t), (s,s); last CTA: omega, or convergence after the half step.
template <typename T, int D, int K>
__global__ void __launch_bounds__(PHB_TILE) kBicgT(Dom<double, D> dom, const T *__restrict__ A, const T *__restrict__ r,
		const T *__restrict__ v, T *__restrict__ t, SysState *st, double *partial, Control *ctrl) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	const int inst = sB[B_INST];
	bool act[K];
	T alpha[K];
#pragma unroll
	for (int k = 0; k < K; ++k) {
		const SysState &s = st[inst * K + k];
		act[k] = s.done == RUNNING;
		alpha[k] = T(s.alpha);
	}
	double acc[3 * K];
#pragma unroll
	for (int k = 0; k < 3 * K; ++k) acc[k] = 0;
	tileBicgT<T, D, K>(dom, sB, l0_, nc_, A, r, v, t, act, alpha, acc);
	if (storePartials<3 * K>(acc, partial, &ctrl->counter)) {
		finalizeSystems<K, 3>(dom.insts, dom.ninst, partial, st, ctrl, [&](SysState &s, int in, const double *red, double) {
			const double critS = sqrt(red[2]) * normScale(dom.insts, in);
			s.halfCrit = critS;
			if (!fin(critS)) { s.done = NONFINITE; s.crit = critS; s.usedIt = s.it; }
			else if (critS < s.tol) { s.halfDone = 1; s.omega = 0.0; }
			else {
				const double omega = red[0] / red[1];
				if (!fin(omega)) { s.done = NONFINITE; s.crit = critS; s.usedIt = s.it; }
				else s.omega = omega;
			}
		});
	}
}

// BiCGStab phase 3 (kBicgUpdate, krylov.cu:754-824): x += alpha p + omega s, r = s - omega t,
// (r0, r), (r, r); last CTA: convergence and beta.
template <typename T, int D, int K>
__global__ void __launch_bounds__(PHB_TILE) kBicgUpdate(Dom<double, D> dom, T *__restrict__ r, const T *__restrict__ r0,
		const T *__restrict__ p, const T *__restrict__ v, const T *__restrict__ t, T *__restrict__ x, SysState *st,
		double *partial, Control *ctrl, LoopCond lc) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	double acc[2 * K];
#pragma unroll
	for (int k = 0; k < 2 * K; ++k) acc[k] = 0;
	tileBicgUpdate<T, D, K>(dom, sB, l0_, nc_, r, r0, p, v, t, x, st, acc);
	if (storePartials<2 * K>(acc, partial, &ctrl->counter)) {
		finalizeSystems<K, 2>(dom.insts, dom.ninst, partial, st, ctrl, [&](SysState &s, int in, const double *red, double) {
			if (s.halfDone) { s.done = CONVERGED; s.crit = s.halfCrit; s.usedIt = s.it; return; }
			const double crit = sqrt(red[1]) * normScale(dom.insts, in);
			s.crit = crit;
			if (!fin(crit)) { s.done = NONFINITE; s.usedIt = s.it; }
			else if (crit < s.tol) { s.done = CONVERGED; s.usedIt = s.it + 1; }
			else {
				++s.it;
				s.usedIt = s.it - 1;
				const double beta = (red[0] / s.rho) * (s.alpha / s.omega);
				s.rho = red[0];
				s.beta = beta;
				if (!fin(beta)) s.done = NONFINITE;
				else if (s.it >= s.maxit) s.done = MAXIT;
			}
		});
		if (threadIdx.x == 0) setLoop(lc, ctrl);
	}
}

// kRestoreBest (krylov.cu:370-375): systems that stopped without converging return their
// best iterate
template <typename T, int K>
__global__ void kRestoreBest(const int32_t *__restrict__ insts, int ninst, int64_t ncells, T *x, const T *xbest, const SysState *st) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ncells * K; i += (int64_t)gridDim.x * blockDim.x) {
		// instance of vector entry i in the [inst][K][cells] layout
		int lo = 0, hi = ninst - 1;
		while (lo < hi) {
			const int mid = (lo + hi + 1) >> 1;
			if ((int64_t)K * insts[mid * PHB_IREC + I_CELLOFF] <= i) lo = mid; else hi = mid - 1;
		}
		const int64_t base = (int64_t)K * insts[lo * PHB_IREC + I_CELLOFF];
		const int k = int((i - base) / insts[lo * PHB_IREC + I_NCELLS]);
		const SysState &s = st[lo * K + k];
		if ((s.done == MAXIT || s.done == RISING) && s.bestIt >= 0 && s.best < s.crit) x[i] = xbest[i];
	}
}

// FP64 refinement residual: r64 = b - A64 x; r32 = float(r64), e32 = 0; last CTA: the
// outer tolerance (resolved from b on the first sweep), outer convergence per system, the
// inner tolerance innerRtol * ||r||/sqrt(n) (infinite for systems that are done) and the
// outer loop condition.
template <int D, int K>
__global__ void __launch_bounds__(PHB_TILE) kRefineResidual(Dom<double, D> dom, const double *__restrict__ A, const double *__restrict__ b,
		const double *__restrict__ x, float *__restrict__ r32, float *__restrict__ e32, SysState *st, double *partial, Control *ctrl,
		double innerRtol, int maxOuter, phb_tolerance tol, SysState *inner, LoopCond lc) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	double acc[2 * K];
#pragma unroll
	for (int k = 0; k < 2 * K; ++k) acc[k] = 0;
	bool act[K];
#pragma unroll
	for (int k = 0; k < K; ++k) act[k] = true;
	tileResidual<double, D, K>(dom, sB, l0_, nc_, A, b, x, act, acc, [&](int, int64_t o, const Quad &q, const double (&rv)[4]) {
		float r4[4], z4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
		for (int i = 0; i < 4; ++i) r4[i] = float(rv[i]);
		st4(r32 + o, q.n, q.al, r4);
		st4(e32 + o, q.n, q.al, z4);
	});
	if (storePartials<2 * K>(acc, partial, &ctrl->counter)) {
		const int nsys = dom.ninst * K;
		// every system is visited, also once done, so that the inner solve of a finished
		// system sees an infinite tolerance and stops at once
		__shared__ int running;
		__shared__ double gsm[NWARPS][2];
		if (threadIdx.x == 0) running = 0;
		__threadfence();
		__syncthreads();
		const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
		int G = NWARPS;
		while (G > 1 && G * nsys > NWARPS) G >>= 1;
		const int NG = NWARPS / G;
		const int group = warp / G, wg = warp - group * G;
		for (int base = 0; base < nsys; base += NG) {
			const int s = base + group;
			double a = 0, bb = 0;
			if (s < nsys) {
				const int inst = s / K, k = s - inst * K;
				const int t0 = dom.insts[inst * PHB_IREC + I_TILESTART], tc = dom.insts[inst * PHB_IREC + I_TILECOUNT];
				for (int t = wg * 32 + lane; t < tc; t += G * 32) {
					const double *pp = partial + (size_t)(t0 + t) * K * 2;
					a += __ldcg(pp + k * 2);
#pragma unroll
					for (int kk = 0; kk < K; ++kk) bb += __ldcg(pp + kk * 2 + 1);
				}
			}
			a = warpSum(a);
			bb = warpSum(bb);
			if (lane == 0) { gsm[warp][0] = a; gsm[warp][1] = bb; }
			__syncthreads();
			if (s < nsys && wg == 0 && lane == 0) {
				a = 0;
				bb = 0;
				for (int w = 0; w < G; ++w) { a += gsm[group * G + w][0]; bb += gsm[group * G + w][1]; }
				const int inst = s / K;
				SysState &o = st[s];
				const double ns = normScale(dom.insts, inst);
				if (o.it == 0 && o.done == RUNNING && tol.mode == 1) o.tol = resolveTol(tol, sqrt(bb / double(K)) * ns);
				const double crit = sqrt(a) * ns;
				o.crit = crit;
				if (o.launched) { o.innerIts += max(inner[s].usedIt, 0); o.launched = 0; }
				if (o.done == RUNNING) {
					if (!fin(crit)) o.done = NONFINITE;
					else if (crit < o.tol) o.done = CONVERGED;
					else if (o.it >= maxOuter) o.done = MAXIT;
					else { ++o.it; o.launched = 1; }
				}
				o.usedIt = o.it;
				inner[s].innerTol = o.done == RUNNING ? fmax(innerRtol * crit, 0.25 * o.tol) : INFINITY;
				if (o.done == RUNNING) atomicAdd(&running, 1);
			}
			__syncthreads();
		}
		if (threadIdx.x == 0) {
			ctrl->allDone = running == 0;
			ctrl->counter = 0;
			setLoop(lc, ctrl);
		}
	}
}

template <int K>
__global__ void kRefineUpdate(int64_t n, double *__restrict__ x, const float *__restrict__ e) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] += double(e[i]);
}

__global__ void kInitOuter(SysState *st, int nsys, phb_tolerance tol, Control *ctrl, int maxLoops, LoopCond arm) {
	for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
		SysState z;
		memset(&z, 0, sizeof(z));
		z.tol = tol.mode == 0 ? tol.atol : tol.mode == 2 ? tol.values[s] : NAN;
		st[s] = z;
	}
	if (threadIdx.x == 0) {
		ctrl->counter = 0; ctrl->allDone = 0; ctrl->loops = 0; ctrl->maxLoops = maxLoops;
		if (arm.active) cudaGraphSetConditional(arm.handle, 1u);
	}
}

// persistent solvers ---------------------------------------------------------------------
// One cooperative launch runs a whole solve. The CTAs are co-resident (cooperative launch)
// and meet at grid barriers instead of kernel boundaries, so an iteration costs a few
// barrier round trips instead of kernel launches and the vectors stay in L2. Every barrier
// wait is bounded: when it runs out it sets Control::barErr and every CTA leaves the kernel
// (phb_solve_results then reports every system non-finite; inside a refinement the unfinished
// inner solve leaves the outer loop unconverged). Each CTA keeps its own copy of the per-system
// scalars in shared memory and reduces the per-tile partials itself, in the same fixed order
// as every other CTA, so all CTAs take the same decisions without broadcasting them.
constexpr unsigned int BARRIER_SPIN_LIMIT = 1u << 24;
constexpr unsigned int BARRIER_ERR_POLL = 1023; // spins between reads of Control::barErr

// Sense-reversing arrival counter: CTA 0 adds 2^31 - (gridDim.x - 1), every other CTA adds 1,
// so the counter's top bit flips exactly when the last CTA of a generation arrives and the
// low bits return to where they were (no reset, no second atomic). The arrival is a release
// and the poll an acquire at GPU scope; with the CTA barriers on both sides that orders every
// thread's writes before the barrier against every thread's reads after it. A CTA that has
// seen the flip does not read barErr: a CTA that gave up at this barrier had arrived at it
// (arrival comes before the wait), so the flip proves the phase complete, and the next
// barrier, where that CTA never arrives, ends everyone else's wait through barErr.
__device__ __forceinline__ unsigned int barrierArrive(unsigned int *count, unsigned int add) {
	unsigned int old;
	asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(count), "r"(add) : "memory");
	return old;
}

__device__ __forceinline__ unsigned int barrierPoll(const unsigned int *count) {
	unsigned int v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
	return v;
}

__device__ __forceinline__ bool gridBarrier(Control *ctrl, unsigned int spinLimit = BARRIER_SPIN_LIMIT) {
	__shared__ int sOk;
	__syncthreads();
	if (threadIdx.x == 0) {
		const unsigned int add = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u;
		const unsigned int old = barrierArrive(&ctrl->barCount, add);
		int ok = 1;
		for (unsigned int spins = 1; ((barrierPoll(&ctrl->barCount) ^ old) & 0x80000000u) == 0; ++spins) {
			if ((spins & BARRIER_ERR_POLL) == 0 && (spins > spinLimit || *(volatile int *)&ctrl->barErr)) {
				atomicExch(&ctrl->barErr, 1);
				ok = 0;
				break;
			}
			__nanosleep(32);
		}
		sOk = ok;
	}
	__syncthreads();
	return sOk;
}

// The bounded wait under test: every CTA but `absent` takes `rounds` grid barriers with spin
// limit `spinLimit`; the absent CTA leaves at once, so the others' waits run out, set barErr
// and end the kernel. rounds_done[0] counts the barriers CTA 0 passed.
__global__ void kBarrierProbe(Control *ctrl, int rounds, int absent, unsigned int spinLimit, int *roundsDone) {
	if ((int)blockIdx.x == absent) return;
	int done = 0;
	for (int i = 0; i < rounds; ++i) {
		if (!gridBarrier(ctrl, spinLimit)) break;
		++done;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) *roundsDone = done;
}

// Block sum of NV values written to dst[0..NV) by the first threads.
template <int NV>
__device__ __forceinline__ void blockSumTo(double (&v)[NV], double *dst) {
	__shared__ double sm[NV][NWARPS];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int q = 0; q < NV; ++q) {
		const double s = warpSum(v[q]);
		if (lane == 0) sm[q][warp] = s;
	}
	__syncthreads();
	if (threadIdx.x < NV) {
		double s = 0;
#pragma unroll
		for (int w = 0; w < NWARPS; ++w) s += sm[threadIdx.x][w];
		dst[threadIdx.x] = s;
	}
	__syncthreads();
}

// Visit this CTA's tiles with the block record staged in sB.
template <int D, typename F>
__device__ __forceinline__ void forMyTiles(const Dom<double, D> &dom, int32_t *sB, F f) {
	int staged = -1; // the block whose record sB holds (uniform over the CTA)
	for (int tile = blockIdx.x; tile < dom.ntiles; tile += gridDim.x) {
		const int b = __ldg(dom.tiles + 2 * tile);
		const int l0 = __ldg(dom.tiles + 2 * tile + 1);
		if (b != staged) {
			__syncthreads();
			if (threadIdx.x < PHB_BREC) sB[threadIdx.x] = __ldg(dom.blocks + b * PHB_BREC + threadIdx.x);
			__syncthreads();
			staged = b;
		}
		const int nc = sB[B_NX] * sB[B_NY] * (D > 2 ? sB[B_NZ] : 1);
		f(tile, l0, nc);
	}
}

// All CTAs: reduce every running system's partials (the group scheme of finalizeSystems) and
// update the CTA's state copy; returns the number of systems still running.
template <int K, int NQ, int INSTQ = -1, typename Fn>
__device__ __forceinline__ int reduceStates(const int32_t *insts, int ninst, const double *partial, SysState *sst, Fn fn) {
	constexpr int NV = NQ + 1;
	__shared__ int running;
	__shared__ double gsm[NWARPS][NV];
	if (threadIdx.x == 0) running = 0;
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int nsys = ninst * K;
	int G = NWARPS;
	while (G > 1 && G * nsys > NWARPS) G >>= 1;
	const int NG = NWARPS / G;
	const int group = warp / G, wg = warp - group * G;
	for (int base = 0; base < nsys; base += NG) {
		const int s = base + group;
		const bool act = s < nsys && sst[s].done == RUNNING;
		double a0[NV], a1[NV];
#pragma unroll
		for (int q = 0; q < NV; ++q) { a0[q] = 0; a1[q] = 0; }
		if (act) {
			const int inst = s / K, k = s - inst * K;
			const int t0 = insts[inst * PHB_IREC + I_TILESTART], tc = insts[inst * PHB_IREC + I_TILECOUNT];
			const int stride = G * 32;
			auto load = [&](int t, double *a) {
				const double *pp = partial + (size_t)(t0 + t) * K * NQ;
#pragma unroll
				for (int q = 0; q < NQ; ++q) a[q] += __ldcg(pp + k * NQ + q);
				if (INSTQ >= 0) {
#pragma unroll
					for (int kk = 0; kk < K; ++kk) a[NQ] += __ldcg(pp + kk * NQ + (INSTQ < 0 ? 0 : INSTQ));
				}
			};
			int t = wg * 32 + lane;
			for (; t + stride < tc; t += 2 * stride) { load(t, a0); load(t + stride, a1); }
			if (t < tc) load(t, a0);
		}
#pragma unroll
		for (int q = 0; q < NV; ++q) {
			const double v = warpSum(a0[q] + a1[q]);
			if (lane == 0) gsm[warp][q] = v;
		}
		__syncthreads();
		if (act && wg == 0 && lane == 0) {
			double red[NV];
#pragma unroll
			for (int q = 0; q < NV; ++q) {
				double v = 0;
				for (int w = 0; w < G; ++w) v += gsm[group * G + w][q];
				red[q] = v;
			}
			fn(sst[s], s / K, red, red[NQ]);
		}
		if (wg == 0 && lane == 0 && s < nsys && sst[s].done == RUNNING) atomicAdd(&running, 1);
		__syncthreads();
	}
	const int r = running;
	__syncthreads();
	return r;
}

// The reference stop rule of the first residual (kResidual) applied to a CTA state copy.
template <int K, bool BICG, bool STOPSTART>
__device__ __forceinline__ void residualDecision(const Dom<double, 3> *, SysState &s, double ns, const double *red, double bb,
		const phb_tolerance &tol) {
	if (tol.mode == 1) s.tol = resolveTol(tol, sqrt(bb / double(K)) * ns);
	const double crit = sqrt(red[0]) * ns;
	s.rho = red[0];
	s.restart = 1;
	s.crit = crit;
	if (!fin(crit)) { s.done = NONFINITE; s.usedIt = 0; }
	else if ((BICG || STOPSTART) ? crit < s.tol : crit == 0.0) { s.done = CONVERGED; s.usedIt = BICG ? -1 : 0; }
}

// PC: AMG-preconditioned CG (float, one right-hand side): every iteration first runs the
// V-cycle of `mg` on r, level by level between grid barriers, and takes the direction from z.
// QUADS (kCgPersistentQuads, for a finest level of at least AMG_QUAD_MIN_CELLS cells): the
// finest restriction and prolongation in their one-coarse-cell-per-thread and quad forms. It is
// a kernel of its own, so that the smaller grids' kernel keeps the compiler's register choice,
// and is held to four resident CTAs per SM (64 registers, some spills), which measured faster
// on large grids than the 128 registers the compiler takes at two CTAs per SM.
template <typename T, int D, int K, bool STOPSTART, bool PC, bool QUADS>
__device__ __forceinline__ void cgPersistentBody(const Dom<double, D> &dom, const T *__restrict__ A, const T *__restrict__ b,
		T *__restrict__ x, T *__restrict__ r, T *__restrict__ p0, T *__restrict__ p1, T *__restrict__ q, T *__restrict__ xbest,
		SysState *st, double *partial, Control *ctrl, const phb_tolerance &tol, int returnBest, int maxit, const AmgView<D> &mg) {
	static_assert(!PC || (std::is_same<T, float>::value && K == 1), "the V-cycle preconditions float single-rhs CG");
	extern __shared__ SysState sst[];
	__shared__ int32_t sB[PHB_BREC];
	__shared__ int32_t sBs[PC ? 4 : 1][PHB_BREC];
	const int nsys = dom.ninst * K;
	for (int s = threadIdx.x; s < nsys; s += blockDim.x) sst[s] = st[s];
	__syncthreads();
	const int64_t N = dom.ncells;
	// consecutive phases write alternate halves of the partials, so that a CTA that has left
	// a barrier cannot overwrite partials another CTA is still reducing
	const size_t half = (size_t)dom.ntiles * K * 3;
	int ph = 0;
	double *pp = partial;
	// r = b - A x, (r, r), (b, b)
	pp = partial + (size_t)(ph++ & 1) * half;
	forMyTiles<D>(dom, sB, [&](int tile, int l0, int nc) {
		const int inst = sB[B_INST];
		bool act[K];
#pragma unroll
		for (int k = 0; k < K; ++k) act[k] = sst[inst * K + k].done == RUNNING;
		double acc[2 * K];
#pragma unroll
		for (int k = 0; k < 2 * K; ++k) acc[k] = 0;
		tileResidual<T, D, K>(dom, sB, l0, nc, A, b, x, act, acc,
				[&](int, int64_t o, const Quad &q, const T (&rv)[4]) { st4(r + o, q.n, q.al, rv); });
		blockSumTo<2 * K>(acc, pp + (size_t)tile * 2 * K);
	});
	if (!gridBarrier(ctrl)) return;
	int running = reduceStates<K, 2, 1>(dom.insts, dom.ninst, pp, sst, [&](SysState &s, int in, const double *red, double bb) {
		residualDecision<K, false, STOPSTART>(nullptr, s, normScale(dom.insts, in), red, bb, tol);
	});
	T *pIn = p0, *pOut = p1;
	// the direction is built from z = M r when preconditioned, from r otherwise
	const T *dsrc = r;
	if constexpr (PC) dsrc = (const T *)mg.x[0];
	for (int iter = 0; running > 0 && iter <= maxit + 1; ++iter) {
		if constexpr (PC) {
			const int L = mg.nlevels;
			constexpr bool quads = QUADS;
			for (int l = 0; l + 1 < L; ++l) {
				if (l == 0 && quads) {
					for (int sub = blockIdx.x; sub < mg.lv[1].ntiles * RESTRICT1_PER_TILE; sub += gridDim.x) amgRestrictCoarseCell<D>(mg, 0, sub, sB);
				} else {
					// up to four of this CTA's sub-tiles per pass, their loads in flight together
					const int nsub = mg.lv[l + 1].ntiles * Restrict<D>::PER_TILE;
					for (int sub = blockIdx.x; sub < nsub; sub += 4 * gridDim.x)
						amgRestrictMulti<D, 4>(mg, l, sub, gridDim.x, nsub, sBs);
				}
				if (!gridBarrier(ctrl)) return;
			}
			amgCoarseRows<D>(mg, int(blockIdx.x * NWARPS + (threadIdx.x >> 5)), int(gridDim.x * NWARPS));
			if (!gridBarrier(ctrl)) return;
			for (int l = L - 2; l >= 1; --l) {
				for (int sub = blockIdx.x; sub < mg.lv[l].ntiles * AMG_SUBTILES; sub += gridDim.x) {
					const int q = sub % AMG_SUBTILES;
					amgProlongTile<D>(mg, l, sub / AMG_SUBTILES, sB, mg.x[l], q, q + 1);
				}
				if (!gridBarrier(ctrl)) return;
			}
			pp = partial + (size_t)(ph++ & 1) * half;
			for (int tile = blockIdx.x; tile < dom.ntiles; tile += gridDim.x) {
				// the finest level on quads: with the wall rows on the vector path it beats the
				// per-cell form on every grid measured (the 442,368-cell duct: 18.5 -> 16.7 ms/step)
				double acc[1] = {amgProlongQuad<D>(mg, 0, tile, sB, mg.x[0])};
				blockSumTo<1>(acc, pp + tile);
			}
			if (!gridBarrier(ctrl)) return;
			reduceStates<1, 1>(dom.insts, dom.ninst, pp, sst, [&](SysState &s, int, const double *red, double) { pcgRho(s, red[0]); });
		}
		// p' = z + beta p (z = r without preconditioner), q = A p', (p', q)
		pp = partial + (size_t)(ph++ & 1) * half;
		forMyTiles<D>(dom, sB, [&](int tile, int l0, int nc) {
			const int inst = sB[B_INST];
			bool act[K], rs[K];
			T beta[K];
#pragma unroll
			for (int k = 0; k < K; ++k) {
				const SysState &s = sst[inst * K + k];
				act[k] = s.done == RUNNING;
				rs[k] = s.restart;
				beta[k] = T(s.beta);
			}
			double acc[K];
#pragma unroll
			for (int k = 0; k < K; ++k) acc[k] = 0;
			tileCgDirection<T, D, K>(dom, sB, l0, nc, A, dsrc, pIn, pOut, q, act, rs, beta, acc);
			blockSumTo<K>(acc, pp + (size_t)tile * K);
		});
		if (!gridBarrier(ctrl)) return;
		reduceStates<K, 1>(dom.insts, dom.ninst, pp, sst, [&](SysState &s, int, const double *red, double) {
			const double alpha = s.rho / red[0];
			s.restart = 0;
			if (!fin(alpha)) { s.done = NONFINITE; s.usedIt = s.it; }
			else s.alpha = alpha;
		});
		// x += alpha p', r -= alpha q, (r, r)
		pp = partial + (size_t)(ph++ & 1) * half;
		forMyTiles<D>(dom, sB, [&](int tile, int l0, int nc) {
			double acc[K];
#pragma unroll
			for (int k = 0; k < K; ++k) acc[k] = 0;
			tileCgUpdate<T, D, K>(dom, sB, l0, nc, r, pOut, q, x, xbest, sst, acc);
			blockSumTo<K>(acc, pp + (size_t)tile * K);
		});
		if (!gridBarrier(ctrl)) return;
		running = reduceStates<K, 1>(dom.insts, dom.ninst, pp, sst, [&](SysState &s, int in, const double *red, double) {
			const double crit = sqrt(red[0]) * normScale(dom.insts, in);
			++s.it;
			s.crit = crit;
			s.saveBest = 0;
			s.usedIt = s.it - 1;
			if (!fin(crit)) { s.done = NONFINITE; return; }
			if (returnBest) {
				if (crit < s.best) { s.best = crit; s.bestIt = s.it - 1; s.saveBest = 1; }
				if (s.it > 1 && crit >= s.last) ++s.rising; else s.rising = 0;
				s.last = crit;
			}
			if (crit < s.tol) s.done = CONVERGED;
			else if (s.it >= s.maxit) s.done = MAXIT;
			else if (returnBest && s.rising >= RISING_CUTOFF) s.done = RISING;
			else if (!PC) {
				s.beta = red[0] / s.rho;
				s.rho = red[0];
				if (!fin(s.beta)) s.done = NONFINITE;
			}
		});
		T *tmp = pIn; pIn = pOut; pOut = tmp;
	}
	// systems that stopped without converging return their best iterate (kRestoreBest)
	if (xbest) {
		forMyTiles<D>(dom, sB, [&](int, int l0, int nc) {
			const int inst = sB[B_INST];
			for (int j = 0; j < CPT; ++j) {
				Cell c;
				if (!cellAt<D>(sB, l0, nc, j, c)) break;
#pragma unroll
				for (int k = 0; k < K; ++k) {
					const SysState &s = sst[inst * K + k];
					if ((s.done == MAXIT || s.done == RISING) && s.bestIt >= 0 && s.best < s.crit) {
						const int64_t o = vk<K>(c.B, c.g, k);
						x[o] = xbest[o];
					}
				}
			}
		});
	}
	if (blockIdx.x == 0) {
		__syncthreads();
		for (int s = threadIdx.x; s < nsys; s += blockDim.x) st[s] = sst[s];
	}
}

// Resident CTAs per SM that the register budget must allow. The preconditioned solve keeps
// at least three (at most 85 registers): a grid of one CTA per 1024-cell tile then stays
// co-resident up to 444 tiles (the 442,368-cell duct has 432). The plain float32 CG is bound
// by HBM on large grids and is faster with more warps in flight: four CTAs in 3D (64
// registers), five in 2D (48), which it fits without spilling. Several right-hand sides and
// float64 need more registers per thread.
template <typename T, int D, int K, bool PC>
constexpr int cgMinBlocks() {
	return PC ? 3 : (std::is_same<T, float>::value && K == 1) ? (D == 2 ? 5 : 4) : (K == 1 ? 3 : 2);
}

template <typename T, int D, int K, bool STOPSTART, bool PC = false>
__global__ void __launch_bounds__(PHB_TILE, (cgMinBlocks<T, D, K, PC>())) kCgPersistent(Dom<double, D> dom, const T *__restrict__ A, const T *__restrict__ b,
		T *__restrict__ x, T *__restrict__ r, T *__restrict__ p0, T *__restrict__ p1, T *__restrict__ q, T *__restrict__ xbest,
		SysState *st, double *partial, Control *ctrl, phb_tolerance tol, int returnBest, int maxit, AmgView<D> mg) {
	cgPersistentBody<T, D, K, STOPSTART, PC, false>(dom, A, b, x, r, p0, p1, q, xbest, st, partial, ctrl, tol, returnBest, maxit, mg);
}

template <typename T, int D, int K, bool STOPSTART>
__global__ void __launch_bounds__(PHB_TILE, 4) kCgPersistentQuads(Dom<double, D> dom, const T *__restrict__ A, const T *__restrict__ b,
		T *__restrict__ x, T *__restrict__ r, T *__restrict__ p0, T *__restrict__ p1, T *__restrict__ q, T *__restrict__ xbest,
		SysState *st, double *partial, Control *ctrl, phb_tolerance tol, int returnBest, int maxit, AmgView<D> mg) {
	cgPersistentBody<T, D, K, STOPSTART, true, true>(dom, A, b, x, r, p0, p1, q, xbest, st, partial, ctrl, tol, returnBest, maxit, mg);
}

template <typename T, int D, int K>
__global__ void __launch_bounds__(PHB_TILE) kBicgPersistent(Dom<double, D> dom, const T *__restrict__ A, const T *__restrict__ b,
		T *__restrict__ x, T *__restrict__ r, T *__restrict__ r0, T *__restrict__ p0, T *__restrict__ p1, T *__restrict__ v0,
		T *__restrict__ v1, T *__restrict__ t, SysState *st, double *partial, Control *ctrl, phb_tolerance tol, int maxit) {
	extern __shared__ SysState sst[];
	__shared__ int32_t sB[PHB_BREC];
	const int nsys = dom.ninst * K;
	for (int s = threadIdx.x; s < nsys; s += blockDim.x) sst[s] = st[s];
	__syncthreads();
	const int64_t N = dom.ncells;
	// consecutive phases write alternate halves of the partials, so that a CTA that has left
	// a barrier cannot overwrite partials another CTA is still reducing
	const size_t half = (size_t)dom.ntiles * K * 3;
	int ph = 0;
	double *pp = partial;
	pp = partial + (size_t)(ph++ & 1) * half;
	forMyTiles<D>(dom, sB, [&](int tile, int l0, int nc) {
		const int inst = sB[B_INST];
		bool act[K];
#pragma unroll
		for (int k = 0; k < K; ++k) act[k] = sst[inst * K + k].done == RUNNING;
		double acc[2 * K];
#pragma unroll
		for (int k = 0; k < 2 * K; ++k) acc[k] = 0;
		tileResidual<T, D, K>(dom, sB, l0, nc, A, b, x, act, acc, [&](int, int64_t o, const Quad &q, const T (&rv)[4]) {
			st4(r + o, q.n, q.al, rv);
			st4(r0 + o, q.n, q.al, rv);
		});
		blockSumTo<2 * K>(acc, pp + (size_t)tile * 2 * K);
	});
	if (!gridBarrier(ctrl)) return;
	int running = reduceStates<K, 2, 1>(dom.insts, dom.ninst, pp, sst, [&](SysState &s, int in, const double *red, double bb) {
		residualDecision<K, true, true>(nullptr, s, normScale(dom.insts, in), red, bb, tol);
	});
	T *pIn = p0, *pOut = p1, *vIn = v0, *vOut = v1;
	for (int iter = 0; running > 0 && iter <= maxit + 1; ++iter) {
		// p = r + beta (p - omega v), v = A p, (r0, v)
		pp = partial + (size_t)(ph++ & 1) * half;
		forMyTiles<D>(dom, sB, [&](int tile, int l0, int nc) {
			const int inst = sB[B_INST];
			bool act[K], rs[K];
			T beta[K], omega[K];
#pragma unroll
			for (int k = 0; k < K; ++k) {
				const SysState &s = sst[inst * K + k];
				act[k] = s.done == RUNNING;
				rs[k] = s.restart;
				beta[k] = T(s.beta);
				omega[k] = T(s.omega);
			}
			double acc[K];
#pragma unroll
			for (int k = 0; k < K; ++k) acc[k] = 0;
			tileBicgV<T, D, K>(dom, sB, l0, nc, A, r, pIn, vIn, pOut, vOut, r0, act, rs, beta, omega, acc);
			blockSumTo<K>(acc, pp + (size_t)tile * K);
		});
		if (!gridBarrier(ctrl)) return;
		reduceStates<K, 1>(dom.insts, dom.ninst, pp, sst, [&](SysState &s, int, const double *red, double) {
			const double alpha = s.rho / red[0];
			s.restart = 0;
			if (!fin(alpha)) { s.done = NONFINITE; s.usedIt = s.it; }
			else s.alpha = alpha;
		});
		// s = r - alpha v, t = A s, (t,s), (t,t), (s,s)
		pp = partial + (size_t)(ph++ & 1) * half;
		forMyTiles<D>(dom, sB, [&](int tile, int l0, int nc) {
			const int inst = sB[B_INST];
			bool act[K];
			T alpha[K];
#pragma unroll
			for (int k = 0; k < K; ++k) {
				const SysState &s = sst[inst * K + k];
				act[k] = s.done == RUNNING;
				alpha[k] = T(s.alpha);
			}
			double acc[3 * K];
#pragma unroll
			for (int k = 0; k < 3 * K; ++k) acc[k] = 0;
			tileBicgT<T, D, K>(dom, sB, l0, nc, A, r, vOut, t, act, alpha, acc);
			blockSumTo<3 * K>(acc, pp + (size_t)tile * 3 * K);
		});
		if (!gridBarrier(ctrl)) return;
		reduceStates<K, 3>(dom.insts, dom.ninst, pp, sst, [&](SysState &s, int in, const double *red, double) {
			const double critS = sqrt(red[2]) * normScale(dom.insts, in);
			s.halfCrit = critS;
			if (!fin(critS)) { s.done = NONFINITE; s.crit = critS; s.usedIt = s.it; }
			else if (critS < s.tol) { s.halfDone = 1; s.omega = 0.0; }
			else {
				const double omega = red[0] / red[1];
				if (!fin(omega)) { s.done = NONFINITE; s.crit = critS; s.usedIt = s.it; }
				else s.omega = omega;
			}
		});
		// x += alpha p + omega s, r = s - omega t, (r0, r), (r, r)
		pp = partial + (size_t)(ph++ & 1) * half;
		forMyTiles<D>(dom, sB, [&](int tile, int l0, int nc) {
			double acc[2 * K];
#pragma unroll
			for (int k = 0; k < 2 * K; ++k) acc[k] = 0;
			tileBicgUpdate<T, D, K>(dom, sB, l0, nc, r, r0, pOut, vOut, t, x, sst, acc);
			blockSumTo<2 * K>(acc, pp + (size_t)tile * 2 * K);
		});
		if (!gridBarrier(ctrl)) return;
		running = reduceStates<K, 2>(dom.insts, dom.ninst, pp, sst, [&](SysState &s, int in, const double *red, double) {
			if (s.halfDone) { s.done = CONVERGED; s.crit = s.halfCrit; s.usedIt = s.it; return; }
			const double crit = sqrt(red[1]) * normScale(dom.insts, in);
			s.crit = crit;
			if (!fin(crit)) { s.done = NONFINITE; s.usedIt = s.it; }
			else if (crit < s.tol) { s.done = CONVERGED; s.usedIt = s.it + 1; }
			else {
				++s.it;
				s.usedIt = s.it - 1;
				const double beta = (red[0] / s.rho) * (s.alpha / s.omega);
				s.rho = red[0];
				s.beta = beta;
				if (!fin(beta)) s.done = NONFINITE;
				else if (s.it >= s.maxit) s.done = MAXIT;
			}
		});
		T *tmp = pIn; pIn = pOut; pOut = tmp;
		tmp = vIn; vIn = vOut; vOut = tmp;
	}
	if (blockIdx.x == 0) {
		__syncthreads();
		for (int s = threadIdx.x; s < nsys; s += blockDim.x) st[s] = sst[s];
	}
}

// host side --------------------------------------------------------------------------------
static size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Dom::vec4 of a launch: every operand on a 16-byte boundary and a cell count that keeps the
// stencil's slot rows aligned
static int vec4Ok(const phb_domain *dom, std::initializer_list<const void *> ptrs) {
	if (dom->ncells % 4) return 0;
	for (const void *p : ptrs)
		if (p && ((uintptr_t)p & 15)) return 0;
	return 1;
}

struct Layout {
	size_t off[12];
	size_t total;
};

static int vecCount(int kind) { return kind == 0 ? 5 : 7; } // CG: r q p0 p1 xbest; BiCG: r r0 p0 p1 v0 v1 t

static Layout solveLayout(const phb_domain *dom, int kind, int vecBytes, int nrhs) {
	Layout L;
	size_t o = 0;
	const size_t vb = align256((size_t)dom->ncells * nrhs * vecBytes);
	for (int i = 0; i < vecCount(kind); ++i) { L.off[i] = o; o += vb; }
	L.off[10] = o; // partials: two halves of up to 3 values per tile and right-hand side
	o += align256((size_t)dom->ntiles * nrhs * 3 * 2 * sizeof(double));
	L.total = o;
	return L;
}

struct StateLayout { size_t ctrl, st, ctrl2, st2, total; };
static StateLayout stateLayout(const phb_domain *dom, int nrhs) {
	StateLayout L;
	const size_t nsys = (size_t)dom->ninst * nrhs;
	L.ctrl = 0;
	L.st = 256;
	L.ctrl2 = align256(L.st + nsys * sizeof(SysState));
	L.st2 = L.ctrl2 + 256;
	L.total = align256(L.st2 + nsys * sizeof(SysState));
	return L;
}

// capture helpers ----------------------------------------------------------------------------
struct Streams { cudaStream_t s[3] = {nullptr, nullptr, nullptr}; int device = -1; };
static thread_local Streams tlStreams;
static int getStreams(Streams *&out) {
	int dev;
	PHB_CUDA(cudaGetDevice(&dev));
	if (tlStreams.device != dev) {
		for (auto &s : tlStreams.s) {
			if (s) cudaStreamDestroy(s);
			s = nullptr;
		}
		for (auto &s : tlStreams.s) PHB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
		tlStreams.device = dev;
	}
	out = &tlStreams;
	return PHB_OK;
}

// Create the condition handle of a WHILE loop on the graph `cap` is capturing. The kernel
// launched just before the loop sets it (armCondition), so that a loop nested in another
// conditional body is re-armed on every pass of the outer body: a handle's default value is
// only applied when the graph that owns it is launched.
static int createCondition(cudaStream_t cap, cudaGraphConditionalHandle *handle) {
	cudaStreamCaptureStatus status;
	cudaGraph_t graph;
	PHB_CUDA(cudaStreamGetCaptureInfo(cap, &status, nullptr, &graph, nullptr, nullptr));
	if (status != cudaStreamCaptureStatusActive) return setError(PHB_ERR_STATE, "createCondition: stream is not capturing");
	PHB_CUDA(cudaGraphConditionalHandleCreate(handle, graph, 1, cudaGraphCondAssignDefault));
	return PHB_OK;
}

// Add a conditional WHILE node on `handle` to the graph `cap` is capturing and capture
// `body` into it on `bodyStream`; the body's last kernel sets the condition.
static int addWhile(cudaStream_t cap, cudaStream_t bodyStream, cudaGraphConditionalHandle handle,
		const std::function<int(cudaStream_t, LoopCond)> &body) {
	cudaStreamCaptureStatus status;
	cudaGraph_t graph;
	const cudaGraphNode_t *deps = nullptr;
	size_t ndeps = 0;
	PHB_CUDA(cudaStreamGetCaptureInfo(cap, &status, nullptr, &graph, &deps, &ndeps));
	if (status != cudaStreamCaptureStatusActive) return setError(PHB_ERR_STATE, "addWhile: stream is not capturing");
	cudaGraphNodeParams params = {};
	params.type = cudaGraphNodeTypeConditional;
	params.conditional.handle = handle;
	params.conditional.type = cudaGraphCondTypeWhile;
	params.conditional.size = 1;
	cudaGraphNode_t node;
	PHB_CUDA(cudaGraphAddNode(&node, graph, deps, ndeps, &params));
	PHB_CUDA(cudaStreamUpdateCaptureDependencies(cap, &node, 1, cudaStreamSetCaptureDependencies));
	cudaGraph_t bodyGraph = params.conditional.phGraph_out[0];
	PHB_CUDA(cudaStreamBeginCaptureToGraph(bodyStream, bodyGraph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
	const int st = body(bodyStream, LoopCond{handle, 1});
	cudaGraph_t ended;
	const cudaError_t e = cudaStreamEndCapture(bodyStream, &ended);
	if (st != PHB_OK) return st;
	PHB_CUDA(e);
	return PHB_OK;
}

struct CachedGraph { cudaGraphExec_t exec; };
static std::mutex gMutex;
static std::map<std::string, CachedGraph> gGraphs;

static int releaseGraphsLocked() {
	for (auto &kv : gGraphs) cudaGraphExecDestroy(kv.second.exec);
	gGraphs.clear();
	return PHB_OK;
}

// Run `emit` (which records work on a capturing stream) either spliced into the caller's
// ongoing capture, or as a cached graph launched on `stream`.
static int runGraph(cudaStream_t stream, const std::string &key, const std::function<int(cudaStream_t, Streams &)> &emit) {
	Streams *ss;
	int rc = getStreams(ss);
	if (rc) return rc;
	cudaStreamCaptureStatus status;
	PHB_CUDA(cudaStreamIsCapturing(stream, &status));
	if (status == cudaStreamCaptureStatusActive) return emit(stream, *ss);
	std::lock_guard<std::mutex> lock(gMutex);
	auto it = gGraphs.find(key);
	if (it == gGraphs.end()) {
		if (gGraphs.size() >= 64) releaseGraphsLocked();
		PHB_CUDA(cudaStreamBeginCapture(ss->s[0], cudaStreamCaptureModeThreadLocal));
		rc = emit(ss->s[0], *ss);
		cudaGraph_t graph = nullptr;
		const cudaError_t e = cudaStreamEndCapture(ss->s[0], &graph);
		if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
		PHB_CUDA(e);
		CachedGraph cg;
		const cudaError_t ei = cudaGraphInstantiate(&cg.exec, graph, 0);
		cudaGraphDestroy(graph);
		PHB_CUDA(ei);
		it = gGraphs.emplace(key, cg).first;
	}
	PHB_CUDA(cudaGraphLaunch(it->second.exec, stream));
	return PHB_OK;
}

template <typename A, typename B>
static std::string makeKey(const char *tag, const A &a, const B &b) {
	std::string k(tag);
	k.append(reinterpret_cast<const char *>(&a), sizeof(A));
	k.append(reinterpret_cast<const char *>(&b), sizeof(B));
	return k;
}

static int gridFor(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

static int numSMs() {
	static int cache[64] = {0};
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
	if (!cache[dev]) {
		int v = 0;
		if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
		cache[dev] = v;
	}
	return cache[dev];
}

// A persistent solve: kInit, then one cooperative launch of the whole iteration (the grid is
// sized so that every CTA is resident; the launch fails rather than deadlocks otherwise).
template <typename T, int D, int K>
static int launchPersistent(const phb_domain *dom, const phb_solve *sv, cudaStream_t s, bool stopStart, int fromInner) {
	Dom<double, D> dm(*dom);
	const Layout L = solveLayout(dom, sv->kind, sizeof(T), K);
	const StateLayout SL = stateLayout(dom, K);
	char *w = (char *)sv->work;
	char *sb = (char *)sv->state;
	Control *ctrl = (Control *)(sb + SL.ctrl);
	SysState *st = (SysState *)(sb + SL.st);
	double *partial = (double *)(w + L.off[10]);
	const T *A = (const T *)sv->A;
	const T *b = (const T *)sv->b;
	T *x = (T *)sv->x;
	dm.vec4 = vec4Ok(dom, {A, b, x, w});
	const int nsys = dom->ninst * K;
	const size_t smem = (size_t)nsys * sizeof(SysState);
	if (smem > 160 * 1024) return setError(PHB_ERR_RANGE, "persistent solve: too many systems for the per-CTA state copy");
	const int maxit = std::max(1, sv->maxit);
	kInit<<<1, 256, 0, s>>>(st, nsys, sv->tol, fromInner, maxit, ctrl, maxit / 2 + 2);
	PHB_CUDA(cudaGetLastError());
	cudaLaunchConfig_t cfg = {};
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cfg.blockDim = dim3(PHB_TILE);
	cfg.dynamicSmemBytes = smem;
	cfg.stream = s;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	auto grid = [&](const void *kern) -> int {
		if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		int perSM = 0;
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, PHB_TILE, smem) != cudaSuccess || perSM < 1) perSM = 1;
		if (sv->ctas_per_sm > 0) perSM = std::min(perSM, sv->ctas_per_sm); // a tuned, smaller grid
		return std::max(1, std::min(dom->ntiles, perSM * numSMs()));
	};
	if (sv->kind == 0) {
		T *r = (T *)(w + L.off[0]), *q = (T *)(w + L.off[1]), *p0 = (T *)(w + L.off[2]), *p1 = (T *)(w + L.off[3]);
		T *xbest = sv->return_best ? (T *)(w + L.off[4]) : nullptr;
		AmgView<D> mg = {};
		auto launch = [&](auto kern) -> int {
			cfg.gridDim = dim3(grid((const void *)kern));
			PHB_CUDA(cudaLaunchKernelEx(&cfg, kern, dm, A, b, x, r, p0, p1, q, xbest, st, partial, ctrl, sv->tol, sv->return_best, maxit, mg));
			return PHB_OK;
		};
		if constexpr (std::is_same<T, float>::value && K == 1) {
			if (sv->amg) {
				mg = makeAmgView<D>(*sv->amg, (const float *)r, sv->amg->levels[0].x);
				if (amgFineQuads(mg))
					return stopStart ? launch(kCgPersistentQuads<T, D, K, true>) : launch(kCgPersistentQuads<T, D, K, false>);
				return stopStart ? launch(kCgPersistent<T, D, K, true, true>) : launch(kCgPersistent<T, D, K, false, true>);
			}
		}
		return stopStart ? launch(kCgPersistent<T, D, K, true>) : launch(kCgPersistent<T, D, K, false>);
	}
	T *r = (T *)(w + L.off[0]), *r0 = (T *)(w + L.off[1]), *p0 = (T *)(w + L.off[2]), *p1 = (T *)(w + L.off[3]);
	T *v0 = (T *)(w + L.off[4]), *v1 = (T *)(w + L.off[5]), *t = (T *)(w + L.off[6]);
	auto kern = kBicgPersistent<T, D, K>;
	cfg.gridDim = dim3(grid((const void *)kern));
	PHB_CUDA(cudaLaunchKernelEx(&cfg, kern, dm, A, b, x, r, r0, p0, p1, v0, v1, t, st, partial, ctrl, sv->tol, maxit));
	return PHB_OK;
}

// the Krylov loop for one solve, recorded on `s`
template <typename T, int D, int K>
static int emitSolve(const phb_domain *dom, const phb_solve *sv, cudaStream_t s, Streams &ss, int useGraph, bool stopStart, int fromInner = 0) {
	if (sv->use_graph >= 2) return launchPersistent<T, D, K>(dom, sv, s, stopStart, fromInner);
	Dom<double, D> dm(*dom);
	const Layout L = solveLayout(dom, sv->kind, sizeof(T), K);
	const StateLayout SL = stateLayout(dom, K);
	char *w = (char *)sv->work;
	char *sb = (char *)sv->state;
	Control *ctrl = (Control *)(sb + SL.ctrl);
	SysState *st = (SysState *)(sb + SL.st);
	double *partial = (double *)(w + L.off[10]);
	const T *A = (const T *)sv->A;
	const T *b = (const T *)sv->b;
	T *x = (T *)sv->x;
	dm.vec4 = vec4Ok(dom, {A, b, x, w});
	const int nsys = dom->ninst * K;
	const int tiles = dom->ntiles;
	const int maxit = std::max(1, sv->maxit);
	if (sv->kind == 0) {
		T *r = (T *)(w + L.off[0]), *q = (T *)(w + L.off[1]), *p0 = (T *)(w + L.off[2]), *p1 = (T *)(w + L.off[3]);
		T *xbest = sv->return_best ? (T *)(w + L.off[4]) : nullptr;
		const int maxLoops = maxit / 2 + 2;
		LoopCond arm{0, 0};
		if (useGraph) {
			const int rc0 = createCondition(s, &arm.handle);
			if (rc0) return rc0;
			arm.active = 1;
		}
		kInit<<<1, 256, 0, s>>>(st, nsys, sv->tol, fromInner, maxit, ctrl, maxLoops);
		if (stopStart) kResidual<T, D, K, false, true><<<tiles, PHB_TILE, 0, s>>>(dm, A, b, x, r, nullptr, st, partial, ctrl, sv->tol, arm);
		else kResidual<T, D, K, false, false><<<tiles, PHB_TILE, 0, s>>>(dm, A, b, x, r, nullptr, st, partial, ctrl, sv->tol, arm);
		int rc = checkLaunch("kResidual");
		if (rc) return rc;
		// preconditioned (float, one right-hand side): V-cycle on r down to level 1, then level
		// 0's prolongation with (r, z) and beta, and the direction taken from z
		bool pc = false;
		AmgView<D> mg = {};
		const T *dsrc = r;
		if constexpr (std::is_same<T, float>::value && K == 1) {
			if (sv->amg) {
				pc = true;
				mg = makeAmgView<D>(*sv->amg, (const float *)r, sv->amg->levels[0].x);
				dsrc = (const T *)mg.x[0];
			}
		}
		auto body = [&](cudaStream_t bs, LoopCond lc) -> int {
			for (int half = 0; half < 2; ++half) {
				T *pIn = half == 0 ? p0 : p1, *pOut = half == 0 ? p1 : p0;
				LoopCond l2 = lc;
				l2.active = half == 1 ? lc.active : 0;
				if (pc) {
					PHB_CUDA(launchAmgCycle<D>(mg, bs, 1));
					kPcgPrecond<D><<<tiles, PHB_TILE, 0, bs>>>(dm, mg, st, partial, ctrl);
					kCgDirection<T, D, K><<<tiles, PHB_TILE, 0, bs>>>(dm, A, dsrc, pIn, pOut, q, st, partial, ctrl);
					kCgUpdate<T, D, K, true><<<tiles, PHB_TILE, 0, bs>>>(dm, r, pOut, q, x, xbest, st, partial, ctrl, sv->return_best, l2);
				} else {
					kCgDirection<T, D, K><<<tiles, PHB_TILE, 0, bs>>>(dm, A, r, pIn, pOut, q, st, partial, ctrl);
					kCgUpdate<T, D, K><<<tiles, PHB_TILE, 0, bs>>>(dm, r, pOut, q, x, xbest, st, partial, ctrl, sv->return_best, l2);
				}
			}
			return checkLaunch("CG body");
		};
		if (useGraph) { rc = addWhile(s, ss.s[useGraph == 2 ? 2 : 1], arm.handle, body); if (rc) return rc; }
		else {
			// host loop (no graph): poll allDone every check_every iterations
			int *hflag = nullptr;
			PHB_CUDA(cudaMallocHost(&hflag, sizeof(int)));
			const int chk = std::max(1, sv->check_every);
			for (int loops = 0; loops < maxLoops; loops += chk) {
				for (int i = 0; i < chk; ++i) { rc = body(s, LoopCond{0, 0}); if (rc) break; }
				if (rc) break;
				cudaMemcpyAsync(hflag, &ctrl->allDone, sizeof(int), cudaMemcpyDeviceToHost, s);
				cudaStreamSynchronize(s);
				if (*hflag) break;
			}
			cudaFreeHost(hflag);
			if (rc) return rc;
		}
		if (xbest) kRestoreBest<T, K><<<gridFor(dom->ncells * K), 256, 0, s>>>(dom->insts, dom->ninst, dom->ncells, x, xbest, st);
		return checkLaunch("CG epilogue");
	}
	T *r = (T *)(w + L.off[0]), *r0 = (T *)(w + L.off[1]), *p0 = (T *)(w + L.off[2]), *p1 = (T *)(w + L.off[3]);
	T *v0 = (T *)(w + L.off[4]), *v1 = (T *)(w + L.off[5]), *t = (T *)(w + L.off[6]);
	const int maxLoops = maxit / 2 + 2;
	LoopCond arm{0, 0};
	if (useGraph) {
		const int rc0 = createCondition(s, &arm.handle);
		if (rc0) return rc0;
		arm.active = 1;
	}
	kInit<<<1, 256, 0, s>>>(st, nsys, sv->tol, fromInner, maxit, ctrl, maxLoops);
	kResidual<T, D, K, true, true><<<tiles, PHB_TILE, 0, s>>>(dm, A, b, x, r, r0, st, partial, ctrl, sv->tol, arm);
	int rc = checkLaunch("kResidual");
	if (rc) return rc;
	auto body = [&](cudaStream_t bs, LoopCond lc) -> int {
		for (int half = 0; half < 2; ++half) {
			T *pIn = half == 0 ? p0 : p1, *pOut = half == 0 ? p1 : p0;
			T *vIn = half == 0 ? v0 : v1, *vOut = half == 0 ? v1 : v0;
			kBicgV<T, D, K><<<tiles, PHB_TILE, 0, bs>>>(dm, A, r, pIn, vIn, pOut, vOut, r0, st, partial, ctrl);
			kBicgT<T, D, K><<<tiles, PHB_TILE, 0, bs>>>(dm, A, r, vOut, t, st, partial, ctrl);
			LoopCond l2 = lc;
			l2.active = half == 1 ? lc.active : 0;
			kBicgUpdate<T, D, K><<<tiles, PHB_TILE, 0, bs>>>(dm, r, r0, pOut, vOut, t, x, st, partial, ctrl, l2);
		}
		return checkLaunch("BiCGStab body");
	};
	if (useGraph) return addWhile(s, ss.s[useGraph == 2 ? 2 : 1], arm.handle, body);
	int *hflag = nullptr;
	PHB_CUDA(cudaMallocHost(&hflag, sizeof(int)));
	const int chk = std::max(1, sv->check_every);
	for (int loops = 0; loops < maxLoops; loops += chk) {
		for (int i = 0; i < chk; ++i) { rc = body(s, LoopCond{0, 0}); if (rc) break; }
		if (rc) break;
		cudaMemcpyAsync(hflag, &ctrl->allDone, sizeof(int), cudaMemcpyDeviceToHost, s);
		cudaStreamSynchronize(s);
		if (*hflag) break;
	}
	cudaFreeHost(hflag);
	return rc;
}

// Y[v] = A X[v], v < nvec, for float64 vectors of one component (stride values apart): the
// products of the basis of a projected initial guess with the system matrix. The centre and
// face terms are summed in the order of the solvers' own products.
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kStencilApply(Dom<double, D> dom, const double *__restrict__ A,
		const double *__restrict__ X, double *__restrict__ Y, int nvec, int64_t stride) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	Quad q;
	quadAt<D, 1>(dom.vec4, sB, l0_, nc_, q);
	bool act[1] = {true};
	for (int v = 0; v < nvec; ++v) {
		FX<double> fx[1];
		fx[0].x = X + v * stride;
		double y[1][4], f[1][4];
		quadApply<double, D, 1>(dom, A, q, act, fx, y, f);
		st4(Y + v * stride + vk<1>(q.B, q.g, 0), q.n, q.al, y[0]);
	}
}

// The coefficients of a Galerkin projection, one CTA: G (m x m, row-major, the Gram matrix
// D A D^T of the basis rows) alpha = c. Jacobi-scaled (s_i = |G_ii|^-1/2), the diagonal
// raised by reg relative to the scaled unit diagonal, Gaussian elimination with partial
// pivoting; a basis row whose pivot falls below 1e-14 of the largest gets coefficient 0, and
// so does every row when a value is not finite (the guess is then the zero vector's
// projection: alpha = 0).
constexpr int PROJ_MAX = 16;
__global__ void kProjectionSolve(const double *__restrict__ G, const double *__restrict__ c, int m, double reg,
		double *__restrict__ alpha) {
	__shared__ double M[PROJ_MAX][PROJ_MAX + 1];
	__shared__ double sc[PROJ_MAX];
	const int t = threadIdx.x;
	if (t < m) {
		const double d = fabs(G[t * m + t]);
		sc[t] = d > 0 && isfinite(d) ? rsqrt(d) : 0.0;
	}
	__syncthreads();
	for (int e = t; e < m * (m + 1); e += blockDim.x) {
		const int i = e / (m + 1), j = e - i * (m + 1);
		double v = j < m ? G[i * m + j] * sc[i] * sc[j] : c[i] * sc[i];
		if (j == i) v += (G[i * m + i] < 0 ? -reg : reg);
		M[i][j] = v;
	}
	__syncthreads();
	if (t == 0) {
		bool ok = true;
		double big = 0;
		for (int i = 0; i < m; ++i) big = fmax(big, fabs(M[i][i]));
		bool skip[PROJ_MAX];
		for (int i = 0; i < m; ++i) skip[i] = false;
		for (int k = 0; k < m && ok; ++k) {
			int p = k;
			for (int i = k + 1; i < m; ++i) if (fabs(M[i][k]) > fabs(M[p][k])) p = i;
			if (p != k) {
				for (int j = 0; j <= m; ++j) { const double tmp = M[k][j]; M[k][j] = M[p][j]; M[p][j] = tmp; }
			}
			if (!(fabs(M[k][k]) > 1e-14 * big)) { skip[k] = true; continue; }
			for (int i = k + 1; i < m; ++i) {
				const double f = M[i][k] / M[k][k];
				for (int j = k; j <= m; ++j) M[i][j] -= f * M[k][j];
			}
		}
		double x[PROJ_MAX];
		for (int k = m - 1; k >= 0; --k) {
			if (skip[k]) { x[k] = 0; continue; }
			double v = M[k][m];
			for (int j = k + 1; j < m; ++j) v -= M[k][j] * x[j];
			x[k] = v / M[k][k];
			if (!isfinite(x[k])) ok = false;
		}
		for (int i = 0; i < m; ++i) alpha[i] = ok ? x[i] * sc[i] : 0.0;
	}
}

// G[i][j] = sum_c V[i][c] Y[j][c] and g[i] = sum_c V[i][c] b[c] (i, j < m): each CTA stages
// chunks of GRAM_CHUNK cells of the m rows of V, the m rows of Y and b in shared memory (rows
// padded by one value against bank conflicts), each thread accumulates (i, j) pairs over its
// CTA's chunks and adds them atomically into G and g, which the caller zeroes.
constexpr int GRAM_CHUNK = 128;
__global__ void __launch_bounds__(256) kProjectionGram(const double *__restrict__ V, const double *__restrict__ Y,
		const double *__restrict__ b, int m, int64_t n, int64_t stride, double *__restrict__ G, double *__restrict__ g) {
	__shared__ double sv[PROJ_MAX][GRAM_CHUNK + 1];
	__shared__ double sy[PROJ_MAX + 1][GRAM_CHUNK + 1];
	const int npair = m * m + m;
	constexpr int PAIRS = (PROJ_MAX * PROJ_MAX + PROJ_MAX + 255) / 256;
	double acc[PAIRS];
#pragma unroll
	for (int q = 0; q < PAIRS; ++q) acc[q] = 0;
	for (int64_t base = (int64_t)blockIdx.x * GRAM_CHUNK; base < n; base += (int64_t)gridDim.x * GRAM_CHUNK) {
		const int64_t rest = n - base;
		const int len = rest < GRAM_CHUNK ? (int)rest : GRAM_CHUNK;
		for (int e = threadIdx.x; e < (2 * m + 1) * GRAM_CHUNK; e += blockDim.x) {
			const int r = e / GRAM_CHUNK, k = e - r * GRAM_CHUNK;
			double v = 0;
			if (k < len) v = r < m ? V[r * stride + base + k] : (r < 2 * m ? Y[(r - m) * stride + base + k] : b[base + k]);
			if (r < m) sv[r][k] = v;
			else sy[r - m][k] = v;
		}
		__syncthreads();
#pragma unroll
		for (int q = 0; q < PAIRS; ++q) {
			const int p = threadIdx.x + q * 256;
			if (p < npair) {
				const int i = p < m * m ? p / m : p - m * m, j = p < m * m ? p - (p / m) * m : m;
				double a = acc[q];
				for (int k = 0; k < len; ++k) a = fma(sv[i][k], sy[j][k], a);
				acc[q] = a;
			}
		}
		__syncthreads();
	}
#pragma unroll
	for (int q = 0; q < PAIRS; ++q) {
		const int p = threadIdx.x + q * 256;
		if (p < npair) atomicAdd(p < m * m ? G + p : g + (p - m * m), acc[q]);
	}
}

#define PHB_SOLVE_DISPATCH(DIMS, VEC, K, ...)                                                   \
	do {                                                                                        \
		if ((DIMS) == 2 && (VEC) == PHB_F64 && (K) == 1) { using T = double; constexpr int D = 2, KK = 1; __VA_ARGS__; } \
		else if ((DIMS) == 2 && (VEC) == PHB_F64 && (K) == 2) { using T = double; constexpr int D = 2, KK = 2; __VA_ARGS__; } \
		else if ((DIMS) == 3 && (VEC) == PHB_F64 && (K) == 1) { using T = double; constexpr int D = 3, KK = 1; __VA_ARGS__; } \
		else if ((DIMS) == 3 && (VEC) == PHB_F64 && (K) == 3) { using T = double; constexpr int D = 3, KK = 3; __VA_ARGS__; } \
		else if ((DIMS) == 2 && (VEC) == PHB_F32 && (K) == 1) { using T = float; constexpr int D = 2, KK = 1; __VA_ARGS__; } \
		else if ((DIMS) == 2 && (VEC) == PHB_F32 && (K) == 2) { using T = float; constexpr int D = 2, KK = 2; __VA_ARGS__; } \
		else if ((DIMS) == 3 && (VEC) == PHB_F32 && (K) == 1) { using T = float; constexpr int D = 3, KK = 1; __VA_ARGS__; } \
		else if ((DIMS) == 3 && (VEC) == PHB_F32 && (K) == 3) { using T = float; constexpr int D = 3, KK = 3; __VA_ARGS__; } \
		else return setError(PHB_ERR_ARG, "unsupported dims/dtype/nrhs combination");            \
	} while (0)

} // namespace phb

using namespace phb;

extern "C" int64_t phb_solve_work_bytes(const phb_domain *dom, int kind, int vec_dtype, int nrhs) {
	if (!dom) return -1;
	return (int64_t)solveLayout(dom, kind, vec_dtype == PHB_F64 ? 8 : 4, nrhs).total;
}
extern "C" int64_t phb_solve_state_bytes(const phb_domain *dom, int nrhs) {
	if (!dom) return -1;
	return (int64_t)stateLayout(dom, nrhs).total;
}

// BiCGStab on instances of at least 2^23 cells runs as per-phase kernels in a CUDA graph even in
// the persistent mode: at that size the separate kernels, each at its own full occupancy, move
// the iteration's bytes faster than the cooperative kernel (measured on one B200 with float32
// iterations: 0.52 against 0.44 of HBM on 256^3, 0.57 against 0.52 on 4096^2); CG keeps the
// persistent kernel (0.62 against 0.53).
static bool bicgPrefersGraph(const phb_domain *dom, int kind) {
	return kind == 1 && dom->ninst > 0 && dom->ncells / dom->ninst >= (int64_t(1) << 23);
}

extern "C" int phb_solve_run(const phb_domain *dom, const phb_solve *s_in, phb_stream stream) {
	phb_solve sAdj;
	const phb_solve *s = s_in;
	if (s_in && dom && s_in->use_graph == 2 && bicgPrefersGraph(dom, s_in->kind)) {
		sAdj = *s_in;
		sAdj.use_graph = 1;
		s = &sAdj;
	}
	if (!dom || !s || !s->A || !s->b || !s->x || !s->work || !s->state || (s->tol.mode == 2 && !s->tol.values)) return setError(PHB_ERR_ARG, "phb_solve_run: null argument");
	if (s->vec_dtype != s->mat_dtype) return setError(PHB_ERR_ARG, "phb_solve_run: matrix and vector dtype must match");
	if (s->kind != 0 && s->kind != 1) return setError(PHB_ERR_ARG, "phb_solve_run: kind must be 0 (CG) or 1 (BiCGStab)");
	if (s->amg) {
		if (s->kind != 0 || s->vec_dtype != PHB_F32 || s->nrhs != 1) return setError(PHB_ERR_ARG, "phb_solve_run: the AMG preconditioner takes float32 CG with one right-hand side");
		const int rc = phbCheckAmg(s->amg);
		if (rc) return rc;
		if (s->amg->levels[0].dom.ncells != dom->ncells || !s->amg->levels[0].x) return setError(PHB_ERR_ARG, "phb_solve_run: hierarchy does not match the domain");
	}
	if (dom->ntiles == 0) return PHB_OK;
	cudaStream_t st = (cudaStream_t)stream;
	std::string key = makeKey("solve", *dom, *s);
	if (s->amg) key.append(reinterpret_cast<const char *>(s->amg), sizeof(phb_amg));
	PHB_SOLVE_DISPATCH(dom->dims, s->vec_dtype, s->nrhs, {
		if (s->use_graph != 1) {
			Streams *ss; int rc = getStreams(ss); if (rc) return rc;
			return emitSolve<T, D, KK>(dom, s, st, *ss, 0, false);
		}
		return runGraph(st, key, [&](cudaStream_t cs, Streams &ss) { return emitSolve<T, D, KK>(dom, s, cs, ss, 1, false); });
	});
	return PHB_OK;
}

extern "C" int phb_solve_results(const phb_domain *dom, const phb_solve *s, phb_solve_result *out, phb_stream stream) {
	if (!dom || !s || !out || !s->state) return setError(PHB_ERR_ARG, "phb_solve_results: null argument");
	const int nsys = dom->ninst * s->nrhs;
	std::vector<SysState> h(nsys);
	const StateLayout SL = stateLayout(dom, s->nrhs);
	Control c{};
	PHB_CUDA(cudaMemcpyAsync(h.data(), (char *)s->state + SL.st, nsys * sizeof(SysState), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
	PHB_CUDA(cudaMemcpyAsync(&c, (char *)s->state + SL.ctrl, sizeof(Control), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
	PHB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
	for (int i = 0; i < nsys; ++i) {
		const SysState &x = h[i];
		phb_solve_result &o = out[i];
		o.final_residual = x.crit;
		o.used_iterations = x.usedIt;
		o.converged = x.done == CONVERGED;
		o.finite = std::isfinite(x.crit);
		o.status = x.done;
		o.inner_iterations = 0;
		o.pad = 0;
		if (c.barErr) { // a persistent solve left early at a grid-barrier wait that ran out
			o.converged = 0;
			o.finite = 0;
			o.status = NONFINITE;
			o.final_residual = NAN;
			continue;
		}
		if (s->return_best && (x.done == MAXIT || x.done == RISING) && x.bestIt >= 0 && x.best < x.crit) {
			o.used_iterations = x.bestIt;
			o.final_residual = x.best;
		}
	}
	return PHB_OK;
}

extern "C" int phb_stencil_apply(const phb_domain *dom, const double *A, const double *X, double *Y, int32_t nvec,
		int64_t stride, phb_stream stream) {
	if (!dom || !A || !X || !Y) return setError(PHB_ERR_ARG, "phb_stencil_apply: null argument");
	// the quad loads of a row take 16-byte vector loads at cells that are multiples of four
	if (nvec < 1 || stride < dom->ncells || (stride & 3) != 0)
		return setError(PHB_ERR_ARG, "phb_stencil_apply: nvec < 1, stride < ncells or stride not a multiple of 4");
	if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) & 31)
		return setError(PHB_ERR_ARG, "phb_stencil_apply: A, X and Y must be 32-byte aligned");
	if (dom->dims != 2 && dom->dims != 3) return setError(PHB_ERR_ARG, "phb_stencil_apply: dims");
	if (dom->ntiles == 0) return PHB_OK;
	cudaStream_t s = (cudaStream_t)stream;
	if (dom->dims == 2) kStencilApply<2><<<dom->ntiles, PHB_TILE, 0, s>>>(Dom<double, 2>(*dom), A, X, Y, nvec, stride);
	else kStencilApply<3><<<dom->ntiles, PHB_TILE, 0, s>>>(Dom<double, 3>(*dom), A, X, Y, nvec, stride);
	return checkLaunch("kStencilApply");
}

extern "C" int phb_projection_gram(const double *V, const double *Y, const double *b, int32_t m, int64_t n, int64_t stride,
		double *G, double *c, phb_stream stream) {
	if (!V || !Y || !b || !G || !c) return setError(PHB_ERR_ARG, "phb_projection_gram: null argument");
	if (m < 1 || m > PROJ_MAX) return setError(PHB_ERR_RANGE, "phb_projection_gram: m outside 1..16");
	if (n < 0 || stride < n) return setError(PHB_ERR_ARG, "phb_projection_gram: n < 0 or stride < n");
	cudaStream_t s = (cudaStream_t)stream;
	PHB_CUDA(cudaMemsetAsync(G, 0, sizeof(double) * m * m, s));
	PHB_CUDA(cudaMemsetAsync(c, 0, sizeof(double) * m, s));
	if (n == 0) return PHB_OK;
	int dev = 0, sms = 0;
	PHB_CUDA(cudaGetDevice(&dev));
	PHB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	const int64_t chunks = (n + GRAM_CHUNK - 1) / GRAM_CHUNK;
	const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(chunks, (int64_t)sms * 4));
	kProjectionGram<<<grid, 256, 0, s>>>(V, Y, b, m, n, stride, G, c);
	return checkLaunch("kProjectionGram");
}

extern "C" int phb_projection_solve(const double *G, const double *c, int32_t m, double reg, double *alpha,
		phb_stream stream) {
	if (!G || !c || !alpha) return setError(PHB_ERR_ARG, "phb_projection_solve: null argument");
	if (m < 1 || m > PROJ_MAX) return setError(PHB_ERR_RANGE, "phb_projection_solve: m outside 1..16");
	kProjectionSolve<<<1, 256, 0, (cudaStream_t)stream>>>(G, c, m, reg, alpha);
	return checkLaunch("kProjectionSolve");
}

extern "C" int phb_release_graphs(void) {
	std::lock_guard<std::mutex> lock(gMutex);
	return releaseGraphsLocked();
}

// refinement ------------------------------------------------------------------------------
extern "C" int64_t phb_refine_work_bytes(const phb_domain *dom, int kind, int nrhs) {
	if (!dom) return -1;
	const size_t inner = solveLayout(dom, kind, 4, nrhs).total;
	const size_t v = align256((size_t)dom->ncells * nrhs * 4);
	return (int64_t)(inner + 2 * v + align256((size_t)dom->ntiles * nrhs * 2 * sizeof(double)));
}

template <int D, int K>
static int emitRefine(const phb_domain *dom, const phb_refine *rf, cudaStream_t s, Streams &ss) {
	Dom<double, D> dm(*dom);
	const size_t inner = solveLayout(dom, rf->kind, 4, K).total;
	const size_t vb = align256((size_t)dom->ncells * K * 4);
	char *w = (char *)rf->work;
	float *r32 = (float *)(w + inner);
	float *e32 = (float *)(w + inner + vb);
	double *partial = (double *)(w + inner + 2 * vb);
	dm.vec4 = vec4Ok(dom, {rf->A64, rf->b, rf->x, w});
	const StateLayout SL = stateLayout(dom, K);
	char *sb = (char *)rf->state;
	Control *ctrlO = (Control *)(sb + SL.ctrl2);
	SysState *stO = (SysState *)(sb + SL.st2);
	SysState *stI = (SysState *)(sb + SL.st);
	const int nsys = dom->ninst * K;
	phb_solve in = {};
	in.kind = rf->kind;
	in.vec_dtype = PHB_F32;
	in.mat_dtype = PHB_F32;
	in.nrhs = K;
	in.maxit = rf->inner_maxit;
	in.return_best = 0;
	in.use_graph = 1;
	in.A = rf->A32;
	in.b = r32;
	in.x = e32;
	in.tol = phb_tolerance{}; // unused: the inner tolerance is SysState::innerTol
	in.work = rf->work;
	in.state = rf->state;
	in.amg = rf->amg;
	in.ctas_per_sm = rf->ctas_per_sm;
	// 1: nested graph loops; 2: graph outer loop, persistent inner solves; 3: host outer loop,
	// persistent inner solves (every launch visible to a kernel profiler); 0: host loops
	const bool graph = rf->use_graph == 1 || rf->use_graph == 2;
	in.use_graph = rf->use_graph >= 2 ? 2 : (graph ? 1 : 0);
	if (rf->use_graph == 2 && bicgPrefersGraph(dom, rf->kind)) in.use_graph = 1; // nested graph loop
	in.check_every = 8;
	cudaGraphConditionalHandle outerHandle{};
	if (graph) {
		const int rc0 = createCondition(s, &outerHandle);
		if (rc0) return rc0;
	}
	kInitOuter<<<1, 256, 0, s>>>(stO, nsys, rf->tol, ctrlO, rf->max_outer + 2, LoopCond{outerHandle, graph ? 1 : 0});
	PHB_CUDA(cudaGetLastError());
	auto outer = [&](cudaStream_t os, LoopCond lc) -> int {
		kRefineResidual<D, K><<<dom->ntiles, PHB_TILE, 0, os>>>(dm, rf->A64, rf->b, rf->x, r32, e32, stO, partial, ctrlO,
			rf->inner_rtol, rf->max_outer, rf->tol, stI, lc);
		int rc = checkLaunch("kRefineResidual");
		if (rc) return rc;
		rc = emitSolve<float, D, K>(dom, &in, os, ss, graph ? 2 : 0, true, 1);
		if (rc) return rc;
		kRefineUpdate<K><<<gridFor(dom->ncells * K), 256, 0, os>>>(dom->ncells * K, rf->x, e32);
		return checkLaunch("kRefineUpdate");
	};
	if (graph) return addWhile(s, ss.s[1], outerHandle, outer);
	// host loop: every kernel launched on its own (profilers see each launch)
	int *hflag = nullptr;
	PHB_CUDA(cudaMallocHost(&hflag, sizeof(int)));
	int rc = PHB_OK;
	for (int sweep = 0; sweep < rf->max_outer + 2; ++sweep) {
		rc = outer(s, LoopCond{0, 0});
		if (rc) break;
		cudaMemcpyAsync(hflag, &ctrlO->allDone, sizeof(int), cudaMemcpyDeviceToHost, s);
		cudaStreamSynchronize(s);
		if (*hflag) break;
	}
	cudaFreeHost(hflag);
	return rc;
}

extern "C" int phb_refine_results(const phb_domain *dom, const phb_refine *r, phb_solve_result *out, int *outer_used, phb_stream stream);

extern "C" int phb_refine_run(const phb_domain *dom, const phb_refine *r, phb_solve_result *out, int *outer_used, phb_stream stream) {
	if (!dom || !r || !r->A64 || !r->A32 || !r->b || !r->x || !r->work || !r->state || (r->tol.mode == 2 && !r->tol.values))
		return setError(PHB_ERR_ARG, "phb_refine_run: null argument");
	if (r->amg) {
		if (r->kind != 0 || r->nrhs != 1) return setError(PHB_ERR_ARG, "phb_refine_run: the AMG preconditioner takes CG with one right-hand side");
		const int rc = phbCheckAmg(r->amg);
		if (rc) return rc;
		if (r->amg->levels[0].dom.ncells != dom->ncells || !r->amg->levels[0].x) return setError(PHB_ERR_ARG, "phb_refine_run: hierarchy does not match the domain");
	}
	if (dom->ntiles == 0) return PHB_OK;
	cudaStream_t st = (cudaStream_t)stream;
	std::string key = makeKey("refine", *dom, *r);
	if (r->amg) key.append(reinterpret_cast<const char *>(r->amg), sizeof(phb_amg));
	int rc = PHB_OK;
	const int K = r->nrhs;
	if (r->use_graph == 0 || r->use_graph == 3) {
		Streams *ss;
		rc = getStreams(ss);
		if (rc) return rc;
		if (dom->dims == 2 && K == 1) rc = emitRefine<2, 1>(dom, r, st, *ss);
		else if (dom->dims == 2 && K == 2) rc = emitRefine<2, 2>(dom, r, st, *ss);
		else if (dom->dims == 3 && K == 1) rc = emitRefine<3, 1>(dom, r, st, *ss);
		else if (dom->dims == 3 && K == 3) rc = emitRefine<3, 3>(dom, r, st, *ss);
		else return setError(PHB_ERR_ARG, "phb_refine_run: unsupported dims/nrhs");
		if (rc) return rc;
		if (out) return phb_refine_results(dom, r, out, outer_used, stream);
		return PHB_OK;
	}
	if (dom->dims == 2 && K == 1) rc = runGraph(st, key, [&](cudaStream_t cs, Streams &ss) { return emitRefine<2, 1>(dom, r, cs, ss); });
	else if (dom->dims == 2 && K == 2) rc = runGraph(st, key, [&](cudaStream_t cs, Streams &ss) { return emitRefine<2, 2>(dom, r, cs, ss); });
	else if (dom->dims == 3 && K == 1) rc = runGraph(st, key, [&](cudaStream_t cs, Streams &ss) { return emitRefine<3, 1>(dom, r, cs, ss); });
	else if (dom->dims == 3 && K == 3) rc = runGraph(st, key, [&](cudaStream_t cs, Streams &ss) { return emitRefine<3, 3>(dom, r, cs, ss); });
	else return setError(PHB_ERR_ARG, "phb_refine_run: unsupported dims/nrhs");
	if (rc) return rc;
	if (out) return phb_refine_results(dom, r, out, outer_used, stream);
	return PHB_OK;
}

extern "C" int phb_refine_results(const phb_domain *dom, const phb_refine *r, phb_solve_result *out, int *outer_used, phb_stream stream) {
	if (!dom || !r || !out || !r->state) return setError(PHB_ERR_ARG, "phb_refine_results: null argument");
	const int K = r->nrhs;
	const int nsys = dom->ninst * K;
	std::vector<SysState> h(nsys);
	const StateLayout SL = stateLayout(dom, K);
	cudaStream_t st = (cudaStream_t)stream;
	PHB_CUDA(cudaMemcpyAsync(h.data(), (char *)r->state + SL.st2, nsys * sizeof(SysState), cudaMemcpyDeviceToHost, st));
	PHB_CUDA(cudaStreamSynchronize(st));
	int mo = 0;
	for (int i = 0; i < nsys; ++i) {
		out[i].final_residual = h[i].crit;
		out[i].used_iterations = h[i].it;
		out[i].converged = h[i].done == CONVERGED;
		out[i].finite = std::isfinite(h[i].crit);
		out[i].status = h[i].done;
		out[i].inner_iterations = h[i].innerIts;
		mo = std::max(mo, h[i].it);
	}
	if (outer_used) *outer_used = mo;
	return PHB_OK;
}

// no-allocation CG -------------------------------------------------------------------------
// Some hosts cannot hand this library device memory for solver workspace: a program that
// carves the GPU into fixed per-environment slices at start-up and forbids any later
// allocation, or a plugin host whose device allocator is not reachable through a C ABI.
// For them the CG solve below keeps its workspace (residual, search directions, partial
// sums, per-system state) in this file-scope array instead of the caller-provided `work`
// and `state` buffers of phb_solve_run. Every GPU that loads the library holds the array
// until the process exits.
static __device__ __align__(256) unsigned char gNoAllocScratch[PHB_NOALLOC_SCRATCH_BYTES];

// Device address of the array on each device. In host code `gNoAllocScratch` names a
// host-side stand-in, not device memory, so the address is looked up with the device
// current: by the first call on a device, and again by every call whose stream is not
// capturing (a cheap host call), so that a context that was reset and re-created, which
// reloads the module and may move the array, is followed. A call made while its stream is
// capturing uses the address of the last call that was not, so the first call on a device
// must come before any capture.
static std::mutex gNoAllocMutex;
static void *gNoAllocPtr[64] = {nullptr};

static int noAllocScratch(cudaStream_t s, void **out) {
	int dev;
	PHB_CUDA(cudaGetDevice(&dev));
	if (dev < 0 || dev >= 64) return setError(PHB_ERR_RANGE, "phb_cg_solve_noalloc: device index out of range");
	cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
	PHB_CUDA(cudaStreamIsCapturing(s, &cap));
	std::lock_guard<std::mutex> lock(gNoAllocMutex);
	if (cap == cudaStreamCaptureStatusNone) {
		void *p = nullptr;
		PHB_CUDA(cudaGetSymbolAddress(&p, gNoAllocScratch));
		gNoAllocPtr[dev] = p;
	} else if (!gNoAllocPtr[dev]) {
		return setError(PHB_ERR_ARG, "phb_cg_solve_noalloc: the first call on a device must not be made while its stream is capturing");
	}
	*out = gNoAllocPtr[dev];
	return PHB_OK;
}

template <typename T, int D, int K>
static int runCgNoAlloc(const phb_domain *dom, const phb_solve *sv, phb_solve_result *out, cudaStream_t s) {
	Dom<double, D> dm(*dom);
	const Layout L = solveLayout(dom, 0, sizeof(T), K);
	const StateLayout SL = stateLayout(dom, K);
	char *w = (char *)sv->work;
	char *sb = (char *)sv->state;
	Control *ctrl = (Control *)(sb + SL.ctrl);
	SysState *st = (SysState *)(sb + SL.st);
	double *partial = (double *)(w + L.off[10]);
	const T *A = (const T *)sv->A;
	const T *b = (const T *)sv->b;
	T *x = (T *)sv->x;
	dm.vec4 = vec4Ok(dom, {A, b, x, w});
	T *r = (T *)(w + L.off[0]), *q = (T *)(w + L.off[1]), *p0 = (T *)(w + L.off[2]), *p1 = (T *)(w + L.off[3]);
	T *xbest = sv->return_best ? (T *)(w + L.off[4]) : nullptr;
	const int nsys = dom->ninst * K;
	const int tiles = dom->ntiles;
	const int maxit = std::max(1, sv->maxit);
	const int maxLoops = maxit / 2 + 2;
	// kInit resets the state and the ticket counter the reductions count with, so nothing
	// left in the array by an earlier call is read before it is written
	kInit<<<1, 256, 0, s>>>(st, nsys, sv->tol, 0, maxit, ctrl, maxLoops);
	kResidual<T, D, K, false, false><<<tiles, PHB_TILE, 0, s>>>(dm, A, b, x, r, nullptr, st, partial, ctrl, sv->tol, LoopCond{0, 0});
	PHB_CUDA(cudaGetLastError());
	const int chk = std::max(1, sv->check_every);
	for (int loops = 0; loops < maxLoops; loops += chk) {
		for (int i = 0; i < chk; ++i) {
			for (int half = 0; half < 2; ++half) {
				T *pIn = half == 0 ? p0 : p1, *pOut = half == 0 ? p1 : p0;
				kCgDirection<T, D, K><<<tiles, PHB_TILE, 0, s>>>(dm, A, r, pIn, pOut, q, st, partial, ctrl);
				kCgUpdate<T, D, K><<<tiles, PHB_TILE, 0, s>>>(dm, r, pOut, q, x, xbest, st, partial, ctrl, sv->return_best, LoopCond{0, 0});
			}
		}
		PHB_CUDA(cudaGetLastError());
		int done = 0; // pageable stack copy: synchronous, no staging buffer of ours
		PHB_CUDA(cudaMemcpyAsync(&done, &ctrl->allDone, sizeof(int), cudaMemcpyDeviceToHost, s));
		PHB_CUDA(cudaStreamSynchronize(s));
		if (done) break;
	}
	if (xbest) kRestoreBest<T, K><<<gridFor(dom->ncells * K), 256, 0, s>>>(dom->insts, dom->ninst, dom->ncells, x, xbest, st);
	PHB_CUDA(cudaGetLastError());
	if (out) {
		for (int i = 0; i < nsys; ++i) {
			SysState h;
			PHB_CUDA(cudaMemcpyAsync(&h, st + i, sizeof(SysState), cudaMemcpyDeviceToHost, s));
			PHB_CUDA(cudaStreamSynchronize(s));
			phb_solve_result &o = out[i];
			o.final_residual = h.crit;
			o.used_iterations = h.usedIt;
			o.converged = h.done == CONVERGED;
			o.finite = std::isfinite(h.crit);
			o.status = h.done;
			o.inner_iterations = 0;
			o.pad = 0;
			if (sv->return_best && (h.done == MAXIT || h.done == RISING) && h.bestIt >= 0 && h.best < h.crit) {
				o.used_iterations = h.bestIt;
				o.final_residual = h.best;
			}
		}
	}
	return PHB_OK;
}

extern "C" int64_t phb_cg_noalloc_bytes(const phb_domain *dom, int dtype, int nrhs) {
	if (!dom) return -1;
	const int vb = dtype == PHB_F64 ? 8 : 4;
	return (int64_t)(solveLayout(dom, 0, vb, nrhs).total + stateLayout(dom, nrhs).total);
}

extern "C" int phb_cg_solve_noalloc(const phb_domain *dom, int dtype, int nrhs, const void *A, const void *b, void *x,
		const phb_tolerance *tol, int maxit, int return_best, phb_solve_result *out, phb_stream stream) {
	if (!dom || !A || !b || !x || !tol || (tol->mode == 2 && !tol->values))
		return setError(PHB_ERR_ARG, "phb_cg_solve_noalloc: null argument");
	if (dtype != PHB_F32 && dtype != PHB_F64) return setError(PHB_ERR_ARG, "phb_cg_solve_noalloc: dtype");
	const int64_t need = phb_cg_noalloc_bytes(dom, dtype, nrhs);
	if (need > (int64_t)PHB_NOALLOC_SCRATCH_BYTES) {
		char msg[256];
		snprintf(msg, sizeof(msg), "phb_cg_solve_noalloc: the solve needs %lld bytes of scratch, more than the %lld of the "
			"static array (PHB_NOALLOC_SCRATCH_BYTES)", (long long)need, (long long)PHB_NOALLOC_SCRATCH_BYTES);
		return setError(PHB_ERR_RANGE, msg);
	}
	if (dom->ntiles == 0) { // nothing to solve: every system reports a converged empty solve
		if (out) {
			for (int i = 0; i < dom->ninst * nrhs; ++i) {
				phb_solve_result &o = out[i];
				o.final_residual = 0.0;
				o.used_iterations = 0;
				o.converged = 1;
				o.finite = 1;
				o.status = CONVERGED;
				o.inner_iterations = 0;
				o.pad = 0;
			}
		}
		return PHB_OK;
	}
	void *scratch = nullptr;
	int rc = noAllocScratch((cudaStream_t)stream, &scratch);
	if (rc) return rc;
	phb_solve sv = {};
	sv.kind = 0;
	sv.vec_dtype = sv.mat_dtype = dtype;
	sv.nrhs = nrhs;
	sv.maxit = maxit;
	sv.return_best = return_best ? 1 : 0;
	sv.use_graph = 0;
	sv.check_every = 16;
	sv.tol = *tol;
	sv.A = A;
	sv.b = b;
	sv.x = x;
	sv.work = scratch;
	sv.state = (char *)scratch + solveLayout(dom, 0, dtype == PHB_F64 ? 8 : 4, nrhs).total;
	cudaStream_t st = (cudaStream_t)stream;
	PHB_SOLVE_DISPATCH(dom->dims, dtype, nrhs, return runCgNoAlloc<T, D, KK>(dom, &sv, out, st));
	return PHB_OK;
}

extern "C" int phb_barrier_selftest(int ctas, int rounds, int absent_cta, unsigned int spin_limit, void *scratch, int *bar_err,
		int *rounds_done, phb_stream stream) {
	if (ctas < 1 || rounds < 0 || !scratch || !bar_err || !rounds_done || spin_limit < 1024)
		return setError(PHB_ERR_ARG, "phb_barrier_selftest: bad argument");
	if (((uintptr_t)scratch & 15) != 0) return setError(PHB_ERR_ARG, "phb_barrier_selftest: scratch must be 16-byte aligned");
	int perSM = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kBarrierProbe, PHB_TILE, 0) != cudaSuccess || perSM < 1) perSM = 1;
	if (ctas > perSM * numSMs()) return setError(PHB_ERR_RANGE, "phb_barrier_selftest: more CTAs than can be co-resident");
	cudaStream_t s = (cudaStream_t)stream;
	Control *ctrl = (Control *)scratch;
	int *done = (int *)((char *)scratch + 256);
	PHB_CUDA(cudaMemsetAsync(scratch, 0, 256 + sizeof(int), s));
	cudaLaunchConfig_t cfg = {};
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cfg.gridDim = dim3(ctas);
	cfg.blockDim = dim3(PHB_TILE);
	cfg.stream = s;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	PHB_CUDA(cudaLaunchKernelEx(&cfg, kBarrierProbe, ctrl, rounds, absent_cta, spin_limit, done));
	PHB_CUDA(cudaMemcpyAsync(bar_err, &ctrl->barErr, sizeof(int), cudaMemcpyDeviceToHost, s));
	PHB_CUDA(cudaMemcpyAsync(rounds_done, done, sizeof(int), cudaMemcpyDeviceToHost, s));
	PHB_CUDA(cudaStreamSynchronize(s));
	return PHB_OK;
}
