// Setup of the aggregation multigrid hierarchy on the device (the numeric part of phiPICT's
// hierarchy_for / galerkin_refresh, solvers/amg.py:450-712): Galerkin products level by
// level, the dense coarsest operator of every instance and its (generalised) inverse. The
// cycle itself is in phb_amg.cuh.
#include <algorithm>
#include <cmath>
#include "phb_amg.cuh"
#include "phb_launch.cuh"

namespace phb {

// omega / diagonal of a level; a zero row (an aggregate that is a whole closed instance, the
// null space) is not smoothed: wd = 0
__global__ void kWdinv(int64_t n, const float *__restrict__ A, float *__restrict__ wd, float omega) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const float d = A[i];
		wd[i] = d != 0.f ? omega / d : 0.f;
	}
}

// Ac = scale * P^T Af P for coarse tile `blockIdx.x`: each coarse stencil entry sums the
// fine entries of the aggregate's cells; couplings between two cells of one aggregate fold
// into the diagonal. scale applies on coarsened blocks only.
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kGalerkin(Dom<float, D> fd, Dom<float, D> cd, const float *__restrict__ Af,
		float *__restrict__ Ac, float scale) {
	__shared__ int32_t sB[PHB_BREC];
	const int tile = blockIdx.x;
	const int bi = __ldg(cd.tiles + 2 * tile);
	const int l0 = __ldg(cd.tiles + 2 * tile + 1);
	const int nc = stageBlock<D>(cd, bi, sB);
	const int32_t *FB = fd.blk(bi);
	const int64_t N = fd.ncells, NC = cd.ncells;
	bool coarsened = false;
#pragma unroll
	for (int a = 0; a < D; ++a) coarsened |= sB[B_NX + a] < FB[B_NX + a];
	const double sc = coarsened ? double(scale) : 1.0;
	for (int j = 0; j < CPT; ++j) {
		Cell cc;
		if (!cellAt<D>(sB, l0, nc, j, cc)) break;
		int base[3], cnt[3];
#pragma unroll
		for (int a = 0; a < 3; ++a) {
			const bool co = a < D && sB[B_NX + a] < FB[B_NX + a];
			base[a] = co ? 2 * cc.p[a] : cc.p[a];
			cnt[a] = (co && base[a] + 1 < FB[B_NX + a]) ? 2 : 1;
		}
		double acc[2 * D + 1];
		double mag = 0; // size of the diagonal's contributions: a sum that cancels to roundoff is zero
#pragma unroll
		for (int s = 0; s < 2 * D + 1; ++s) acc[s] = 0;
		for (int oz = 0; oz < cnt[2]; ++oz)
			for (int oy = 0; oy < cnt[1]; ++oy)
				for (int ox = 0; ox < cnt[0]; ++ox) {
					const int o[3] = {ox, oy, oz};
					const int p[3] = {base[0] + ox, base[1] + oy, base[2] + oz};
					const int64_t g = FB[B_CELLOFF] + flat(FB, p);
					acc[0] += Af[g];
					mag += fabs(double(Af[g]));
#pragma unroll
					for (int f = 0; f < 2 * D; ++f) {
						const int a = f >> 1;
						// the neighbour across f is the other cell of the aggregate
						const bool inside = cnt[a] == 2 && ((f & 1) ? o[a] == 0 : o[a] == 1);
						const double v = Af[(f + 1) * N + g];
						if (inside) {
							acc[0] += v;
							mag += fabs(v);
						} else acc[f + 1] += v;
					}
				}
		// across a periodic face of a block one cell wide along that axis the neighbour is the
		// cell itself: that coupling belongs to the diagonal (the stencil applies the same
		// operator either way, but the smoother and the test below need the true diagonal)
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			if (sB[B_NX + (f >> 1)] == 1 && fType(sB, f) == FT_PERIODIC) {
				acc[0] += acc[f + 1];
				mag += fabs(acc[f + 1]);
				acc[f + 1] = 0.0;
			}
		}
		// the fine values are float32: a diagonal below 1e-5 of its contributions is a
		// cancellation (an aggregate with no coupling left outside it) and exactly zero
		if (fabs(acc[0]) <= 1e-5 * mag) acc[0] = 0.0;
#pragma unroll
		for (int s = 0; s < 2 * D + 1; ++s) Ac[s * NC + cc.g] = float(sc * acc[s]);
	}
}

// Dense operator of the coarsest level per instance: dense[inst][row][col] (local cells).
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kDense(Dom<float, D> cd, const float *__restrict__ Ac, int cn, double *__restrict__ dense) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<float, D>(cd, sB, l0, nc);
	const int64_t N = cd.ncells;
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const int inst = c.B[B_INST];
		const int off = c.B[B_INSTOFF];
		if (c.g - off >= cn) continue; // an instance larger than the stride: rejected by the host
		double *row = dense + ((size_t)inst * cn + (c.g - off)) * cn;
		atomicAdd(row + (c.g - off), double(Ac[c.g]));
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			const int64_t nb = neighborIndex<float, D>(cd, c, f);
			if (nb >= 0 && nb - off < cn) atomicAdd(row + (nb - off), double(Ac[(f + 1) * N + c.g]));
		}
	}
}

// In-place Gauss-Jordan inversion of each instance's coarsest operator (one CTA per
// instance). The operators are symmetric and (semi)definite, so no pivoting is needed.
// A pure-Neumann pressure or potential system is singular with the constant as null space
// (phiPICT's rank-deficient systems, whose V-cycle projects the constant out,
// solvers/amg.py hierarchy_for(project_constant=...)). Its coarse operator is built from
// float32 stencils, so its row sums are roundoff rather than zero and the null pivot would
// be inverted into a huge eigenvalue of either sign. Such an operator (every row sum below
// ZERO_ROWSUM of the largest diagonal) is inverted as A + c 1 1^T with c n = sign(diag) *
// max|diag|: the constant then has an eigenvalue of the operator's own sign and size, and the
// inverse is a definite operator that solves every consistent coarse system. A pivot that
// still falls to roundoff (a second null direction, e.g. two unconnected blocks) is left out:
// that row and column of the inverse are zero.
constexpr int INV_THREADS = 512;
constexpr int INV_MAX = 1024;
constexpr double ZERO_ROWSUM = 1e-4;
// instances whose n x n operator fits are inverted in shared memory
constexpr size_t INV_SMEM_MAX = 200 * 1024;

// M: the n x n operator with row stride ld (shared or global memory), inverted in place
__device__ void invertDense(double *M, int n, int ld) {
	__shared__ double rowk[INV_MAX], colk[INV_MAX];
	__shared__ unsigned char skip[INV_MAX];
	__shared__ double red[3][INV_THREADS / 32];
	__shared__ double sThr, sShift;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	// largest |diagonal|, largest |row sum| and the sum of the diagonal (its sign), one warp per row
	double m = 0, rs = 0, ds = 0;
	for (int i = warp; i < n; i += INV_THREADS / 32) {
		double s = 0;
		for (int j = lane; j < n; j += 32) s += M[(size_t)i * ld + j];
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		const double dg = M[(size_t)i * ld + i];
		m = fmax(m, fabs(dg));
		rs = fmax(rs, fabs(s));
		ds += dg;
	}
	if (lane == 0) { red[0][warp] = m; red[1][warp] = rs; red[2][warp] = ds; }
	for (int i = threadIdx.x; i < n; i += blockDim.x) skip[i] = 0;
	__syncthreads();
	if (threadIdx.x == 0) {
		double v = 0, r = 0, d = 0;
		for (int w = 0; w < INV_THREADS / 32; ++w) { v = fmax(v, red[0][w]); r = fmax(r, red[1][w]); d += red[2][w]; }
		sThr = 1e-10 * v;
		sShift = (n > 1 && v > 0 && r <= ZERO_ROWSUM * v) ? (d < 0 ? -v : v) / n : 0.0;
	}
	__syncthreads();
	const double thr = sThr;
	const double shift = sShift;
	// element loops: warp w takes rows w, w + NW, ..., lane c columns c, c + 32, ... (no
	// integer division in the hot loop)
	constexpr int NW = INV_THREADS / 32;
	if (shift != 0.0) {
		for (int i = warp; i < n; i += NW)
			for (int j = lane; j < n; j += 32) M[(size_t)i * ld + j] += shift;
		__syncthreads();
	}
	for (int k = 0; k < n; ++k) {
		const double p = M[(size_t)k * ld + k];
		if (!(fabs(p) > thr)) {
			if (threadIdx.x == 0) skip[k] = 1;
			__syncthreads();
			continue;
		}
		for (int j = threadIdx.x; j < n; j += blockDim.x) {
			rowk[j] = M[(size_t)k * ld + j] / p;
			colk[j] = M[(size_t)j * ld + k];
		}
		__syncthreads();
		const double rp = 1.0 / p;
		for (int i = warp; i < n; i += NW) {
			double *Mi = M + (size_t)i * ld;
			const double ci = colk[i];
			if (i == k) {
				for (int j = lane; j < n; j += 32) Mi[j] = j == k ? rp : rowk[j];
			} else {
				for (int j = lane; j < n; j += 32) Mi[j] = j == k ? -ci * rp : Mi[j] - ci * rowk[j];
			}
		}
		__syncthreads();
	}
	for (int i = warp; i < n; i += NW)
		for (int j = lane; j < n; j += 32)
			if (skip[i] || skip[j]) M[(size_t)i * ld + j] = 0.0;
	__syncthreads();
}

// One CTA per instance: dense[inst] is cn x cn, of which the instance's n x n block is used.
// SHARED: the block is staged through dynamic shared memory.
template <bool SHARED>
__global__ void __launch_bounds__(INV_THREADS) kInvert(double *dense, int cn, const int32_t *insts) {
	extern __shared__ double sm[];
	double *G = dense + (size_t)blockIdx.x * cn * cn;
	const int n = min(cn, insts[blockIdx.x * PHB_IREC + I_NCELLS]);
	if (SHARED) {
		const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
		for (int i = warp; i < n; i += INV_THREADS / 32)
			for (int j = lane; j < n; j += 32) sm[i * n + j] = G[(size_t)i * cn + j];
		__syncthreads();
		invertDense(sm, n, n);
		for (int i = warp; i < n; i += INV_THREADS / 32)
			for (int j = lane; j < n; j += 32) G[(size_t)i * cn + j] = sm[i * n + j];
	} else {
		invertDense(G, n, cn);
	}
}

// --- the cycle below a small level as one dense operator --------------------------------
// One cycle at level l (x0 = S b, restriction, the coarse correction C_{l+1}, prolongation,
// a second sweep) is the linear map
//   C_l = S~ + W C_{l+1} W^T,   S = omega D^-1,  S~ = 2S - S A S,  W = (I - S A) P,
// so the levels below a small level T fold, from the coarsest inverse up, into one dense
// matrix per instance (FP64, rows and columns indexed by the instance's local cells).

// W [inst][n][nc] = (I - S A) P of level l (zeroed by the caller): the row of cell i holds
// 1 - wd_i A_ii at its own aggregate and -wd_i A_ij at the aggregate of each neighbour j
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kTailW(Dom<float, D> fd, Dom<float, D> cd, const float *__restrict__ A,
		const float *__restrict__ wd, double *__restrict__ W, int n, int nc) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, ncb;
	loadTile<float, D>(fd, sB, l0, ncb);
	const int bi = __ldg(fd.tiles + 2 * blockIdx.x);
	const int32_t *CB = cd.blk(bi);
	const int64_t N = fd.ncells;
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, ncb, j, c)) break;
		const int inst = sB[B_INST];
		const int64_t i = c.g - sB[B_INSTOFF];
		if (i >= n) continue;
		const int coff = CB[B_INSTOFF];
		double *row = W + ((size_t)inst * n + i) * nc;
		const double wi = wd[c.g];
		const int64_t ai = coarseCell<D>(CB, sB, c.p) - coff;
		if (ai < nc) row[ai] += 1.0 - wi * A[c.g];
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			if (atBound(sB, f, c.p) && fType(sB, f) == FT_FIXED) continue;
			const Nbr nb = neighbor<float, D>(fd, c, f);
			const int32_t *nCB = nb.B == sB ? CB : cd.blk(int((nb.B - fd.blocks) / PHB_BREC));
			const int64_t aj = coarseCell<D>(nCB, nb.B, nb.p) - coff;
			if (aj < nc) row[aj] -= wi * A[(f + 1) * N + c.g];
		}
	}
}

// C [inst][n][n] += S~ of level l: 2 wd_i - wd_i A_ii wd_i on the diagonal, -wd_i A_ij wd_j
// at each neighbour j
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kTailSbar(Dom<float, D> fd, const float *__restrict__ A, const float *__restrict__ wd,
		double *__restrict__ C, int n) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, ncb;
	loadTile<float, D>(fd, sB, l0, ncb);
	const int64_t N = fd.ncells;
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, ncb, j, c)) break;
		const int inst = sB[B_INST];
		const int off = sB[B_INSTOFF];
		const int64_t i = c.g - off;
		if (i >= n) continue;
		double *row = C + ((size_t)inst * n + i) * n;
		const double wi = wd[c.g];
		row[i] += 2.0 * wi - wi * A[c.g] * wi;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			const int64_t nb = neighborIndex<float, D>(fd, c, f);
			if (nb >= 0 && nb - off < n) row[nb - off] -= wi * A[(f + 1) * N + c.g] * double(wd[nb]);
		}
	}
}

// Batched C = A op(B) over instances (blockIdx.z): A [m][k], op(B) [k][n] (TB: B stored
// [n][k]), C [m][n], each instance's matrices `stride*` apart. Setup only, FP64.
constexpr int GT = 16;
template <bool TB>
__global__ void __launch_bounds__(GT * GT) kGemm(int m, int n, int k, const double *__restrict__ A, size_t sA,
		const double *__restrict__ B, size_t sB, double *__restrict__ C, size_t sC) {
	__shared__ double As[GT][GT + 1], Bs[GT][GT + 1];
	const int tx = threadIdx.x % GT, ty = threadIdx.x / GT;
	const int row = blockIdx.y * GT + ty, col = blockIdx.x * GT + tx;
	const double *Ai = A + blockIdx.z * sA;
	const double *Bi = B + blockIdx.z * sB;
	double acc = 0;
	for (int kk = 0; kk < k; kk += GT) {
		As[ty][tx] = (row < m && kk + tx < k) ? Ai[(size_t)row * k + kk + tx] : 0.0;
		const int bk = kk + ty;
		if (TB) Bs[ty][tx] = (bk < k && col < n) ? Bi[(size_t)col * k + bk] : 0.0;
		else Bs[ty][tx] = (bk < k && col < n) ? Bi[(size_t)bk * n + col] : 0.0;
		__syncthreads();
#pragma unroll
		for (int t = 0; t < GT; ++t) acc += As[ty][t] * Bs[t][tx];
		__syncthreads();
	}
	if (row < m && col < n) C[blockIdx.z * sC + (size_t)row * n + col] = acc;
}

static int gemm(bool tb, int ninst, int m, int n, int k, const double *A, const double *B, double *C, cudaStream_t s) {
	dim3 grid((n + GT - 1) / GT, (m + GT - 1) / GT, ninst);
	if (tb) kGemm<true><<<grid, GT * GT, 0, s>>>(m, n, k, A, (size_t)m * k, B, (size_t)n * k, C, (size_t)m * n);
	else kGemm<false><<<grid, GT * GT, 0, s>>>(m, n, k, A, (size_t)m * k, B, (size_t)k * n, C, (size_t)m * n);
	return checkLaunch("kGemm");
}

static int tailLevel(const phb_amg *amg) {
	return (amg->tail_level >= 1 && amg->tail_level < amg->nlevels) ? amg->tail_level : amg->nlevels - 1;
}

// rows of the dense operator of level l >= T per instance (level T: the coarse_n stride)
static int denseN(const phb_amg *amg, int l) { return l == tailLevel(amg) ? amg->coarse_n : amg->levels[l].inst_cells; }

// dense operator buffers: the coarsest inverse and the folded levels above it are built in
// `work` ([C_a | C_b | W | Tmp], each sized for the largest level) and the last one, C_T,
// in coarse_inv
static void tailSizes(const phb_amg *amg, int64_t &cmax, int64_t &wmax) {
	const int T = tailLevel(amg), L = amg->nlevels;
	cmax = 0;
	wmax = 0;
	for (int l = T; l < L; ++l) {
		const int64_t n = denseN(amg, l);
		cmax = std::max(cmax, n * n);
		if (l + 1 < L) wmax = std::max(wmax, n * (int64_t)denseN(amg, l + 1));
	}
}
static int64_t tailWorkDoubles(const phb_amg *amg) {
	int64_t c, w;
	tailSizes(amg, c, w);
	return (int64_t)amg->levels[0].dom.ninst * (2 * c + 2 * w);
}

template <int D>
static int setup(const phb_amg *amg, cudaStream_t s) {
	const int L = amg->nlevels;
	for (int l = 0; l + 1 < L; ++l) {
		const phb_amg_level &F = amg->levels[l], &C = amg->levels[l + 1];
		if (C.dom.ntiles == 0) continue;
		kGalerkin<D><<<C.dom.ntiles, PHB_TILE, 0, s>>>(Dom<float, D>(F.dom), Dom<float, D>(C.dom), F.A, C.A, amg->coarse_scale);
		const int rc = checkLaunch("kGalerkin");
		if (rc) return rc;
	}
	for (int l = 0; l < L; ++l) {
		const phb_amg_level &v = amg->levels[l];
		const int64_t n = v.dom.ncells;
		kWdinv<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 8), 256, 0, s>>>(n, v.A, v.wdinv, amg->omega);
	}
	int rc = checkLaunch("kWdinv");
	if (rc) return rc;
	// the coarsest inverse (into coarse_inv when it is the last level of the cycle)
	const int T = tailLevel(amg);
	const int ninst = amg->levels[0].dom.ninst;
	const phb_amg_level &C = amg->levels[L - 1];
	const int nL = denseN(amg, L - 1);
	double *cur = T == L - 1 ? amg->coarse_inv : amg->work;
	PHB_CUDA(cudaMemsetAsync(cur, 0, sizeof(double) * (size_t)ninst * nL * nL, s));
	if (C.dom.ntiles) kDense<D><<<C.dom.ntiles, PHB_TILE, 0, s>>>(Dom<float, D>(C.dom), C.A, nL, cur);
	rc = checkLaunch("kDense");
	if (rc) return rc;
	const size_t smem = (size_t)nL * nL * sizeof(double);
	if (smem <= INV_SMEM_MAX) {
		static int configured[64] = {0};
		int dev = 0;
		PHB_CUDA(cudaGetDevice(&dev));
		if (dev >= 0 && dev < 64 && !configured[dev]) {
			PHB_CUDA(cudaFuncSetAttribute(kInvert<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INV_SMEM_MAX));
			configured[dev] = 1;
		}
		kInvert<true><<<ninst, INV_THREADS, smem, s>>>(cur, nL, C.dom.insts);
	} else {
		kInvert<false><<<ninst, INV_THREADS, 0, s>>>(cur, nL, C.dom.insts);
	}
	rc = checkLaunch("kInvert");
	if (rc) return rc;
	// fold the levels above it: C_l = S~_l + W_l C_{l+1} W_l^T, down to level T
	int64_t cmax, wmax;
	tailSizes(amg, cmax, wmax);
	double *bufA = amg->work, *bufB = amg->work + ninst * cmax;
	double *W = amg->work + 2 * ninst * cmax, *Tm = W + ninst * wmax;
	int ncur = nL;
	for (int l = L - 2; l >= T; --l) {
		const phb_amg_level &F = amg->levels[l], &G = amg->levels[l + 1];
		const int n = denseN(amg, l);
		double *next = l == T ? amg->coarse_inv : (cur == bufA ? bufB : bufA);
		PHB_CUDA(cudaMemsetAsync(W, 0, sizeof(double) * (size_t)ninst * n * ncur, s));
		kTailW<D><<<F.dom.ntiles, PHB_TILE, 0, s>>>(Dom<float, D>(F.dom), Dom<float, D>(G.dom), F.A, F.wdinv, W, n, ncur);
		rc = checkLaunch("kTailW");
		if (rc) return rc;
		rc = gemm(false, ninst, n, ncur, ncur, W, cur, Tm, s); // Tm = W C_{l+1}
		if (rc) return rc;
		rc = gemm(true, ninst, n, n, ncur, Tm, W, next, s);    // C_l = Tm W^T
		if (rc) return rc;
		kTailSbar<D><<<F.dom.ntiles, PHB_TILE, 0, s>>>(Dom<float, D>(F.dom), F.A, F.wdinv, next, n);
		rc = checkLaunch("kTailSbar");
		if (rc) return rc;
		cur = next;
		ncur = n;
	}
	return PHB_OK;
}

} // namespace phb

using namespace phb;

// Shared with the Krylov solvers: validates a hierarchy before any launch.
int phbCheckAmg(const phb_amg *amg) {
	if (!amg) return setError(PHB_ERR_ARG, "AMG: null hierarchy");
	if (amg->nlevels < 2 || amg->nlevels > PHB_AMG_MAX_LEVELS) return setError(PHB_ERR_RANGE, "AMG: nlevels must be 2..PHB_AMG_MAX_LEVELS");
	if (amg->coarse_n < 1 || amg->coarse_n > INV_MAX) return setError(PHB_ERR_RANGE, "AMG: coarse_n must be 1..1024");
	if (!amg->coarse_inv) return setError(PHB_ERR_ARG, "AMG: coarse_inv missing");
	const int d = amg->levels[0].dom.dims;
	if (d != 2 && d != 3) return setError(PHB_ERR_ARG, "AMG: dims must be 2 or 3");
	for (int l = 0; l < amg->nlevels; ++l) {
		const phb_amg_level &v = amg->levels[l];
		if (v.dom.dims != d || !v.dom.blocks || !v.dom.tiles || !v.dom.insts || !v.A || !v.wdinv) return setError(PHB_ERR_ARG, "AMG: incomplete level");
		if (l > 0 && (!v.b || !v.x)) return setError(PHB_ERR_ARG, "AMG: level vectors missing");
		if (v.dom.ninst != amg->levels[0].dom.ninst) return setError(PHB_ERR_ARG, "AMG: levels disagree on the instance count");
	}
	const int T = tailLevel(amg);
	for (int l = T; l < amg->nlevels; ++l) {
		const phb_amg_level &v = amg->levels[l];
		if (v.inst_cells < 1 || v.inst_cells > INV_MAX || v.dom.ncells > (int64_t)v.dom.ninst * v.inst_cells)
			return setError(PHB_ERR_RANGE, "AMG: inst_cells of a dense level missing, too small, or above 1024");
	}
	if (amg->coarse_n < amg->levels[T].inst_cells) return setError(PHB_ERR_RANGE, "AMG: coarse_n below the cells of an instance on the dense level");
	if (T < amg->nlevels - 1 && (!amg->work || amg->work_doubles < tailWorkDoubles(amg)))
		return setError(PHB_ERR_ARG, "AMG: setup work buffer missing or smaller than phb_amg_work_doubles()");
	return PHB_OK;
}

extern "C" int64_t phb_amg_work_doubles(const phb_amg *amg) {
	if (!amg || amg->nlevels < 2 || amg->nlevels > PHB_AMG_MAX_LEVELS) return -1;
	return tailWorkDoubles(amg);
}

extern "C" int phb_amg_setup(const phb_amg *amg, phb_stream stream) {
	const int rc = phbCheckAmg(amg);
	if (rc) return rc;
	cudaStream_t s = (cudaStream_t)stream;
	return amg->levels[0].dom.dims == 2 ? setup<2>(amg, s) : setup<3>(amg, s);
}

extern "C" int phb_amg_refresh_fine(const phb_amg *amg, phb_stream stream) {
	const int rc = phbCheckAmg(amg);
	if (rc) return rc;
	const phb_amg_level &v = amg->levels[0];
	const int64_t n = v.dom.ncells;
	if (n == 0) return PHB_OK;
	kWdinv<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 8), 256, 0, (cudaStream_t)stream>>>(n, v.A, v.wdinv, amg->omega);
	return checkLaunch("kWdinv");
}

extern "C" int phb_amg_vcycle(const phb_amg *amg, const float *r, float *z, phb_stream stream) {
	const int rc = phbCheckAmg(amg);
	if (rc) return rc;
	if (!r || !z) return setError(PHB_ERR_ARG, "phb_amg_vcycle: null vector");
	cudaStream_t s = (cudaStream_t)stream;
	if (amg->levels[0].dom.dims == 2) PHB_CUDA(launchAmgCycle<2>(makeAmgView<2>(*amg, r, z), s, 0));
	else PHB_CUDA(launchAmgCycle<3>(makeAmgView<3>(*amg, r, z), s, 0));
	return PHB_OK;
}
