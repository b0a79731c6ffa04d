// Aggregation multigrid on the block structure: the V-cycle that preconditions the CG of
// the pressure and potential solves (phiPICT solvers/amg.py, run on the device by
// solvers/krylov/krylov.cu:1248-1546).
//
// phiPICT builds a Ruge-Stueben hierarchy with pyamg on the host and applies it to CSR
// levels. Here every level stays a structured multi-block stencil: a coarse cell
// aggregates up to 2^d cells of one block (2 per axis, 1 at an odd end), the coarse blocks
// keep the topology of the fine ones (periodic and connected faces), and the coarse operator
// is the Galerkin product P^T A P with piecewise-constant P (optionally scaled per coarsening;
// 0.5 would give the rediscretised operator). Neighbours come from the same index
// arithmetic on every level; there are no column indices. The coarsest level is solved with
// a dense inverse per instance, as phiPICT's coarse pseudo-inverse (solvers/amg.py:579-585).
//
// One cycle, for the right-hand side b_l of level l:
//   x0 = omega D^-1 b_l                       (pre-smoothing Jacobi sweep from zero)
//   b_{l+1} = P^T (b_l - A_l x0)              (restriction of the residual)
//   e = cycle(b_{l+1})                        (coarsest level: e = inverse * b)
//   x1 = x0 + P e;  z_l = x1 + omega D^-1 (b_l - A_l x1)   (post-smoothing sweep)
// x0 is never stored: the restriction and the prolongation re-evaluate it at the stencil
// points, so a cycle costs one pass per level down and one per level up. With a symmetric
// smoother on both sides and R = P^T the cycle is a symmetric operator, as CG requires.
#pragma once

#include "phb_device.cuh"

namespace phb {

constexpr int AMG_MAX_LEVELS = PHB_AMG_MAX_LEVELS;

// Device view of a hierarchy. Level 0's b is the residual being preconditioned and its x the
// result z; both are set per solve.
template <int D>
struct AmgView {
	Dom<float, D> lv[AMG_MAX_LEVELS];
	const float *A[AMG_MAX_LEVELS];
	const float *wd[AMG_MAX_LEVELS]; // omega / diagonal
	float *b[AMG_MAX_LEVELS];
	float *x[AMG_MAX_LEVELS];
	const double *inv; // dense operator of the last level of the cycle, per instance
	int cn, nlevels;   // its row stride; levels of the cycle (the last one dense)
	float omega;
};

template <int D>
__host__ inline AmgView<D> makeAmgView(const phb_amg &a, const float *r, float *z) {
	AmgView<D> v = {};
	for (int l = 0; l < a.nlevels && l < AMG_MAX_LEVELS; ++l) {
		v.lv[l] = Dom<float, D>(a.levels[l].dom);
		v.A[l] = a.levels[l].A;
		v.wd[l] = a.levels[l].wdinv;
		v.b[l] = a.levels[l].b;
		v.x[l] = a.levels[l].x;
	}
	v.b[0] = const_cast<float *>(r);
	v.x[0] = z;
	v.inv = a.coarse_inv;
	v.cn = a.coarse_n;
	// the cycle ends at level T, whose dense operator stands for everything below it
	v.nlevels = ((a.tail_level >= 1 && a.tail_level < a.nlevels) ? a.tail_level : a.nlevels - 1) + 1;
	v.omega = a.omega;
	return v;
}

__device__ __forceinline__ double amgWarpSum(double v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

__device__ __forceinline__ float amgDiag(const float *A, int64_t g) {
	const float d = __ldg(A + g);
	return d != 0.f ? d : 1.f;
}

// Coarse cell of fine position p in fine block FB; CB is the same block on the coarse level
// (an axis is coarsened when the coarse block is shorter along it).
template <int D>
__device__ __forceinline__ int64_t coarseCell(const int32_t *CB, const int32_t *FB, const int *p) {
	int q[3];
#pragma unroll
	for (int a = 0; a < 3; ++a) q[a] = (a < D && CB[B_NX + a] < FB[B_NX + a]) ? p[a] >> 1 : p[a];
	if (D < 3) q[2] = 0;
	return CB[B_CELLOFF] + flat(CB, q);
}

// Stage the record of `blk` of level `d` into shared memory (all threads take part).
template <int D>
__device__ __forceinline__ int stageBlock(const Dom<float, D> &d, int blk, int32_t *sB) {
	__syncthreads();
	if (threadIdx.x < PHB_BREC) sB[threadIdx.x] = __ldg(d.blocks + blk * PHB_BREC + threadIdx.x);
	__syncthreads();
	return sB[B_NX] * sB[B_NY] * (D > 2 ? sB[B_NZ] : 1);
}

// The restriction gives each coarse cell a group of 2^d lanes, one fine cell of its aggregate
// per lane, and sums the group with a fixed shuffle tree (deterministic): short dependency
// chains per thread and all fine cells in flight at once. A CTA covers RSUB coarse cells, a
// coarse tile RSUB_PER_TILE such sub-tiles.
template <int D> struct Restrict {
	static constexpr int G = 1 << D;                       // lanes per coarse cell
	static constexpr int CELLS = PHB_TILE / G;             // coarse cells per CTA
	static constexpr int PER_TILE = PHB_TILE_CELLS / CELLS; // CTAs per coarse tile
};

// One part (Restrict::CELLS coarse cells) of a coarse tile whose block `bi` (nc cells, tile
// starting at l0) is staged in sB.
template <int D>
__device__ __forceinline__ void amgRestrictPart(const AmgView<D> &mg, int l, int bi, int l0, int nc, int part, const int32_t *sB) {
	using R = Restrict<D>;
	const Dom<float, D> &fd = mg.lv[l];
	const float *A = mg.A[l];
	const float *wd = mg.wd[l];
	const float *b = mg.b[l];
	float *bc = mg.b[l + 1];
	const int32_t *FB = fd.blk(bi);
	const int64_t N = fd.ncells;
	const int lc = l0 + part * R::CELLS + int(threadIdx.x) / R::G; // coarse cell of the block
	const int o = int(threadIdx.x) % R::G;                        // fine cell of its aggregate
	const bool cvalid = lc < nc && lc < l0 + PHB_TILE_CELLS;
	float v = 0.f;
	if (cvalid) {
		const int nx = sB[B_NX], ny = sB[B_NY];
		const int cp[3] = {lc % nx, (lc / nx) % ny, D > 2 ? lc / (nx * ny) : 0};
		Cell c;
		bool fvalid = true;
#pragma unroll
		for (int a = 0; a < 3; ++a) {
			const int fs = __ldg(FB + B_NX + a);
			const int oa = (o >> a) & 1;
			const bool co = a < D && sB[B_NX + a] < fs;
			c.p[a] = co ? 2 * cp[a] + oa : cp[a];
			fvalid &= co ? c.p[a] < fs : oa == 0;
		}
		if (fvalid) {
			c.B = FB;
			c.b = bi;
			c.g = __ldg(FB + B_CELLOFF) + flat(FB, c.p);
			c.mi = c.g;
			const float bi_ = b[c.g];
			float y = __ldg(A + c.g) * (bi_ * __ldg(wd + c.g)); // A_ii x0_i
#pragma unroll
			for (int f = 0; f < 2 * D; ++f) {
				const int64_t nb = neighborIndex<float, D>(fd, c, f);
				if (nb >= 0) y += __ldg(A + (f + 1) * N + c.g) * (b[nb] * __ldg(wd + nb));
			}
			v = bi_ - y;
		}
	}
#pragma unroll
	for (int m = 1; m < R::G; m <<= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
	if (cvalid && o == 0) bc[sB[B_CELLOFF] + lc] = v;
}

// parts of coarse tile (l0, nc) that hold cells
template <int D>
__device__ __forceinline__ int restrictParts(int l0, int nc) {
	const int cells = min(PHB_TILE_CELLS, nc - l0);
	return (cells + Restrict<D>::CELLS - 1) / Restrict<D>::CELLS;
}

// Restriction for coarse sub-tile `sub` (part sub % PER_TILE of tile sub / PER_TILE) of level
// l+1: b_{l+1} = P^T (b_l - A_l omega D^-1 b_l). Level vectors are read with plain loads: in
// the persistent solver other CTAs wrote them earlier in the same launch.
template <int D>
__device__ __forceinline__ void amgRestrictSub(const AmgView<D> &mg, int l, int sub, int32_t *sB) {
	const Dom<float, D> &cd = mg.lv[l + 1];
	const int tile = sub / Restrict<D>::PER_TILE, part = sub - tile * Restrict<D>::PER_TILE;
	const int bi = __ldg(cd.tiles + 2 * tile);
	const int l0 = __ldg(cd.tiles + 2 * tile + 1);
	const int nc = stageBlock<D>(cd, bi, sB);
	if (part < restrictParts<D>(l0, nc)) amgRestrictPart<D>(mg, l, bi, l0, nc, part, sB);
}

// Prolongation and post-smoothing for fine tile `tile` of level l (l < nlevels-1), cells
// j0, j0 + 1, ... < j1 of each thread (j0 = 0, j1 = CPT: the whole tile; a quarter tile:
// j1 = j0 + 1): out = x1 + omega D^-1 (b - A x1), x1 = omega D^-1 b + P e, e = x_{l+1}.
// Returns this thread's share of (b, out).
template <int D>
__device__ __forceinline__ double amgProlongTile(const AmgView<D> &mg, int l, int tile, int32_t *sB, float *out, int j0 = 0,
		int j1 = CPT) {
	const Dom<float, D> &fd = mg.lv[l], &cd = mg.lv[l + 1];
	const float *A = mg.A[l];
	const float *wd = mg.wd[l];
	const float *b = mg.b[l];
	const float *e = mg.x[l + 1];
	const int bi = __ldg(fd.tiles + 2 * tile);
	const int l0 = __ldg(fd.tiles + 2 * tile + 1);
	const int nc = stageBlock<D>(fd, bi, sB);
	const int32_t *CB = cd.blk(bi);
	const int64_t N = fd.ncells;
	double dot = 0;
	for (int j = j0; j < j1; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const float d = amgDiag(A, c.g);
		const float wdi = __ldg(wd + c.g);
		const float bc = b[c.g];
		const float xi = bc * wdi + e[coarseCell<D>(CB, sB, c.p)];
		float y = d * xi;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			const int ax = f >> 1;
			int64_t ng, ce;
			if (!atBound(sB, f, c.p)) {
				int64_t step = 1;
				if (ax >= 1) step *= sB[B_NX];
				if (ax >= 2) step *= sB[B_NY];
				ng = (f & 1) ? c.g + step : c.g - step;
				int p2[3] = {c.p[0], c.p[1], c.p[2]};
				p2[ax] += (f & 1) ? 1 : -1;
				ce = coarseCell<D>(CB, sB, p2);
			} else {
				if (fType(sB, f) == FT_FIXED) continue;
				const Nbr n = neighbor<float, D>(fd, c, f);
				ng = n.g;
				const int32_t *nCB = n.B == sB ? CB : cd.blk(int((n.B - fd.blocks) / PHB_BREC));
				ce = coarseCell<D>(nCB, n.B, n.p);
			}
			y += __ldg(A + (f + 1) * N + c.g) * (b[ng] * __ldg(wd + ng) + e[ce]);
		}
		const float z = xi + wdi * (bc - y);
		out[c.g] = z;
		dot += double(bc) * double(z);
	}
	return dot;
}

// Last level of the cycle: x = C b per instance with its dense operator C (the coarsest
// inverse, or the folded cycle below it), one warp per row; rows are dealt out to warps
// `warp`, `warp + nwarps`, ...
template <int D>
__device__ __forceinline__ void amgCoarseRows(const AmgView<D> &mg, int warp, int nwarps, int row0 = 0, int row1 = -1) {
	const int L = mg.nlevels - 1;
	const Dom<float, D> &cd = mg.lv[L];
	const int lane = threadIdx.x & 31;
	const int cn = mg.cn;
	const float *b = mg.b[L];
	float *x = mg.x[L];
	const int rows = row1 < 0 ? cd.ninst * cn : row1;
	for (int row = row0 + warp; row < rows; row += nwarps) {
		const int inst = row / cn, r = row - inst * cn;
		const int off = __ldg(cd.insts + inst * PHB_IREC + I_CELLOFF);
		const int n = min(cn, __ldg(cd.insts + inst * PHB_IREC + I_NCELLS));
		if (r >= n) continue;
		const double *M = mg.inv + ((size_t)inst * cn + r) * cn;
		double s = 0;
		for (int c = lane; c < n; c += 32) s += __ldg(M + c) * double(b[off + c]);
		s = amgWarpSum(s);
		if (lane == 0) x[off + r] = float(s);
	}
}

// kernels of one cycle, launched level by level (the non-persistent solver modes and
// phb_amg_vcycle)
// quarter tiles of the prolongation: one cell per thread on the coarse levels
constexpr int AMG_SUBTILES = CPT;

template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAmgRestrict(AmgView<D> mg, int l) {
	__shared__ int32_t sB[PHB_BREC];
	amgRestrictSub<D>(mg, l, blockIdx.x, sB);
}

// one quarter tile per CTA (the coarse levels have few tiles)
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAmgProlong(AmgView<D> mg, int l) {
	__shared__ int32_t sB[PHB_BREC];
	const int q = blockIdx.x % AMG_SUBTILES;
	amgProlongTile<D>(mg, l, blockIdx.x / AMG_SUBTILES, sB, mg.x[l], q, q + 1);
}

template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAmgCoarse(AmgView<D> mg) {
	amgCoarseRows<D>(mg, int(blockIdx.x * (PHB_TILE / 32) + (threadIdx.x >> 5)), int(gridDim.x * (PHB_TILE / 32)));
}

// Launch the cycle down to the coarsest level and back up to level `stop` (0: the whole
// cycle; 1: the caller runs level 0's prolongation itself).
template <int D>
__host__ inline cudaError_t launchAmgCycle(const AmgView<D> &mg, cudaStream_t s, int stop) {
	const int L = mg.nlevels;
	for (int l = 0; l + 1 < L; ++l) kAmgRestrict<D><<<mg.lv[l + 1].ntiles * Restrict<D>::PER_TILE, PHB_TILE, 0, s>>>(mg, l);
	const int rows = mg.lv[L - 1].ninst * mg.cn;
	const int warpsPerCta = PHB_TILE / 32;
	kAmgCoarse<D><<<(rows + warpsPerCta - 1) / warpsPerCta, PHB_TILE, 0, s>>>(mg);
	for (int l = L - 2; l >= stop; --l) kAmgProlong<D><<<mg.lv[l].ntiles * AMG_SUBTILES, PHB_TILE, 0, s>>>(mg, l);
	return cudaGetLastError();
}

} // namespace phb
