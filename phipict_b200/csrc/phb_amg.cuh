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
	// level 0 runs on quads of four consecutive cells: vector loads when its operands allow
	{
		const void *ps[4] = {v.A[0], v.wd[0], r, z};
		int ok = v.lv[0].ncells % 4 == 0;
		for (const void *p : ps) ok = ok && ((uintptr_t)p & 15) == 0;
		v.lv[0].vec4 = ok;
	}
	v.inv = a.coarse_inv;
	v.cn = a.coarse_n;
	// the cycle ends at level T, whose dense operator stands for everything below it
	v.nlevels = ((a.tail_level >= 1 && a.tail_level < a.nlevels) ? a.tail_level : a.nlevels - 1) + 1;
	v.omega = a.omega;
	return v;
}

// The finest level of a large grid (bandwidth-bound: several tiles per resident CTA) runs its
// restriction one coarse cell per thread and its prolongation on quads, which move the same
// bytes with far fewer instructions; a smaller grid is bound by latency and keeps the
// per-cell forms, which spread the work over more threads. Both give the same bits.
constexpr int64_t AMG_QUAD_MIN_CELLS = 1 << 20;
template <int D>
__host__ __device__ __forceinline__ bool amgFineQuads(const AmgView<D> &mg) { return mg.lv[0].ncells >= AMG_QUAD_MIN_CELLS; }

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

// Fine residual b_i - (A omega D^-1 b)_i at cell c of level fd (x0 = omega D^-1 b evaluated
// at the stencil points).
template <int D>
__device__ __forceinline__ float amgFineResidual(const Dom<float, D> &fd, const float *A, const float *wd, const float *b, const Cell &c) {
	const int64_t N = fd.ncells;
	const float bi_ = b[c.g];
	float y = __ldg(A + c.g) * (bi_ * __ldg(wd + c.g)); // A_ii x0_i
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		const int64_t nb = neighborIndex<float, D>(fd, c, f);
		if (nb >= 0) y = fmaf(__ldg(A + (f + 1) * N + c.g), b[nb] * __ldg(wd + nb), y);
	}
	return bi_ - y;
}

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
			v = amgFineResidual<D>(fd, A, wd, b, c);
		}
	}
#pragma unroll
	for (int m = 1; m < R::G; m <<= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
	if (cvalid && o == 0) bc[sB[B_CELLOFF] + lc] = v;
}

// Restriction of a fine level, one coarse cell per thread (PHB_TILE consecutive coarse cells
// per CTA, RESTRICT1_PER_TILE CTAs per coarse tile): where the blocks halve along every axis
// and the aggregate's neighbour rows lie inside the block, the thread evaluates the 2^d fine
// residuals of its aggregate row by row, two x-adjacent fine cells at a time (8-byte vector
// loads when aligned); any other aggregate takes amgFineResidual per fine cell. Both sum in
// the order of the lane shuffle tree of amgRestrictPart (x pairs, then y, then z), so all
// three forms give the same bits.
constexpr int RESTRICT1_PER_TILE = PHB_TILE_CELLS / PHB_TILE;

__device__ __forceinline__ void ld2f(const float *p, bool al, float (&v)[2]) {
	if (al) {
		const float2 f = *reinterpret_cast<const float2 *>(p);
		v[0] = f.x;
		v[1] = f.y;
	} else {
		v[0] = p[0];
		v[1] = p[1];
	}
}

template <int D>
__device__ __forceinline__ void amgRestrictCoarseCell(const AmgView<D> &mg, int l, int sub, int32_t *sB) {
	const Dom<float, D> &fd = mg.lv[l], &cd = mg.lv[l + 1];
	const int tile = sub / RESTRICT1_PER_TILE, part = sub - tile * RESTRICT1_PER_TILE;
	const int bi = __ldg(cd.tiles + 2 * tile);
	const int l0 = __ldg(cd.tiles + 2 * tile + 1);
	const int nc = stageBlock<D>(cd, bi, sB);
	const int lc = l0 + part * PHB_TILE + int(threadIdx.x);
	if (lc >= nc || lc >= l0 + PHB_TILE_CELLS) return;
	const int32_t *FB = fd.blk(bi);
	const float *A = mg.A[l];
	const float *wd = mg.wd[l];
	const float *b = mg.b[l];
	const int64_t N = fd.ncells;
	const int cnx = sB[B_NX], cny = sB[B_NY], cnz = D > 2 ? sB[B_NZ] : 1;
	const int cx = lc % cnx, cy = (lc / cnx) % cny, cz = D > 2 ? lc / (cnx * cny) : 0;
	const int fnx = __ldg(FB + B_NX), fny = __ldg(FB + B_NY), fnz = D > 2 ? __ldg(FB + B_NZ) : 1;
	const int64_t foff = __ldg(FB + B_CELLOFF);
	bool fast = fnx == 2 * cnx && fny == 2 * cny && cy >= 1 && cy <= cny - 2;
	if (D > 2) fast = fast && fnz == 2 * cnz && cz >= 1 && cz <= cnz - 2;
	constexpr int R = D > 2 ? 4 : 2; // fine rows of an aggregate: (y0 + (r & 1), z0 + (r >> 1))
	float rx[R];
	if (!fast) {
		Cell c;
		c.B = FB;
		c.b = bi;
		const int cp[3] = {cx, cy, cz};
		const bool co[3] = {fnx > cnx, fny > cny, D > 2 && fnz > cnz};
#pragma unroll
		for (int r = 0; r < R; ++r) {
			float s2[2];
#pragma unroll
			for (int ox = 0; ox < 2; ++ox) {
				const int o[3] = {ox, r & 1, r >> 1};
				bool valid = true;
#pragma unroll
				for (int a = 0; a < 3; ++a) {
					const int fs = a == 0 ? fnx : a == 1 ? fny : fnz;
					c.p[a] = co[a] ? 2 * cp[a] + o[a] : cp[a];
					valid &= co[a] ? c.p[a] < fs : o[a] == 0;
				}
				if (D < 3) c.p[2] = 0;
				s2[ox] = 0.f;
				if (valid) {
					c.g = (int)(foff + flat(FB, c.p));
					c.mi = c.g;
					s2[ox] = amgFineResidual<D>(fd, A, wd, b, c);
				}
			}
			rx[r] = s2[0] + s2[1];
		}
	} else {
		const int x0 = 2 * cx;
		const int64_t sy = fnx, sz = (int64_t)fnx * fny;
		const bool al = fd.vec4 && ((foff | fnx) & 1) == 0;
		// b wd at the two fine cells of fine row (y, z) starting at x0
		auto bw2 = [&](int y, int z, float (&v)[2]) {
			const int64_t g = foff + x0 + sy * y + sz * z;
			float bb[2], ww[2];
			ld2f(b + g, al, bb);
			ld2f(wd + g, al, ww);
			v[0] = bb[0] * ww[0];
			v[1] = bb[1] * ww[1];
		};
		const int y0 = 2 * cy, z0 = 2 * cz;
		// x neighbours at the row ends: inside the block, across its x face, or none (fixed)
		const bool wIn = x0 > 0, eIn = x0 + 2 <= fnx - 1;
		const bool wHas = wIn || fType(FB, 0) != FT_FIXED, eHas = eIn || fType(FB, 1) != FT_FIXED;
		float c2[R][2]; // b wd at the aggregate's own cells
#pragma unroll
		for (int r = 0; r < R; ++r) bw2(y0 + (r & 1), z0 + (r >> 1), c2[r]);
#pragma unroll
		for (int r = 0; r < R; ++r) {
			const int y = y0 + (r & 1), z = z0 + (r >> 1);
			const int64_t g = foff + x0 + sy * y + sz * z;
			float bb[2];
			ld2f(b + g, al, bb);
			float w = 0.f, e = 0.f;
			if (wIn) w = b[g - 1] * __ldg(wd + g - 1);
			else if (wHas) {
				Cell c;
				c.B = FB; c.b = bi; c.p[0] = 0; c.p[1] = y; c.p[2] = z; c.g = (int)g; c.mi = c.g;
				const int64_t nb = neighborIndex<float, D>(fd, c, 0);
				w = b[nb] * __ldg(wd + nb);
			}
			if (eIn) e = b[g + 2] * __ldg(wd + g + 2);
			else if (eHas) {
				Cell c;
				c.B = FB; c.b = bi; c.p[0] = x0 + 1; c.p[1] = y; c.p[2] = z; c.g = (int)(g + 1); c.mi = c.g;
				const int64_t nb = neighborIndex<float, D>(fd, c, 1);
				e = b[nb] * __ldg(wd + nb);
			}
			// y and z neighbour rows: the aggregate's own rows or the rows just outside it
			float ym[2], yp[2], zm[2] = {0.f, 0.f}, zp[2] = {0.f, 0.f};
			if (r & 1) { ym[0] = c2[r - 1][0]; ym[1] = c2[r - 1][1]; bw2(y + 1, z, yp); }
			else { bw2(y - 1, z, ym); yp[0] = c2[r + 1][0]; yp[1] = c2[r + 1][1]; }
			if (D > 2) {
				if (r >> 1) { zm[0] = c2[r - 2][0]; zm[1] = c2[r - 2][1]; bw2(y, z + 1, zp); }
				else { bw2(y, z - 1, zm); zp[0] = c2[(r + 2) % R][0]; zp[1] = c2[(r + 2) % R][1]; }
			}
			float a[2], yv[2];
			ld2f(A + g, al, a);
			yv[0] = a[0] * c2[r][0];
			yv[1] = a[1] * c2[r][1];
			ld2f(A + N + g, al, a);
			if (wHas) yv[0] = fmaf(a[0], w, yv[0]);
			yv[1] = fmaf(a[1], c2[r][0], yv[1]);
			ld2f(A + 2 * N + g, al, a);
			yv[0] = fmaf(a[0], c2[r][1], yv[0]);
			if (eHas) yv[1] = fmaf(a[1], e, yv[1]);
			ld2f(A + 3 * N + g, al, a);
			yv[0] = fmaf(a[0], ym[0], yv[0]);
			yv[1] = fmaf(a[1], ym[1], yv[1]);
			ld2f(A + 4 * N + g, al, a);
			yv[0] = fmaf(a[0], yp[0], yv[0]);
			yv[1] = fmaf(a[1], yp[1], yv[1]);
			if (D > 2) {
				ld2f(A + 5 * N + g, al, a);
				yv[0] = fmaf(a[0], zm[0], yv[0]);
				yv[1] = fmaf(a[1], zm[1], yv[1]);
				ld2f(A + 6 * N + g, al, a);
				yv[0] = fmaf(a[0], zp[0], yv[0]);
				yv[1] = fmaf(a[1], zp[1], yv[1]);
			}
			rx[r] = (bb[0] - yv[0]) + (bb[1] - yv[1]);
		}
	}
	float v = rx[0] + rx[1];
	if (D > 2) v = v + (rx[2 % R] + rx[3 % R]);
	mg.b[l + 1][sB[B_CELLOFF] + lc] = v;
}

// parts of coarse tile (l0, nc) that hold cells
template <int D>
__device__ __forceinline__ int restrictParts(int l0, int nc) {
	const int cells = min(PHB_TILE_CELLS, nc - l0);
	return (cells + Restrict<D>::CELLS - 1) / Restrict<D>::CELLS;
}

// Restriction of up to NS sub-tiles sub0, sub0 + stride, ... (< nsub) of level l+1 at once:
// their block records staged together into sBs, every thread's fine residuals evaluated for
// all of them before the shuffle trees and stores, so that their loads overlap. Same
// arithmetic and summation order as amgRestrictPart.
template <int D, int NS>
__device__ __forceinline__ void amgRestrictMulti(const AmgView<D> &mg, int l, int sub0, int stride, int nsub,
		int32_t (*sBs)[PHB_BREC]) {
	using R = Restrict<D>;
	const Dom<float, D> &fd = mg.lv[l], &cd = mg.lv[l + 1];
	const float *A = mg.A[l];
	const float *wd = mg.wd[l];
	const float *b = mg.b[l];
	float *bc = mg.b[l + 1];
	int bi[NS], l0[NS], part[NS];
	__syncthreads();
#pragma unroll
	for (int s = 0; s < NS; ++s) {
		const int sub = sub0 + s * stride;
		bi[s] = -1;
		if (sub < nsub) {
			const int tile = sub / R::PER_TILE;
			part[s] = sub - tile * R::PER_TILE;
			bi[s] = __ldg(cd.tiles + 2 * tile);
			l0[s] = __ldg(cd.tiles + 2 * tile + 1);
			if (threadIdx.x < PHB_BREC) sBs[s][threadIdx.x] = __ldg(cd.blocks + bi[s] * PHB_BREC + threadIdx.x);
		}
	}
	__syncthreads();
	const int o = int(threadIdx.x) % R::G; // fine cell of its aggregate
	float v[NS];
	bool store[NS];
#pragma unroll
	for (int s = 0; s < NS; ++s) {
		v[s] = 0.f;
		store[s] = false;
		if (bi[s] < 0) continue;
		const int32_t *sB = sBs[s];
		const int nc = sB[B_NX] * sB[B_NY] * (D > 2 ? sB[B_NZ] : 1);
		if (part[s] >= restrictParts<D>(l0[s], nc)) continue;
		const int lc = l0[s] + part[s] * R::CELLS + int(threadIdx.x) / R::G;
		if (!(lc < nc && lc < l0[s] + PHB_TILE_CELLS)) continue;
		store[s] = o == 0;
		const int32_t *FB = fd.blk(bi[s]);
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
			c.b = bi[s];
			c.g = __ldg(FB + B_CELLOFF) + flat(FB, c.p);
			c.mi = c.g;
			v[s] = amgFineResidual<D>(fd, A, wd, b, c);
		}
	}
#pragma unroll
	for (int s = 0; s < NS; ++s) {
#pragma unroll
		for (int m = 1; m < R::G; m <<= 1) v[s] += __shfl_xor_sync(0xffffffffu, v[s], m);
	}
#pragma unroll
	for (int s = 0; s < NS; ++s) {
		if (!store[s]) continue;
		const int lc = l0[s] + part[s] * R::CELLS + int(threadIdx.x) / R::G;
		bc[sBs[s][B_CELLOFF] + lc] = v[s];
	}
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

// Prolongation and post-smoothing at one fine cell c of level l (block record in sB, its
// coarse block CB): out = x1 + omega D^-1 (b - A x1), x1 = omega D^-1 b + P e, e = x_{l+1}.
template <int D>
__device__ __forceinline__ float amgProlongCell(const AmgView<D> &mg, int l, const int32_t *sB, const int32_t *CB, const Cell &c) {
	const Dom<float, D> &fd = mg.lv[l], &cd = mg.lv[l + 1];
	const float *A = mg.A[l];
	const float *wd = mg.wd[l];
	const float *b = mg.b[l];
	const float *e = mg.x[l + 1];
	const int64_t N = fd.ncells;
	const float d = amgDiag(A, c.g);
	const float wdi = __ldg(wd + c.g);
	const float bc = b[c.g];
	const float xi = fmaf(bc, wdi, e[coarseCell<D>(CB, sB, c.p)]);
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
		y = fmaf(__ldg(A + (f + 1) * N + c.g), fmaf(b[ng], __ldg(wd + ng), e[ce]), y);
	}
	return fmaf(wdi, bc - y, xi);
}

// Prolongation and post-smoothing for fine tile `tile` of level l (l < nlevels-1), cells
// j0, j0 + 1, ... < j1 of each thread (j0 = 0, j1 = CPT: the whole tile; a quarter tile:
// j1 = j0 + 1). Returns this thread's share of (b, out).
template <int D>
__device__ __forceinline__ double amgProlongTile(const AmgView<D> &mg, int l, int tile, int32_t *sB, float *out, int j0 = 0,
		int j1 = CPT) {
	const Dom<float, D> &fd = mg.lv[l], &cd = mg.lv[l + 1];
	const float *b = mg.b[l];
	const int bi = __ldg(fd.tiles + 2 * tile);
	const int l0 = __ldg(fd.tiles + 2 * tile + 1);
	const int nc = stageBlock<D>(fd, bi, sB);
	const int32_t *CB = cd.blk(bi);
	double dot = 0;
	// every cell's value first, then the stores: amgProlongCell reads b, the stencil and the
	// coarse correction, never `out`, so the loads of all cells can be in flight together
	float z[CPT], bv[CPT];
	int g[CPT];
	int cnt = 0;
#pragma unroll
	for (int jj = 0; jj < CPT; ++jj) {
		const int j = j0 + jj;
		if (j >= j1) break;
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		z[jj] = amgProlongCell<D>(mg, l, sB, CB, c);
		bv[jj] = b[c.g];
		g[jj] = c.g;
		cnt = jj + 1;
	}
#pragma unroll
	for (int jj = 0; jj < CPT; ++jj) {
		if (jj >= cnt) break;
		out[g[jj]] = z[jj];
		dot = fma(double(bv[jj]), double(z[jj]), dot);
	}
	return dot;
}

// The same for a whole tile on quads (four consecutive cells per thread): inside a row whose
// y and z neighbours are in the block or absent behind a prescribed face (Quad::fastW), the x1
// values of the cell groups at the centre and at +-y, +-z are formed from vector loads and the
// coarse corrections of their aggregates; only row ends resolve the x neighbour across the
// block face. Same arithmetic and order as amgProlongCell for every cell.
template <int D>
__device__ __forceinline__ double amgProlongQuad(const AmgView<D> &mg, int l, int tile, int32_t *sB, float *out) {
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
	Quad q;
	quadAt<D, 1>(fd.vec4, sB, l0, nc, q);
	double dot = 0;
	if (!q.fastW) {
#pragma unroll
		for (int i = 0; i < 4; ++i) {
			if (i >= q.n) break;
			Cell c;
			quadCell<D>(q, i, c);
			const float z = amgProlongCell<D>(mg, l, sB, CB, c);
			out[c.g] = z;
			dot = fma(double(b[c.g]), double(z), dot);
		}
		return dot;
	}
	// coarse cell of fine position (x, y, z) of this block
	const bool kx = CB[B_NX] < sB[B_NX], ky = CB[B_NY] < sB[B_NY], kz = D > 2 && CB[B_NZ] < sB[B_NZ];
	const int cnx = CB[B_NX], cny = CB[B_NY];
	const int64_t coff = CB[B_CELLOFF];
	auto cidx = [&](int x, int y, int z) -> int64_t {
		return coff + (kx ? x >> 1 : x) + (int64_t)cnx * ((ky ? y >> 1 : y) + (int64_t)cny * (kz ? z >> 1 : z));
	};
	// x1 of the four cells of the group at offset off, row (y, z)
	auto x1Group = [&](int64_t off, bool al, int y, int z, float (&x1)[4]) {
		float bv[4], wv[4];
		ld4(b + q.g + off, 4, al, bv);
		ld4(wd + q.g + off, 4, al, wv);
#pragma unroll
		for (int i = 0; i < 4; ++i) x1[i] = fmaf(bv[i], wv[i], e[cidx(q.p[0] + i, y, z)]);
	};
	const int py = q.p[1], pz = q.p[2];
	float bc[4], wc[4], xc[4];
	ld4(b + q.g, 4, q.al, bc);
	ld4(wd + q.g, 4, q.al, wc);
#pragma unroll
	for (int i = 0; i < 4; ++i) xc[i] = fmaf(bc[i], wc[i], e[cidx(q.p[0] + i, py, pz)]);
	// x neighbours of the row ends
	bool hasW = true, hasE = true;
	float xw = 0.f, xe = 0.f;
	{
		Cell c;
		c.B = sB;
		c.b = bi;
		c.p[1] = py;
		c.p[2] = pz;
		if (q.p[0] > 0) {
			xw = fmaf(b[q.g - 1], __ldg(wd + q.g - 1), e[cidx(q.p[0] - 1, py, pz)]);
		} else if (fType(sB, 0) == FT_FIXED) {
			hasW = false;
		} else {
			c.p[0] = 0;
			c.g = (int)q.g;
			c.mi = c.g;
			const Nbr n = neighbor<float, D>(fd, c, 0);
			const int32_t *nCB = n.B == sB ? CB : cd.blk(int((n.B - fd.blocks) / PHB_BREC));
			xw = fmaf(b[n.g], __ldg(wd + n.g), e[coarseCell<D>(nCB, n.B, n.p)]);
		}
		if (q.p[0] + 4 <= sB[B_NX] - 1) {
			xe = fmaf(b[q.g + 4], __ldg(wd + q.g + 4), e[cidx(q.p[0] + 4, py, pz)]);
		} else if (fType(sB, 1) == FT_FIXED) {
			hasE = false;
		} else {
			c.p[0] = q.p[0] + 3;
			c.g = (int)(q.g + 3);
			c.mi = c.g;
			const Nbr n = neighbor<float, D>(fd, c, 1);
			const int32_t *nCB = n.B == sB ? CB : cd.blk(int((n.B - fd.blocks) / PHB_BREC));
			xe = fmaf(b[n.g], __ldg(wd + n.g), e[coarseCell<D>(nCB, n.B, n.p)]);
		}
	}
	float a[4], y[4];
	ld4(A + q.g, 4, q.al, a);
#pragma unroll
	for (int i = 0; i < 4; ++i) y[i] = (a[i] != 0.f ? a[i] : 1.f) * xc[i];
	ld4(A + N + q.g, 4, q.al, a);
	if (hasW) y[0] = fmaf(a[0], xw, y[0]);
#pragma unroll
	for (int i = 1; i < 4; ++i) y[i] = fmaf(a[i], xc[i - 1], y[i]);
	ld4(A + 2 * N + q.g, 4, q.al, a);
#pragma unroll
	for (int i = 0; i < 3; ++i) y[i] = fmaf(a[i], xc[i + 1], y[i]);
	if (hasE) y[3] = fmaf(a[3], xe, y[3]);
#pragma unroll
	for (int sl = 3; sl < 2 * D + 1; ++sl) {
		if ((q.miss >> (sl - 3)) & 1) continue; // behind a prescribed face: no neighbour
		const bool ys = sl < 5;
		const int dir = (sl & 1) ? -1 : 1; // slots 3, 5: the minus side
		const int64_t off = (ys ? (int64_t)q.sy : (int64_t)q.sz) * dir;
		float xn[4];
		x1Group(off, ys ? q.alY : q.alZ, ys ? py + dir : py, ys ? pz : pz + dir, xn);
		ld4(A + sl * N + q.g, 4, q.al, a);
#pragma unroll
		for (int i = 0; i < 4; ++i) y[i] = fmaf(a[i], xn[i], y[i]);
	}
	float z[4];
#pragma unroll
	for (int i = 0; i < 4; ++i) {
		z[i] = fmaf(wc[i], bc[i] - y[i], xc[i]);
		dot = fma(double(bc[i]), double(z[i]), dot);
	}
	st4(out + q.g, 4, q.al, z);
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

// the finest restriction on a large grid: one coarse cell per thread
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAmgRestrictFine(AmgView<D> mg) {
	__shared__ int32_t sB[PHB_BREC];
	amgRestrictCoarseCell<D>(mg, 0, blockIdx.x, sB);
}

// one quarter tile per CTA (the coarse levels have few tiles)
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAmgProlong(AmgView<D> mg, int l) {
	__shared__ int32_t sB[PHB_BREC];
	const int q = blockIdx.x % AMG_SUBTILES;
	amgProlongTile<D>(mg, l, blockIdx.x / AMG_SUBTILES, sB, mg.x[l], q, q + 1);
}

// the finest prolongation: whole tiles on quads
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAmgProlongFine(AmgView<D> mg) {
	__shared__ int32_t sB[PHB_BREC];
	amgProlongQuad<D>(mg, 0, blockIdx.x, sB, mg.x[0]);
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
	for (int l = 0; l + 1 < L; ++l) {
		if (l == 0 && amgFineQuads(mg)) kAmgRestrictFine<D><<<mg.lv[1].ntiles * RESTRICT1_PER_TILE, PHB_TILE, 0, s>>>(mg);
		else kAmgRestrict<D><<<mg.lv[l + 1].ntiles * Restrict<D>::PER_TILE, PHB_TILE, 0, s>>>(mg, l);
	}
	const int rows = mg.lv[L - 1].ninst * mg.cn;
	const int warpsPerCta = PHB_TILE / 32;
	kAmgCoarse<D><<<(rows + warpsPerCta - 1) / warpsPerCta, PHB_TILE, 0, s>>>(mg);
	for (int l = L - 2; l >= stop; --l) {
		if (l == 0 && amgFineQuads(mg)) kAmgProlongFine<D><<<mg.lv[0].ntiles, PHB_TILE, 0, s>>>(mg);
		else kAmgProlong<D><<<mg.lv[l].ntiles * AMG_SUBTILES, PHB_TILE, 0, s>>>(mg, l);
	}
	return cudaGetLastError();
}

} // namespace phb
