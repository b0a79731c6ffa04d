// Non-orthogonal Laplace terms of curvilinear grids (phiPICT piso/device/nonortho_laplace.cuh,
// nonortho_rhs.cuh and the corner interpolation of block_data.cuh:477-620).
//
// On a grid whose cell transform M has a non-diagonal metric, the Laplacian of a face
// carries cross terms det Minv[n] . Minv[t] times the tangential derivative at the face. The
// tangential derivative is the difference of the two corner values of the face, each an
// average of the cells around the corner (normally four). Depending on the flag bits, the
// parts of that average that fall on the cell itself and on its face neighbours go to the
// matrix (CENTER_MATRIX, DIRECT_MATRIX) and the rest, the diagonal cells, to the right-hand
// side from the last result (DIAGONAL_RHS, DIRECT_RHS).
//
// These are per-cell gathers with short, data-dependent walks around the corners; they run
// only on domains whose metric has cross terms and are not on the rectilinear hot path.
// Block records, metrics and fields are read through the read-only cache.
#pragma once

#include "phb_device.cuh"

namespace phb {

// flag bits (piso/non_ortho_flags.h:23-27)
enum { NO_DIRECT_MATRIX = 1, NO_DIRECT_RHS = 2, NO_DIAGONAL_MATRIX = 4, NO_DIAGONAL_RHS = 8, NO_CENTER_MATRIX = 16 };
constexpr int NO_MATRIX_BITS = NO_CENTER_MATRIX | NO_DIRECT_MATRIX;
constexpr int NO_RHS_BITS = NO_DIRECT_RHS | NO_DIAGONAL_RHS;

// What a corner walk reads (GridDataType of block_data.cuh): nothing but the fixed faces
// (matrix assembly), the pressure result [cells], component w of the velocity result
// [inst][d][cells], or channel w of the scalar result [inst][channels][cells].
enum { NF_MARK = 0, NF_PRESSURE = 1, NF_VELOCITY = 2, NF_SCALAR = 3 };

template <typename S>
struct NField {
	int kind;
	int w;
	const S *cells;
	ScalarView sv; // NF_SCALAR: face types and values of the channels
};

// A position in a block (block index, coordinates).
struct BPos {
	int b;
	int p[3];
};

// The value of components F.w .. F.w+NC-1 at cell q (zeros for a matrix walk, which reads no
// cell data).
template <typename S, int D, int NC = 1>
__device__ __forceinline__ void nfCell(const Dom<S, D> &dom, const NField<S> &F, const BPos &q, S (&v)[NC]) {
	if (F.kind == NF_MARK || !F.cells) {
#pragma unroll
		for (int j = 0; j < NC; ++j) v[j] = 0;
		return;
	}
	const int32_t *B = dom.blk(q.b);
	const int64_t g = B[B_CELLOFF] + flat(B, q.p);
#pragma unroll
	for (int j = 0; j < NC; ++j) {
		if (F.kind == NF_PRESSURE) v[j] = __ldg(F.cells + g);
		else if (F.kind == NF_VELOCITY) v[j] = __ldg(F.cells + vidx<D>(B, g, F.w + j));
		else v[j] = __ldg(F.cells + sidx(B, g, F.w + j, F.sv.channels));
	}
}
// getFixedBoundaryType (block_data.cuh:111-135): true for a Neumann face
template <typename S, int D>
__device__ __forceinline__ bool nfNeumann(const Dom<S, D> &dom, const NField<S> &F, const int32_t *B, int f) {
	const int fid = fRec(B, f)[5];
	if (F.kind == NF_VELOCITY) return dom.fix(fid)[F_VELTYPE] != 0;
	if (F.kind == NF_SCALAR) return F.sv.types[(int64_t)fid * F.sv.channels + F.w] != 0;
	return false;
}
// getFixedBoundaryData (block_data.cuh:137-205) at the face cell of p; the fixed faces carry
// no pressure data
template <typename S, int D, int NC = 1>
__device__ __forceinline__ void nfFixed(const Dom<S, D> &dom, const NField<S> &F, const int32_t *B, int f, const int *p, S (&v)[NC]) {
	const int fid = fRec(B, f)[5];
	const int32_t *FR = dom.fix(fid);
#pragma unroll
	for (int j = 0; j < NC; ++j) {
		if (F.kind == NF_MARK) v[j] = S(1);
		else if (F.kind == NF_VELOCITY) v[j] = fixedVel<S, D>(dom, FR, faceCell(B, f, p), F.w + j);
		else if (F.kind == NF_SCALAR) v[j] = F.sv.values ? scalarFixed<S>(F.sv, FR, fid, F.w + j, faceCell(B, f, p)) : S(0);
		else v[j] = S(0);
	}
}

// computeConnectedDir (topology.cuh:226-236): direction dir of block B as seen from the
// block across B's connected face f
__device__ __forceinline__ int connDir(const int32_t *B, int f, int dir, int dims) {
	return fRec(B, f)[2 + posMod((dir >> 1) - (f >> 1), dims)] ^ (dir & 1);
}

// One step from q across direction dir; false at a fixed face (q unchanged). A connected
// face lands one cell inside the other block (computeConnectedPos with borderOffset 1, as
// the reference's neighbour reads and corner walks call it, block_data.cuh:299,397,571).
template <typename S, int D>
__device__ __forceinline__ bool stepAcross(const Dom<S, D> &dom, BPos &q, int dir) {
	const int32_t *B = dom.blk(q.b);
	const int ax = dir >> 1;
	if (!atBound(B, dir, q.p)) { q.p[ax] += (dir & 1) ? 1 : -1; return true; }
	const int t = fType(B, dir);
	if (t == FT_FIXED) return false;
	if (t == FT_PERIODIC) { q.p[ax] = (dir & 1) ? 0 : B[B_NX + ax] - 1; return true; }
	int ob, op[3];
	connectedPos<S, D>(dom, B, dir, q.p, 1, ob, op);
	q.b = ob;
	q.p[0] = op[0]; q.p[1] = op[1]; q.p[2] = op[2];
	return true;
}
// getBlockDataNeighbor (block_data.cuh:276-318)
template <typename S, int D, int NC = 1>
__device__ void neighborData(const Dom<S, D> &dom, const NField<S> &F, BPos q, int dir, S (&v)[NC]) {
	if (!stepAcross<S, D>(dom, q, dir)) nfFixed<S, D, NC>(dom, F, dom.blk(q.b), dir, q.p, v);
	else nfCell<S, D, NC>(dom, F, q, v);
}
// getBlockDataNeighborDiagonal (block_data.cuh:372-420): dir1 first unless the starting
// block's dir1 face is fixed; the second step keeps its direction index in the block reached
template <typename S, int D, int NC = 1>
__device__ void diagonalData(const Dom<S, D> &dom, const NField<S> &F, BPos q, int dir1, int dir2, S (&v)[NC]) {
	const bool first1 = fType(dom.blk(q.b), dir1) != FT_FIXED;
	const int dirs[2] = {first1 ? dir1 : dir2, first1 ? dir2 : dir1};
	for (int i = 0; i < 2; ++i)
		if (!stepAcross<S, D>(dom, q, dirs[i])) {
			nfFixed<S, D, NC>(dom, F, dom.blk(q.b), dirs[i], q.p, v);
			return;
		}
	nfCell<S, D, NC>(dom, F, q, v);
}

template <typename S, int NC = 1>
struct CornerValue {
	S data[NC];
	int numCells; // 0: the value came from a fixed face
	bool neumann; // that face's type
};

// getCornerValue (block_data.cuh:501-620) with includeDepth0 false and maxDepth 2: two walks
// go around the corner between dir1 and dir2 in opposite senses, one cell per depth each,
// until they meet or a fixed face ends one of them. At depth 2 the walks normally meet at
// the diagonal cell (four cells); three blocks meeting at a corner give three. One walk gives
// the corner values of NC components.
template <typename S, int D, int NC = 1>
__device__ CornerValue<S, NC> cornerWalk(const Dom<S, D> &dom, const NField<S> &F, const BPos &start, int dir1, int dir2, bool depth1) {
	CornerValue<S, NC> out;
	S data[NC], v[NC];
#pragma unroll
	for (int j = 0; j < NC; ++j) data[j] = 0;
	{
		// a cell at least one cell away from every face of its block: the walks reach the two
		// face neighbours at depth 1 and meet at the diagonal cell at depth 2 (four cells), with
		// the data summed in the walk's order
		const int32_t *B = dom.blk(start.b);
		bool inner = true;
#pragma unroll
		for (int a = 0; a < D; ++a) inner = inner && start.p[a] >= 1 && start.p[a] <= B[B_NX + a] - 2;
		if (inner) {
			BPos n1 = start, n2 = start;
			n1.p[dir1 >> 1] += (dir1 & 1) ? 1 : -1;
			n2.p[dir2 >> 1] += (dir2 & 1) ? 1 : -1;
			BPos dg = n1;
			dg.p[dir2 >> 1] += (dir2 & 1) ? 1 : -1;
			if (depth1) {
				nfCell<S, D, NC>(dom, F, n1, v);
#pragma unroll
				for (int j = 0; j < NC; ++j) data[j] += v[j];
				nfCell<S, D, NC>(dom, F, n2, v);
#pragma unroll
				for (int j = 0; j < NC; ++j) data[j] += v[j];
			}
			nfCell<S, D, NC>(dom, F, dg, v);
#pragma unroll
			for (int j = 0; j < NC; ++j) out.data[j] = (data[j] + v[j]) / S(4);
			out.numCells = 4;
			out.neumann = false;
			return out;
		}
	}
	BPos w[2] = {start, start};
	int d1[2] = {dir1, dir2}, d2[2] = {dir2, dir1};
	int num = 1;
#pragma unroll
	for (int depth = 1; depth <= 2; ++depth) {
#pragma unroll
		for (int d = 0; d < 2; ++d) {
			const int32_t *B = dom.blk(w[d].b);
			const int a = d1[d], t2 = d2[d];
			const int ax = a >> 1;
			if (atBound(B, a, w[d].p)) {
				const int t = fType(B, a);
				if (t == FT_FIXED) {
					out.neumann = nfNeumann<S, D>(dom, F, B, a);
					out.numCells = 0;
					nfFixed<S, D, NC>(dom, F, B, a, w[d].p, out.data);
					if (atBound(B, t2, w[d].p)) return out;
					int q[3] = {w[d].p[0], w[d].p[1], w[d].p[2]};
					q[t2 >> 1] += (t2 & 1) ? 1 : -1;
					nfFixed<S, D, NC>(dom, F, B, a, q, v);
#pragma unroll
					for (int j = 0; j < NC; ++j) out.data[j] = (out.data[j] + v[j]) * S(0.5);
					return out;
				}
				if (t == FT_CONNECTED) {
					const int n1 = connDir(B, a, t2, D);
					const int n2 = connDir(B, a, a, D) ^ 1;
					int ob, op[3];
					connectedPos<S, D>(dom, B, a, w[d].p, 1, ob, op);
					w[d].b = ob;
					w[d].p[0] = op[0]; w[d].p[1] = op[1]; w[d].p[2] = op[2];
					d1[d] = n1;
					d2[d] = n2;
				} else {
					w[d].p[ax] = (a & 1) ? 0 : B[B_NX + ax] - 1;
					d1[d] = t2;
					d2[d] = a ^ 1;
				}
			} else {
				w[d].p[ax] += (a & 1) ? 1 : -1;
				d1[d] = t2;
				d2[d] = a ^ 1;
			}
			const BPos &o = w[d ^ 1];
			if (w[d].b == o.b && w[d].p[0] == o.p[0] && w[d].p[1] == o.p[1] && w[d].p[2] == o.p[2]) {
#pragma unroll
				for (int j = 0; j < NC; ++j) out.data[j] = data[j] / S(num);
				out.numCells = num;
				out.neumann = false;
				return out;
			}
			if (depth > 1 || depth1) {
				nfCell<S, D, NC>(dom, F, w[d], v);
#pragma unroll
				for (int j = 0; j < NC; ++j) data[j] += v[j];
			}
			++num;
		}
	}
#pragma unroll
	for (int j = 0; j < NC; ++j) out.data[j] = data[j] / S(num);
	out.numCells = num;
	out.neumann = false;
	return out;
}

// det Minv[a] . Minv[c] at metric index mi (discretization.cuh:419-469)
template <typename S, int D>
__device__ __forceinline__ S lapCross(const Dom<S, D> &dom, int64_t mi, int a, int c) {
	S s = 0;
#pragma unroll
	for (int j = 0; j < D; ++j) s += dom.m(Tr<D>::MINV + a * D + j, mi) * dom.m(Tr<D>::MINV + c * D + j, mi);
	return dom.m(Tr<D>::DET, mi) * s;
}
// the same with the face metrics of fixed-face cell fi
template <typename S, int D>
__device__ __forceinline__ S lapCrossFace(const Dom<S, D> &dom, int64_t fi, int a, int c) {
	S s = 0;
#pragma unroll
	for (int j = 0; j < D; ++j) s += dom.fm(Tr<D>::MINV + a * D + j, fi) * dom.fm(Tr<D>::MINV + c * D + j, fi);
	return dom.fm(Tr<D>::DET, fi) * s;
}
__device__ __forceinline__ int64_t metricIndex(const int32_t *B, const int *p) { return B[B_METOFF] + flat(B, p); }
__device__ __forceinline__ int64_t cellIndex(const int32_t *B, const int *p) { return B[B_CELLOFF] + flat(B, p); }

// interpolateNonOrthoLaplaceComponents (nonortho_laplace.cuh:52-129) without face
// transforms: ia[f][i-1] is the cross coefficient of face f with tangential axis (f/2+i) % d,
// averaged between the cell and its face neighbour with weights ra(B, g). A face gets one when
// its cell is not at either end of the face's axis or the block's face in that direction is
// not fixed, as the reference tests it.
template <typename S, int D, typename RA>
__device__ __forceinline__ void nonOrthoInterp(const Dom<S, D> &dom, const BPos &c, RA ra, S (&ia)[2 * D][2]) {
	const int32_t *B = dom.blk(c.b);
	const int64_t miP = metricIndex(B, c.p);
	const S raP = ra(cellIndex(B, c.p));
	// the cell's cross coefficients, one per axis pair (lapCross is symmetric bit for bit)
	S cP[3];
#pragma unroll
	for (int a = 0; a < D; ++a)
#pragma unroll
		for (int b = a + 1; b < D; ++b) cP[a + b - 1] = lapCross<S, D>(dom, miP, a, b);
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		const int ax = f >> 1;
		ia[f][0] = 0;
		ia[f][1] = 0;
		if (!((0 < c.p[ax] && c.p[ax] < B[B_NX + ax] - 1) || fType(B, f) != FT_FIXED)) continue;
		const int32_t *NB = B;
		int np[3] = {c.p[0], c.p[1], c.p[2]};
		if (atBound(B, f, c.p) && fType(B, f) == FT_CONNECTED) {
			int ob;
			connectedPos<S, D>(dom, B, f, c.p, 0, ob, np);
			NB = dom.blk(ob);
		} else if (atBound(B, f, c.p) && fType(B, f) == FT_PERIODIC) {
			np[ax] = (f & 1) ? 0 : B[B_NX + ax] - 1;
		} else {
			np[ax] += (f & 1) ? 1 : -1;
		}
		const int64_t miN = metricIndex(NB, np);
		const S raN = ra(cellIndex(NB, np));
		S rowN[D];
#pragma unroll
		for (int j = 0; j < D; ++j) rowN[j] = dom.m(Tr<D>::MINV + ax * D + j, miN);
		const S detN = dom.m(Tr<D>::DET, miN);
#pragma unroll
		for (int i = 1; i < D; ++i) {
			const int o = (ax + i) % D;
			S dN = 0; // as lapCross(miN, o, ax)
#pragma unroll
			for (int j = 0; j < D; ++j) dN += dom.m(Tr<D>::MINV + o * D + j, miN) * rowN[j];
			const int lo = ax < o ? ax : o, hi = ax < o ? o : ax;
			ia[f][i - 1] = (cP[lo + hi - 1] * raP + detN * dN * raN) * S(0.5);
		}
	}
}

// The non-orthogonal matrix terms of free face f of one row (pressure.cu:103-156,
// advection.cu:176-240), added right after the face's orthogonal terms: per tangential axis
// and side, a corner interpolated from numCells cells adds its centre and direct-neighbour
// shares (CENTER_MATRIX, DIRECT_MATRIX); a corner on a fixed gradient face (every fixed face
// for the pressure) turns into a one-sided difference from the other side; a corner on a
// fixed value face adds nothing here. sgn: +1 as the pressure matrix adds them, -1 as the
// advection matrix does. a[i-1]: the face's cross coefficient with axis (f/2 + i) % d.
// inner: the cell is at least one cell away from every face of its block, where every corner
// interpolates four cells (cornerWalk's first case) and no walk is needed.
template <typename S, int D>
__device__ void nonOrthoMatrixFace(const Dom<S, D> &dom, const NField<S> &F, const BPos &c, int f, int flags, int sgn, bool pressure,
		const S *a, S *rv, bool inner = false) {
	const bool center = flags & NO_CENTER_MATRIX, direct = flags & NO_DIRECT_MATRIX;
	const int faceSign = (f & 1) ? 1 : -1;
	for (int i = 1; i < D; ++i) {
		const int tAxis = ((f >> 1) + i) % D;
		if (a[i - 1] == S(0)) continue;
		for (int tUp = 0; tUp < 2; ++tUp) {
			const int tFace = 2 * tAxis + tUp;
			const int tSign = tUp ? 1 : -1;
			const CornerValue<S> cv = inner ? CornerValue<S>{S(0), 4, false} : cornerWalk<S, D>(dom, F, c, f, tFace, false);
			if (cv.numCells < 1) {
				if (!(pressure || cv.neumann)) continue;
				const S coef = S(faceSign * tSign) * a[i - 1] * S(0.25);
				if (center) rv[0] += S(sgn * 3) * coef;
				if (direct) { rv[f + 1] += S(sgn * 3) * coef; rv[(tFace ^ 1) + 1] -= S(sgn) * coef; }
			} else {
				const S coef = S(faceSign * tSign) * a[i - 1] * S(1.0 / double(cv.numCells));
				if (center) rv[0] += S(sgn) * coef;
				if (direct) { rv[f + 1] += S(sgn) * coef; rv[tFace + 1] += S(sgn) * coef; }
			}
		}
	}
}

// Whether cell p of block B is at least one cell away from every face of its block.
template <int D>
__device__ __forceinline__ bool innerCell(const int32_t *B, const int *p) {
	bool inner = true;
#pragma unroll
	for (int a = 0; a < D; ++a) inner = inner && p[a] >= 1 && p[a] <= B[B_NX + a] - 2;
	return inner;
}

// nonOrthoRhs for an inner cell (innerCell), all NC components of a field at once: the
// neighbours and corner cells lie in the block at fixed strides, every corner interpolates
// four cells, and the face coefficients are computed once for all components. Component w's
// value at cell index h is cells[h + base + w * cstride]; out[w] receives its sum in the
// order of nonOrthoRhs (faces, tangential axes, corners).
template <typename S, int D, int NC, typename RA>
__device__ __forceinline__ void nonOrthoRhsInner(const Dom<S, D> &dom, const S *__restrict__ cells, int64_t base, int64_t cstride,
		const int32_t *B, const int *p, int flags, RA ra, S (&out)[NC]) {
	const bool direct = flags & NO_DIRECT_RHS;
	const int64_t sy = B[B_NX], sz = (int64_t)B[B_NX] * B[B_NY];
	auto stride = [&](int a) -> int64_t { return a == 0 ? 1 : a == 1 ? sy : sz; };
	const int64_t g = cellIndex(B, p), mi = metricIndex(B, p);
	const S raP = ra(g);
	// the cell's cross coefficients, one per axis pair ((0,1), (0,2), (1,2)); the dot product
	// is symmetric in its operands, so lapCross(a, b) and lapCross(b, a) agree bit for bit
	S cP[3];
#pragma unroll
	for (int a = 0; a < D; ++a)
#pragma unroll
		for (int b = a + 1; b < D; ++b) cP[a + b - 1] = lapCross<S, D>(dom, mi, a, b);
#pragma unroll
	for (int w = 0; w < NC; ++w) out[w] = 0;
	// faces one at a time (not unrolled): every face's loads stay in flight together without
	// holding all faces' values in registers
#pragma unroll 1
	for (int f = 0; f < 2 * D; ++f) {
		const int ax = f >> 1;
		const int faceSign = (f & 1) ? 1 : -1;
		const int64_t sN = (f & 1) ? stride(ax) : -stride(ax);
		const S raN = ra(g + sN);
		// the neighbour's inverse-transform row of the face axis and its determinant, read once
		const int64_t mN = mi + sN;
		S rowN[D];
#pragma unroll
		for (int j = 0; j < D; ++j) rowN[j] = dom.m(Tr<D>::MINV + ax * D + j, mN);
		const S detN = dom.m(Tr<D>::DET, mN);
#pragma unroll
		for (int i = 1; i < D; ++i) {
			const int tAxis = (ax + i) % D;
			S dN = 0; // as lapCross(mN, tAxis, ax)
#pragma unroll
			for (int j = 0; j < D; ++j) dN += dom.m(Tr<D>::MINV + tAxis * D + j, mN) * rowN[j];
			const int lo = ax < tAxis ? ax : tAxis, hi = ax < tAxis ? tAxis : ax;
			const S faceAlpha = (cP[lo + hi - 1] * raP + detN * dN * raN) * S(0.5);
#pragma unroll
			for (int w = 0; w < NC; ++w) {
				const S *cw = cells + base + w * cstride;
				S tGrad = 0;
#pragma unroll
				for (int tUp = 0; tUp < 2; ++tUp) {
					const int64_t sT = tUp ? stride(tAxis) : -stride(tAxis);
					S data = 0;
					if (direct) {
						data += __ldg(cw + g + sN);
						data += __ldg(cw + g + sT);
					}
					data += __ldg(cw + g + sN + sT);
					tGrad += S(tUp ? 1 : -1) * (data / S(4));
				}
				out[w] -= S(faceSign) * faceAlpha * tGrad;
			}
		}
	}
}

// getNonOrthoLaplaceRHS_v2 (nonortho_rhs.cuh:27-180) without face transforms: the explicit
// cross terms of components F.w .. F.w+NC-1 of field F at cell c into sum[NC]. ra(g): the
// weight of cell g (1/A for the pressure, the viscosity for the velocity, 1 for a scalar);
// raFixed: the weight at a fixed face. Every corner is walked once for all NC components.
template <typename S, int D, int NC, typename RA>
__device__ void nonOrthoRhs(const Dom<S, D> &dom, const NField<S> &F, const BPos &c, int flags, RA ra, S raFixed, S (&sum)[NC]) {
	const bool direct = flags & NO_DIRECT_RHS, diagonal = flags & NO_DIAGONAL_RHS;
	const int32_t *B = dom.blk(c.b);
	const int64_t miP = metricIndex(B, c.p);
	const S raP = ra(cellIndex(B, c.p));
#pragma unroll
	for (int j = 0; j < NC; ++j) sum[j] = 0;
	for (int f = 0; f < 2 * D; ++f) {
		const int ax = f >> 1;
		const int faceSign = (f & 1) ? 1 : -1;
		if (atBound(B, f, c.p) && fType(B, f) == FT_FIXED) {
			if (F.kind == NF_PRESSURE || nfNeumann<S, D>(dom, F, B, f)) continue;
			const int32_t *FR = dom.fix(fRec(B, f)[5]);
			const int64_t fi = FR[F_TOFF] + faceCell(B, f, c.p);
			for (int i = 1; i < D; ++i) {
				const int tAxis = (ax + i) % D;
				const bool tLow = c.p[tAxis] == 0, tHigh = c.p[tAxis] == B[B_NX + tAxis] - 1;
				int lo[3] = {c.p[0], c.p[1], c.p[2]}, hi[3] = {c.p[0], c.p[1], c.p[2]};
				if (!tLow) lo[tAxis] -= 1;
				if (!tHigh) hi[tAxis] += 1;
				const S factor = (tLow || tHigh) ? S(1) : S(0.5);
				S vh[NC], vl[NC];
				nfFixed<S, D, NC>(dom, F, B, f, hi, vh);
				nfFixed<S, D, NC>(dom, F, B, f, lo, vl);
				const S alpha = lapCrossFace<S, D>(dom, fi, tAxis, ax);
#pragma unroll
				for (int j = 0; j < NC; ++j) sum[j] -= S(faceSign) * alpha * (factor * (vh[j] - vl[j])) * raFixed;
			}
			continue;
		}
		// resolveNeighborCell (topology.cuh:343-383) with the axis mapping of a connection
		// (getLaplaceCoefficientsSingleAxisNeighbor, discretization.cuh:565-600)
		const int32_t *NB = B;
		int np[3] = {c.p[0], c.p[1], c.p[2]};
		int map[3] = {0, 1, 2};
		if (atBound(B, f, c.p) && fType(B, f) == FT_CONNECTED) {
			int ob;
			connectedPos<S, D>(dom, B, f, c.p, 0, ob, np);
			NB = dom.blk(ob);
#pragma unroll
			for (int k = 0; k < D; ++k) map[k] = connDir(B, f, 2 * k, D) >> 1;
		} else if (atBound(B, f, c.p)) {
			np[ax] = (f & 1) ? 0 : B[B_NX + ax] - 1;
		} else {
			np[ax] += (f & 1) ? 1 : -1;
		}
		const int64_t miN = metricIndex(NB, np);
		const S raN = ra(cellIndex(NB, np));
		for (int i = 1; i < D; ++i) {
			const int tAxis = (ax + i) % D;
			const S faceAlpha = (lapCross<S, D>(dom, miP, ax, tAxis) * raP + lapCross<S, D>(dom, miN, map[tAxis], map[ax]) * raN) * S(0.5);
			S tGrad[NC];
#pragma unroll
			for (int j = 0; j < NC; ++j) tGrad[j] = 0;
			for (int tUp = 0; tUp < 2; ++tUp) {
				const int tFace = 2 * tAxis + tUp;
				const int tSign = tUp ? 1 : -1;
				const CornerValue<S, NC> cv = cornerWalk<S, D, NC>(dom, F, c, f, tFace, direct);
				if (cv.numCells == 0 && (cv.neumann || F.kind == NF_PRESSURE)) {
					const int tOther = tFace ^ 1;
					S v[NC];
					if (direct) {
						neighborData<S, D, NC>(dom, F, c, f, v);
#pragma unroll
						for (int j = 0; j < NC; ++j) tGrad[j] += S(tSign) * v[j] * S(0.75);
						neighborData<S, D, NC>(dom, F, c, tOther, v);
#pragma unroll
						for (int j = 0; j < NC; ++j) tGrad[j] += S(-tSign) * v[j] * S(0.25);
					}
					if (diagonal) {
						diagonalData<S, D, NC>(dom, F, c, f, tOther, v);
#pragma unroll
						for (int j = 0; j < NC; ++j) tGrad[j] += S(-tSign) * v[j] * S(0.25);
					}
				} else {
#pragma unroll
					for (int j = 0; j < NC; ++j) tGrad[j] += S(tSign) * cv.data[j];
				}
			}
#pragma unroll
			for (int j = 0; j < NC; ++j) sum[j] -= S(faceSign) * faceAlpha * tGrad[j];
		}
	}
}

} // namespace phb
