// CPU oracle for the phiPICT PISO/MHD step.
//
// TEST INFRASTRUCTURE ONLY. This file restates the reference algorithm on the CPU so
// that the CUDA product can be checked against it; only tests/, the smoke check and
// the CPU-baseline leg of bench.py may load it. Nothing in phipict_b200 links it.
//
// Each function names the reference file:line it follows (paths relative to the
// phiPICT source tree). Scalars are templated (double and float instantiations),
// every loop over cells is a plain OpenMP loop, and CSR rows are written exactly as
// the reference kernels write them: entries sorted by column, all values of an
// advection row divided by the cell determinant.
//
// Packed domain description (int32, produced by phipict_b200/_topology.py from the
// user's blocks and boundaries; it only carries input data, no derived topology):
//   header[HDR]   : dims, nblocks, ncells, nfixed, 0...
//   block record  : nx, ny, nz, cellOffset, then per face f=0..5 (-x,+x,-y,+y,-z,+z):
//                   type (0 fixed, 1 periodic, 2 connected), other block,
//                   axes[0..2] (connection encoding of Block::ConnectBlock), fixed id
//   fixed record  : block, face, velStatic, velType (0 Dirichlet, 1 Neumann),
//                   potType, potMaskOff, potValOff, velOff, faceCells, tOff, 0, 0
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>
#include <functional>

namespace orc {

constexpr int HDR = 8, BREC = 40, FREC = 12;
enum { FT_FIXED = 0, FT_PERIODIC = 1, FT_CONNECTED = 2 };
enum { PB_INSULATING = 0, PB_OPEN = 1, PB_DIRICHLET = 2, PB_THIN_WALL = 3 };

template <typename S>
struct Dom {
	const int32_t *desc;
	const S *Tc;     // cell transforms, [ncells][TS]
	const S *Tf;     // boundary face transforms, concatenated [faceCells][TS]
	const S *fvel;   // fixed boundary velocities
	const S *fpot;   // fixed boundary potential values
	const S *fcw;    // fixed boundary wall conductance, [nfixed]
	const int8_t *fmask; // fixed boundary potential type masks
	int dims, nb, n, nf, TS;

	Dom(const int32_t *d, const S *tc, const S *tf, const S *fv, const S *fp, const S *cw, const int8_t *fm)
		: desc(d), Tc(tc), Tf(tf), fvel(fv), fpot(fp), fcw(cw), fmask(fm) {
		dims = d[0]; nb = d[1]; n = d[2]; nf = d[3]; TS = 2 * dims * dims + 1;
	}
	const int32_t *blk(int b) const { return desc + HDR + b * BREC; }
	const int32_t *fix(int k) const { return desc + HDR + nb * BREC + k * FREC; }
	int sz(int b, int a) const { return a < dims ? blk(b)[a] : 1; }
	int off(int b) const { return blk(b)[3]; }
	int ncellsBlock(int b) const { return sz(b, 0) * sz(b, 1) * sz(b, 2); }
	const int32_t *face(int b, int f) const { return blk(b) + 4 + f * 6; }
	int ftype(int b, int f) const { return face(b, f)[0]; }
	int flat(int b, const int *p) const { return p[0] + sz(b, 0) * (p[1] + sz(b, 1) * p[2]); }
	int glob(int b, const int *p) const { return off(b) + flat(b, p); }
	const S *T(int b, const int *p) const { return Tc + (size_t)glob(b, p) * TS; }
	const S *Minv(const S *t, int row) const { return t + dims * dims + row * dims; }
	S det(const S *t) const { return t[2 * dims * dims]; }
	void unflat(int b, int local, int *p) const {
		p[0] = local % sz(b, 0);
		p[1] = (local / sz(b, 0)) % sz(b, 1);
		p[2] = local / (sz(b, 0) * sz(b, 1));
	}
	// fixed face helpers -------------------------------------------------------------
	int fixedId(int b, int f) const { return face(b, f)[5]; }
	// face cell index of pos on face f: flattenIndex with the normal coordinate 0 and the
	// normal size 1 (domain_structs_gpu.h FixedBoundaryGPU, block_data.cuh:176-184)
	int faceCell(int b, int f, const int *p) const {
		const int ax = f >> 1;
		int s[3] = {sz(b, 0), sz(b, 1), sz(b, 2)};
		int q[3] = {p[0], p[1], p[2]};
		s[ax] = 1; q[ax] = 0;
		return q[0] + s[0] * (q[1] + s[1] * q[2]);
	}
	const S *faceT(int b, int f, const int *p) const {
		const int32_t *fr = fix(fixedId(b, f));
		return Tf + ((size_t)fr[9] + faceCell(b, f, p)) * TS;
	}
	// velocity component w of the fixed boundary at the face cell of p (block_data.cuh:137-205)
	S fixedVel(int b, int f, const int *p, int w) const {
		const int32_t *fr = fix(fixedId(b, f));
		if (fr[2]) return fvel[fr[7] + w];
		return fvel[fr[7] + w * fr[8] + faceCell(b, f, p)];
	}
	int velType(int b, int f) const { return fix(fixedId(b, f))[3]; }
	int potBC(int b, int f, const int *p) const { // topology.cuh:46-54
		const int32_t *fr = fix(fixedId(b, f));
		if (fr[5] < 0) return fr[4];
		return fmask[fr[5] + faceCell(b, f, p)];
	}
	S potValue(int b, int f, const int *p) const { // topology.cuh:59-66
		const int32_t *fr = fix(fixedId(b, f));
		if (fr[6] < 0) return S(0);
		return fpot[fr[6] + faceCell(b, f, p)];
	}
	S potCw(int b, int f) const { return fcw[fixedId(b, f)]; }
	bool isEmpty(int b, int f) const { return ftype(b, f) == FT_FIXED; }
	bool atBound(int b, int f, const int *p) const {
		const int ax = f >> 1;
		return (f & 1) ? p[ax] == sz(b, ax) - 1 : p[ax] == 0;
	}
};

static inline int posMod(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

// topology.cuh:168-189 computeConnectedPos
template <typename S>
static void connectedPos(const Dom<S> &D, int b, int f, const int *pos, int borderOffset, int &ob, int *op) {
	const int32_t *fc = D.face(b, f);
	const int boundaryDim = f >> 1;
	ob = fc[1];
	const int *axes = fc + 2;
	op[0] = pos[0]; op[1] = pos[1]; op[2] = pos[2];
	int cAxis = axes[0] >> 1;
	op[cAxis] = (axes[0] & 1) ? D.sz(ob, cAxis) - 1 - borderOffset : borderOffset;
	if (D.dims > 1) {
		int axis = (boundaryDim + 1) % D.dims;
		cAxis = axes[1] >> 1;
		op[cAxis] = (axes[1] & 1) ? D.sz(ob, cAxis) - 1 - pos[axis] : pos[axis];
		if (D.dims > 2) {
			axis = (boundaryDim + 2) % D.dims;
			cAxis = axes[2] >> 1;
			op[cAxis] = (axes[2] & 1) ? D.sz(ob, cAxis) - 1 - pos[axis] : pos[axis];
		}
	}
}
// topology.cuh:193-203: component of the connected block that component w maps to
template <typename S>
static int connectedChannel(const Dom<S> &D, int b, int f, int w) {
	const int32_t *fc = D.face(b, f);
	const int idx = posMod(w - (f >> 1), D.dims);
	return fc[2 + idx] >> 1;
}
template <typename S>
static bool connectedSameSide(const Dom<S> &D, int b, int f) {
	const int32_t *fc = D.face(b, f);
	return ((fc[2] & 1) != 0) == ((f & 1) != 0);
}

// Neighbor across face f for a non-prescribed face: (block, pos, component mapping of w)
template <typename S>
static void neighbor(const Dom<S> &D, int b, int f, const int *pos, int &nbk, int *np) {
	const int ax = f >> 1;
	if (D.atBound(b, f, pos)) {
		if (D.ftype(b, f) == FT_CONNECTED) { connectedPos(D, b, f, pos, 0, nbk, np); return; }
		// periodic
		nbk = b; np[0] = pos[0]; np[1] = pos[1]; np[2] = pos[2];
		np[ax] = (f & 1) ? 0 : D.sz(b, ax) - 1;
		return;
	}
	nbk = b; np[0] = pos[0]; np[1] = pos[1]; np[2] = pos[2];
	np[ax] += (f & 1) ? 1 : -1;
}

template <typename S>
static inline S dotv(const S *a, const S *v, int d) {
	S r = 0;
	for (int i = 0; i < d; ++i) r += a[i] * v[i];
	return r;
}
// discretization.cuh:360-375 getLaplaceCoefficientOrthogonal: det*|Minv[c]|^2
template <typename S>
static inline S alphaOf(const Dom<S> &D, const S *t, int c) {
	const S *m = D.Minv(t, c);
	return D.det(t) * dotv(m, m, D.dims);
}
// velocity.cuh:188-199 getContravariantComponent on a flat [comp][ncells] field
template <typename S>
static inline S contra(const Dom<S> &D, int b, const int *p, int c, const S *field) {
	const int g = D.glob(b, p);
	S v[3];
	for (int k = 0; k < D.dims; ++k) v[k] = field[(size_t)k * D.n + g];
	const S *t = D.T(b, p);
	return D.det(t) * dotv(D.Minv(t, c), v, D.dims);
}
// velocity.cuh:216-237 getContravariantComponentBoundaryFixed (with boundary transform)
template <typename S>
static inline S contraFixed(const Dom<S> &D, int b, int f, const int *p, int c) {
	S v[3] = {0, 0, 0};
	if (D.velType(b, f) == 0)
		for (int k = 0; k < D.dims; ++k) v[k] = D.fixedVel(b, f, p, k);
	const S *t = D.faceT(b, f, p);
	return D.det(t) * dotv(D.Minv(t, c), v, D.dims);
}

// discretization.cuh:758-838 computeFluxesNDLoop (fluxes NOT multiplied by the face sign)
template <typename S>
static void fluxes(const Dom<S> &D, int b, const int *p, const S *field, S *fl) {
	for (int f = 0; f < 2 * D.dims; ++f) {
		const int dim = f >> 1;
		const S velC = contra(D, b, p, dim, field);
		if (D.atBound(b, f, p)) {
			const int t = D.ftype(b, f);
			if (t == FT_FIXED) {
				fl[f] = contraFixed(D, b, f, p, dim);
			} else if (t == FT_CONNECTED) {
				int ob, op[3];
				connectedPos(D, b, f, p, 0, ob, op);
				const int oc = D.face(b, f)[2] >> 1;
				S velN = contra(D, ob, op, oc, field);
				if (connectedSameSide(D, b, f)) velN = -velN;
				fl[f] = (velN + velC) * S(0.5);
			} else {
				int q[3] = {p[0], p[1], p[2]};
				q[dim] = (f & 1) ? 0 : D.sz(b, dim) - 1;
				fl[f] = (contra(D, b, q, dim, field) + velC) * S(0.5);
			}
		} else {
			int q[3] = {p[0], p[1], p[2]};
			q[dim] += (f & 1) ? 1 : -1;
			fl[f] = (contra(D, b, q, dim, field) + velC) * S(0.5);
		}
	}
}

// Row assembly helper: entries [diag, -x, +x, -y, +y, -z, +z], written sorted by column
// as PISO_build_matrix does (advection.cu:269-288, csr_rows.cuh:24-35). div: divide every
// value by it (advection rows) or 1.
template <typename S>
static void writeRow(int *idx, S *val, int rowStart, int rowSize, const int *cols, S *vals, S div, int *colOut, S *valOut) {
	int ind[7];
	for (int i = 0; i < 7; ++i) ind[i] = cols[i];
	for (int i = 0; i < rowSize; ++i) {
		int best = -1, bv = std::numeric_limits<int>::max();
		for (int j = 0; j < 7; ++j) if (ind[j] >= 0 && ind[j] < bv) { bv = ind[j]; best = j; }
		vals[best] /= div;
		colOut[rowStart + i] = ind[best];
		valOut[rowStart + i] = vals[best];
		ind[best] = -1;
	}
	(void)idx; (void)val;
}

// CSR row pointers of the shared pattern: 2d+1 entries minus prescribed faces (block.cpp:1145-1155)
template <typename S>
static void rowPointers(const Dom<S> &D, int *row) {
	row[0] = 0;
	for (int b = 0; b < D.nb; ++b) {
		const int nc = D.ncellsBlock(b);
		for (int l = 0; l < nc; ++l) {
			int p[3]; D.unflat(b, l, p);
			int rs = 2 * D.dims + 1;
			for (int f = 0; f < 2 * D.dims; ++f) if (D.atBound(b, f, p) && D.isEmpty(b, f)) --rs;
			row[D.off(b) + l + 1] = rs;
		}
	}
	for (int i = 0; i < D.n; ++i) row[i + 1] += row[i];
}

template <typename S>
static void forEachCell(const Dom<S> &D, const std::function<void(int, const int *, int)> &fn) {
	for (int b = 0; b < D.nb; ++b) {
		const int nc = D.ncellsBlock(b);
		#pragma omp parallel for schedule(static)
		for (int l = 0; l < nc; ++l) {
			int p[3]; D.unflat(b, l, p);
			fn(b, p, D.off(b) + l);
		}
	}
}

// shared_stencils.cuh:35-43 hasFarUpwindCell: downwind and far-upwind cells inside the block
template <typename S>
static bool farUpwind(const Dom<S> &D, int b, const int *p, int f, bool outflow) {
	const int ax = f >> 1, sign = (f & 1) ? 1 : -1, last = D.sz(b, ax) - 1;
	const int iD = p[ax] + sign;
	if (iD < 0 || iD > last) return false;
	const int iUU = outflow ? p[ax] - sign : p[ax] + 2 * sign;
	return iUU >= 0 && iUU <= last;
}
// advection.cu:892-934 (velocity) and :652-688 (scalar): LINEAR_UPWIND deferred correction,
// r -= F 0.5 psi (phi_D - phi_U) per upwinded face, psi = (phi_U - phi_UU)/(phi_D - phi_U);
// field(g) is the lagged block field at global cell g
template <typename S, typename F>
static void upwindCorrection(const Dom<S> &D, int b, const int *p, const S *fl, F field, S &r) {
	for (int f = 0; f < 2 * D.dims; ++f) {
		const int ax = f >> 1, sign = (f & 1) ? 1 : -1;
		const S fout = S(sign) * fl[f];
		const bool outflow = fout >= S(0);
		if (!farUpwind(D, b, p, f, outflow)) continue;
		int q[3] = {p[0], p[1], p[2]};
		const S phiP = field(D.glob(b, q));
		q[ax] = p[ax] + sign;
		const S phiN = field(D.glob(b, q));
		q[ax] = outflow ? p[ax] - sign : p[ax] + 2 * sign;
		const S phiUU = field(D.glob(b, q));
		const S phiU = outflow ? phiP : phiN, phiD = outflow ? phiN : phiP;
		const S dD = phiD - phiU;
		if ((dD < 0 ? -dD : dD) < S(1e-20)) continue;
		const S psi = (phiU - phiUU) / dD;
		r -= fout * S(0.5) * psi * dD;
	}
}

// ---------------------------------------------------------------------------------------
// Non-orthogonal Laplace terms (piso/device/nonortho_laplace.cuh, nonortho_rhs.cuh,
// block_data.cuh:477-620). Flag bits as piso/non_ortho_flags.h:23-27.
enum { NO_DIRECT_MATRIX = 1, NO_DIRECT_RHS = 2, NO_DIAGONAL_MATRIX = 4, NO_DIAGONAL_RHS = 8, NO_CENTER_MATRIX = 16 };
// the field a corner walk or neighbour read looks at (GridDataType of block_data.cuh)
enum { NF_MARK = 0, NF_PRESSURE = 1, NF_VELOCITY = 2, NF_SCALAR = 3 };

template <typename S>
struct NField {
	int kind = NF_MARK;
	int w = 0;                 // velocity component (scalar channel: the arrays below are the channel's)
	const S *cells = nullptr;  // [n] cell values of component w
	const int8_t *sTypes = nullptr;
	const S *sValues = nullptr;
	const int64_t *sOffsets = nullptr;
	const int8_t *sStatic = nullptr;
};
template <typename S>
static S nfCell(const Dom<S> &D, const NField<S> &F, int b, const int *p) {
	return F.cells ? F.cells[D.glob(b, p)] : S(0);
}
// getFixedBoundaryType (block_data.cuh:111-135): 1 for a Neumann face
template <typename S>
static int nfNeumann(const Dom<S> &D, const NField<S> &F, int b, int f) {
	if (F.kind == NF_VELOCITY) return D.velType(b, f) != 0;
	if (F.kind == NF_SCALAR) return F.sTypes[D.fixedId(b, f)] != 0;
	return 0;
}
// getFixedBoundaryData (block_data.cuh:137-205); the fixed faces carry no pressure data
template <typename S>
static S nfFixed(const Dom<S> &D, const NField<S> &F, int b, int f, const int *p) {
	if (F.kind == NF_MARK) return S(1);
	if (F.kind == NF_VELOCITY) return D.fixedVel(b, f, p, F.w);
	if (F.kind == NF_SCALAR) {
		if (!F.sValues) return S(0); // a matrix walk reads only the face types
		const int fid = D.fixedId(b, f);
		return F.sStatic[fid] ? F.sValues[F.sOffsets[fid]] : F.sValues[F.sOffsets[fid] + D.faceCell(b, f, p)];
	}
	return S(0);
}
// computeConnectedDir (topology.cuh:226-236): direction dir of block b seen from the block
// across its connected face f
template <typename S>
static int connDir(const Dom<S> &D, int b, int f, int dir) {
	const int32_t *axes = D.face(b, f) + 2;
	return axes[posMod((dir >> 1) - (f >> 1), D.dims)] ^ (dir & 1);
}
// one step of a walk from (b, p) across direction dir through periodic or connected faces;
// false at a fixed face. Connected faces land one cell inside the other block
// (computeConnectedPos with borderOffset 1, as block_data.cuh:299,397,571 call it).
template <typename S>
static bool stepAcross(const Dom<S> &D, int &b, int *p, int dir) {
	const int ax = dir >> 1;
	if (!D.atBound(b, dir, p)) { p[ax] += (dir & 1) ? 1 : -1; return true; }
	const int t = D.ftype(b, dir);
	if (t == FT_FIXED) return false;
	if (t == FT_PERIODIC) { p[ax] = (dir & 1) ? 0 : D.sz(b, ax) - 1; return true; }
	int ob, op[3];
	connectedPos(D, b, dir, p, 1, ob, op);
	b = ob; p[0] = op[0]; p[1] = op[1]; p[2] = op[2];
	return true;
}
// getBlockDataNeighbor (block_data.cuh:276-318)
template <typename S>
static S neighborData(const Dom<S> &D, const NField<S> &F, int b, const int *pos, int dir) {
	int p[3] = {pos[0], pos[1], pos[2]};
	if (!stepAcross(D, b, p, dir)) return nfFixed(D, F, b, dir, p);
	return nfCell(D, F, b, p);
}
// getBlockDataNeighborDiagonal (block_data.cuh:372-420): dir1 first unless the block's dir1
// face is fixed; the second step keeps its direction index in the block reached
template <typename S>
static S diagonalData(const Dom<S> &D, const NField<S> &F, int b, const int *pos, int dir1, int dir2) {
	const bool first1 = !D.isEmpty(b, dir1);
	const int dirs[2] = {first1 ? dir1 : dir2, first1 ? dir2 : dir1};
	int p[3] = {pos[0], pos[1], pos[2]};
	for (int i = 0; i < 2; ++i)
		if (!stepAcross(D, b, p, dirs[i])) return nfFixed(D, F, b, dirs[i], p);
	return nfCell(D, F, b, p);
}

template <typename S>
struct CornerValue {
	S data;
	int numCells; // 0: the value came from a fixed face
	int neumann;  // the fixed face's type when numCells is 0
};
// getCornerValue (block_data.cuh:501-620) with includeDepth0 false and maxDepth 2: walk around
// the corner between directions dir1 and dir2 both ways until the walks meet or a fixed face
// ends one of them.
template <typename S>
static CornerValue<S> cornerWalk(const Dom<S> &D, const NField<S> &F, int b0, const int *pos, int dir1, int dir2, bool depth1) {
	struct Walk { int d1, d2, b, p[3]; };
	Walk w[2] = {{dir1, dir2, b0, {pos[0], pos[1], pos[2]}}, {dir2, dir1, b0, {pos[0], pos[1], pos[2]}}};
	S data = 0;
	int num = 1;
	for (int depth = 1; depth <= 2; ++depth) {
		for (int d = 0; d < 2; ++d) {
			Walk &c = w[d];
			const int ax = c.d1 >> 1;
			if (D.atBound(c.b, c.d1, c.p)) {
				const int t = D.ftype(c.b, c.d1);
				if (t == FT_FIXED) {
					const int neu = nfNeumann(D, F, c.b, c.d1);
					const S v0 = nfFixed(D, F, c.b, c.d1, c.p);
					if (D.atBound(c.b, c.d2, c.p)) return {v0, 0, neu};
					int q[3] = {c.p[0], c.p[1], c.p[2]};
					q[c.d2 >> 1] += (c.d2 & 1) ? 1 : -1;
					return {(v0 + nfFixed(D, F, c.b, c.d1, q)) * S(0.5), 0, neu};
				}
				if (t == FT_CONNECTED) {
					const int nd1 = connDir(D, c.b, c.d1, c.d2);
					const int nd2 = connDir(D, c.b, c.d1, c.d1) ^ 1;
					int ob, op[3];
					connectedPos(D, c.b, c.d1, c.p, 1, ob, op);
					c.b = ob; c.p[0] = op[0]; c.p[1] = op[1]; c.p[2] = op[2];
					c.d1 = nd1; c.d2 = nd2;
				} else { // periodic
					c.p[ax] = (c.d1 & 1) ? 0 : D.sz(c.b, ax) - 1;
					const int od1 = c.d1;
					c.d1 = c.d2; c.d2 = od1 ^ 1;
				}
			} else {
				c.p[ax] += (c.d1 & 1) ? 1 : -1;
				const int od1 = c.d1;
				c.d1 = c.d2; c.d2 = od1 ^ 1;
			}
			const Walk &o = w[d ^ 1];
			if (c.b == o.b && c.p[0] == o.p[0] && c.p[1] == o.p[1] && c.p[2] == o.p[2])
				return {data / S(num), num, 0};
			if (depth > 1 || depth1) data += nfCell(D, F, c.b, c.p);
			++num;
		}
	}
	return {data / S(num), num, 0};
}

// det Minv[a] . Minv[c] of transform t (discretization.cuh:419-446, 447-469)
template <typename S>
static inline S lapCross(const Dom<S> &D, const S *t, int a, int c) {
	return D.det(t) * dotv(D.Minv(t, a), D.Minv(t, c), D.dims);
}

// interpolateNonOrthoLaplaceComponents (nonortho_laplace.cuh:52-129) without face transforms:
// out[f][i-1] is the cross coefficient of face f with the tangential axis (f/2 + i) % d,
// interpolated between the cell and its neighbour with weights ra (1/A, viscosity or 1).
// A face gets one when its cell is not at either end of the face's axis or the block's face
// in that direction is not fixed, as the reference tests it.
template <typename S, typename RA>
static void nonOrthoInterp(const Dom<S> &D, int b, const int *p, RA ra, S out[6][2]) {
	const S *tP = D.T(b, p);
	const S raP = ra(b, p);
	for (int f = 0; f < 2 * D.dims; ++f) {
		const int ax = f >> 1;
		for (int i = 0; i < 2; ++i) out[f][i] = 0;
		if (!((0 < p[ax] && p[ax] < D.sz(b, ax) - 1) || !D.isEmpty(b, f))) continue;
		int nb = b, np[3] = {p[0], p[1], p[2]};
		if (D.atBound(b, f, p) && D.ftype(b, f) == FT_CONNECTED) {
			connectedPos(D, b, f, p, 0, nb, np);
		} else if (D.atBound(b, f, p) && D.ftype(b, f) == FT_PERIODIC) {
			np[ax] = (f & 1) ? 0 : D.sz(b, ax) - 1;
		} else {
			np[ax] += (f & 1) ? 1 : -1;
		}
		const S *tN = D.T(nb, np);
		const S raN = ra(nb, np);
		for (int i = 1; i < D.dims; ++i) {
			const int o = (ax + i) % D.dims;
			out[f][i - 1] = (lapCross(D, tP, ax, o) * raP + lapCross(D, tN, o, ax) * raN) * S(0.5);
		}
	}
}

// The non-orthogonal matrix terms of free face f of one row (pressure.cu:103-156 for the
// pressure matrix, advection.cu:176-240 for the advection matrix), added right after the
// face's orthogonal terms as the reference does: for each tangential axis, the corner values
// either side are interpolations of numCells cells (their centre and direct-neighbour parts go
// to the row when CENTER_MATRIX / DIRECT_MATRIX are set) or, at a fixed gradient face, a
// one-sided difference from the other side. sgn = +1 adds them as the pressure matrix does,
// -1 as the advection matrix does; a[i-1] is the face's cross coefficient with tangential
// axis (f/2 + i) % d.
template <typename S>
static void nonOrthoMatrixFace(const Dom<S> &D, const NField<S> &F, int b, const int *p, int f, int flags, int sgn,
		bool pressure, const S *a, S *rv) {
	const bool center = flags & NO_CENTER_MATRIX, direct = flags & NO_DIRECT_MATRIX;
	if (D.dims < 2 || !(center || direct)) return;
	const int faceSign = (f & 1) ? 1 : -1;
	for (int i = 1; i < D.dims; ++i) {
		const int tAxis = ((f >> 1) + i) % D.dims;
		if (a[i - 1] == S(0)) continue;
		for (int tUp = 0; tUp < 2; ++tUp) {
			const int tFace = 2 * tAxis + tUp;
			const int tSign = tUp ? 1 : -1;
			const CornerValue<S> cv = cornerWalk(D, F, b, p, f, tFace, false);
			if (cv.numCells < 1) {
				if (!(pressure || cv.neumann)) continue; // a prescribed value goes to the right-hand side
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

// getNonOrthoLaplaceRHS_v2 (nonortho_rhs.cuh:27-180) without face transforms: the explicit
// part of the cross terms at cell (b, p) for field F; ra(b, p) the weight (1/A for the
// pressure, the viscosity for the velocity, 1 for the scalar), raFixed the weight at a fixed
// face (viscosity or 1).
template <typename S, typename RA>
static S nonOrthoRhs(const Dom<S> &D, const NField<S> &F, int b, const int *p, int flags, RA ra, S raFixed) {
	if (!(flags & (NO_DIRECT_RHS | NO_DIAGONAL_RHS)) || D.dims < 2) return S(0);
	const bool direct = flags & NO_DIRECT_RHS, diagonal = flags & NO_DIAGONAL_RHS;
	const S *tP = D.T(b, p);
	const S raP = ra(b, p);
	S Ssum = 0;
	for (int f = 0; f < 2 * D.dims; ++f) {
		const int ax = f >> 1;
		const int faceSign = (f & 1) ? 1 : -1;
		if (D.atBound(b, f, p) && D.isEmpty(b, f)) {
			if (F.kind == NF_PRESSURE || nfNeumann(D, F, b, f)) continue;
			const S *tf = D.faceT(b, f, p);
			for (int i = 1; i < D.dims; ++i) {
				const int tAxis = (ax + i) % D.dims;
				const bool tLow = p[tAxis] == 0, tHigh = p[tAxis] == D.sz(b, tAxis) - 1;
				int lo[3] = {p[0], p[1], p[2]}, hi[3] = {p[0], p[1], p[2]};
				if (!tLow) lo[tAxis] -= 1;
				if (!tHigh) hi[tAxis] += 1;
				const S factor = (tLow || tHigh) ? S(1) : S(0.5);
				const S tGrad = factor * (nfFixed(D, F, b, f, hi) - nfFixed(D, F, b, f, lo));
				Ssum -= S(faceSign) * lapCross(D, tf, tAxis, ax) * tGrad * raFixed;
			}
			continue;
		}
		// resolveNeighborCell (topology.cuh:343-383): the direct neighbour with the axis mapping
		// of a connection (getLaplaceCoefficientsSingleAxisNeighbor, discretization.cuh:565-600)
		int nb = b, np[3] = {p[0], p[1], p[2]};
		int map[3] = {0, 1, 2};
		if (D.atBound(b, f, p) && D.ftype(b, f) == FT_CONNECTED) {
			connectedPos(D, b, f, p, 0, nb, np);
			for (int k = 0; k < D.dims; ++k) map[k] = connDir(D, b, f, 2 * k) >> 1;
		} else if (D.atBound(b, f, p)) {
			np[ax] = (f & 1) ? 0 : D.sz(b, ax) - 1;
		} else {
			np[ax] += (f & 1) ? 1 : -1;
		}
		const S *tN = D.T(nb, np);
		const S raN = ra(nb, np);
		for (int i = 1; i < D.dims; ++i) {
			const int tAxis = (ax + i) % D.dims;
			const S faceAlpha = (lapCross(D, tP, ax, tAxis) * raP + lapCross(D, tN, map[tAxis], map[ax]) * raN) * S(0.5);
			S tGrad = 0;
			for (int tUp = 0; tUp < 2; ++tUp) {
				const int tFace = 2 * tAxis + tUp;
				const int tSign = tUp ? 1 : -1;
				const CornerValue<S> cv = cornerWalk(D, F, b, p, f, tFace, direct);
				if (cv.numCells == 0 && (cv.neumann || F.kind == NF_PRESSURE)) {
					const int tOther = tFace ^ 1;
					if (direct) {
						tGrad += S(tSign) * neighborData(D, F, b, p, f) * S(0.75);
						tGrad += S(-tSign) * neighborData(D, F, b, p, tOther) * S(0.25);
					}
					if (diagonal) tGrad += S(-tSign) * diagonalData(D, F, b, p, f, tOther) * S(0.25);
				} else {
					tGrad += S(tSign) * cv.data;
				}
			}
			Ssum -= S(faceSign) * faceAlpha * tGrad;
		}
	}
	return Ssum;
}

// advection.cu:27-305 PISO_build_matrix (domain viscosity; non-orthogonal terms by flags). With
// faceTypes (forPassiveScalar): the wall diffusion of a fixed face follows the scalar
// channel's type faceTypes[fixed id] instead of the velocity type (advection.cu:254-266), and
// nu is the channel's diffusivity.
template <typename S>
static void advMatrix(const Dom<S> &D, const S *u, S dt, S nu, const int *row, int *col, S *val, S *Adiag,
		const int8_t *faceTypes = nullptr, int scheme = 0, int flags = 0) {
	NField<S> F;
	F.kind = faceTypes ? NF_SCALAR : NF_VELOCITY;
	F.sTypes = faceTypes;
	const bool nonOrtho = D.dims > 1 && (flags & (NO_CENTER_MATRIX | NO_DIRECT_MATRIX));
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		// the velocity matrix weights the cross coefficients with the viscosity, the scalar
		// matrix scales them by its diffusivity afterwards (advection.cu:181-195)
		S ia[6][2] = {};
		if (nonOrtho) nonOrthoInterp(D, b, p, [&](int, const int *) { return faceTypes ? S(1) : nu; }, ia);
		S fl[6];
		fluxes(D, b, p, u, fl);
		const S *tP = D.T(b, p);
		const S det = D.det(tP);
		S diag = det / dt;
		S alphaP[3] = {1, 1, 1};
		for (int d = 0; d < D.dims; ++d) alphaP[d] = alphaOf(D, tP, d);
		int cols[7] = {g, -1, -1, -1, -1, -1, -1};
		S rv[7] = {0, 0, 0, 0, 0, 0, 0};
		for (int f = 0; f < 2 * D.dims; ++f) {
			const int dim = f >> 1;
			const S faceSign = (f & 1) ? S(1) : S(-1);
			const bool ab = D.atBound(b, f, p);
			if (!ab || !D.isEmpty(b, f)) {
				const S fout = faceSign * fl[f];
				if (scheme != 0 && farUpwind(D, b, p, f, fout >= S(0))) { // advection.cu:131-139
					if (fout >= S(0)) diag += fout;
					else rv[f + 1] += fout;
				} else {
					const S half = S(0.5) * fout;
					diag += half;
					rv[f + 1] += half;
				}
				int nbk, np[3];
				neighbor(D, b, f, p, nbk, np);
				int comp = dim;
				if (ab && D.ftype(b, f) == FT_CONNECTED) comp = connectedChannel(D, b, f, dim);
				const S alphaN = alphaOf(D, D.T(nbk, np), comp);
				cols[f + 1] = D.glob(nbk, np);
				const S coeff = (alphaP[dim] * nu + alphaN * nu) * S(0.5);
				diag += coeff;
				rv[f + 1] -= coeff;
				if (nonOrtho) {
					const S a[2] = {ia[f][0] * (faceTypes ? nu : S(1)), ia[f][1] * (faceTypes ? nu : S(1))};
					rv[0] = diag;
					nonOrthoMatrixFace(D, F, b, p, f, flags, -1, false, a, rv);
					diag = rv[0];
				}
			} else {
				const int type = faceTypes ? int(faceTypes[D.fixedId(b, f)]) : D.velType(b, f);
				const S slip = type == 0 ? S(0) : S(1);
				diag += (S(1) - slip) * S(2) * nu * alphaP[dim];
			}
		}
		rv[0] = diag;
		writeRow<S>(nullptr, nullptr, row[g], row[g + 1] - row[g], cols, rv, det, col, val);
		Adiag[g] = rv[0];
	});
}

// advection.cu:800-954 kPISO_build_advection_RHS (no pressure gradient); with ures the
// non-orthogonal terms of the velocity result
template <typename S>
static void advRhs(const Dom<S> &D, const S *u, const S *src, int srcStatic, S dt, S nu, S *rhs, int scheme = 0,
		int flags = 0, const S *ures = nullptr) {
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		const S det = D.det(D.T(b, p));
		S fl[6];
		if (scheme != 0) fluxes(D, b, p, u, fl);
		for (int dim = 0; dim < D.dims; ++dim) {
			S r = det * u[(size_t)dim * D.n + g] / dt;
			for (int f = 0; f < 2 * D.dims; ++f) {
				if (!D.atBound(b, f, p) || D.ftype(b, f) != FT_FIXED) continue;
				const S faceNormal = (f & 1) ? S(1) : S(-1);
				const S vel = D.fixedVel(b, f, p, dim);
				const S *tf = D.faceT(b, f, p);
				const S alpha = alphaOf(D, tf, f >> 1);
				const S flux = contraFixed(D, b, f, p, f >> 1) * faceNormal;
				r -= vel * flux;
				const S slip = D.velType(b, f) == 0 ? S(0) : S(1);
				r += vel * (S(1) - slip) * nu * S(2) * alpha;
			}
			if (scheme != 0) upwindCorrection(D, b, p, fl, [&](int gg) { return u[(size_t)dim * D.n + gg]; }, r);
			if (ures) { // advection.cu:936-937: the velocity result's cross terms, viscosity-weighted
				NField<S> F;
				F.kind = NF_VELOCITY;
				F.w = dim;
				F.cells = ures + (size_t)dim * D.n;
				r -= nonOrthoRhs(D, F, b, p, flags, [&](int, const int *) { return nu; }, nu);
			}
			r /= det;
			if (src) r += srcStatic ? src[dim] : src[(size_t)dim * D.n + g];
			rhs[(size_t)dim * D.n + g] = r;
		}
	});
}

// advection.cu:545-698 kPISO_build_scalar_advection_RHS for one channel:
// det phi/dt, at fixed faces Dirichlet -phi_b F + phi_b nu 2 alpha, Neumann -phi_P F +
// (dphi/dn) nu |S_f| (|S_f| = det_f |Minv_f[dim]|, discretization.cuh:618-634), over det.
// faceTypes[fixed id]: 0 Dirichlet, 1 Neumann; faceValue(fixed id, face cell) the face data.
template <typename S>
static void scalarRhs(const Dom<S> &D, const S *phi, S dt, S nu, const int8_t *faceTypes, const S *faceValues,
		const int64_t *faceOffsets, const int8_t *faceStatic, S *rhs, const S *u = nullptr, int scheme = 0, int flags = 0,
		const S *phires = nullptr) {
	NField<S> F;
	F.kind = NF_SCALAR;
	F.cells = phires;
	F.sTypes = faceTypes;
	F.sValues = faceValues;
	F.sOffsets = faceOffsets;
	F.sStatic = faceStatic;
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		const S det = D.det(D.T(b, p));
		S fl[6];
		if (scheme != 0) fluxes(D, b, p, u, fl);
		S r = det * phi[g] / dt;
		for (int f = 0; f < 2 * D.dims; ++f) {
			if (!D.atBound(b, f, p) || D.ftype(b, f) != FT_FIXED) continue;
			const S faceNormal = (f & 1) ? S(1) : S(-1);
			const int fid = D.fixedId(b, f);
			const S value = faceStatic[fid] ? faceValues[faceOffsets[fid]] : faceValues[faceOffsets[fid] + D.faceCell(b, f, p)];
			const S *tf = D.faceT(b, f, p);
			const S flux = contraFixed(D, b, f, p, f >> 1) * faceNormal;
			if (faceTypes[fid] == 0) {
				r -= value * flux;
				r += value * nu * S(2) * alphaOf(D, tf, f >> 1);
			} else {
				const S *mi = D.Minv(tf, f >> 1);
				const S area = D.det(tf) * std::sqrt(dotv(mi, mi, D.dims));
				r -= phi[g] * flux;
				r += value * nu * area;
			}
		}
		if (scheme != 0) upwindCorrection(D, b, p, fl, [&](int gg) { return phi[gg]; }, r);
		// advection.cu:684-689: the scalar result's cross terms, times the diffusivity
		if (phires) r -= nonOrthoRhs(D, F, b, p, flags, [&](int, const int *) { return S(1); }, S(1)) * nu;
		rhs[g] = r / det;
	});
}

// pressure.cu:26-191 PISO_build_pressure_matrix (orthogonal, no face transforms).
// With unitWeight it is PISO_build_epot_matrix (potential.cu:30-233): 1/A replaced by 1,
// Dirichlet ghost diagonal and the thin-wall Robin terms.
template <typename S>
static void laplaceMatrix(const Dom<S> &D, const S *Adiag, bool epot, const int *row, int *col, S *val, int flags = 0) {
	const NField<S> F; // the matrix walks only look for fixed faces (GridDataType::IS_FIXED_BOUNDARY)
	const bool nonOrtho = !epot && D.dims > 1 && (flags & (NO_CENTER_MATRIX | NO_DIRECT_MATRIX));
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		S ia[6][2] = {};
		if (nonOrtho) nonOrthoInterp(D, b, p, [&](int bb, const int *pp) { return S(1) / Adiag[D.glob(bb, pp)]; }, ia);
		const S *tP = D.T(b, p);
		S alphaP[3];
		for (int d = 0; d < D.dims; ++d) alphaP[d] = alphaOf(D, tP, d);
		const S raP = epot ? S(1) : S(1) / Adiag[g];
		int cols[7] = {g, -1, -1, -1, -1, -1, -1};
		S rv[7] = {0, 0, 0, 0, 0, 0, 0};
		for (int f = 0; f < 2 * D.dims; ++f) {
			const int dim = f >> 1;
			const bool ab = D.atBound(b, f, p);
			if (!(ab && D.isEmpty(b, f))) {
				int nbk, np[3];
				neighbor(D, b, f, p, nbk, np);
				int comp = dim;
				if (ab && D.ftype(b, f) == FT_CONNECTED) comp = connectedChannel(D, b, f, dim);
				const S alphaN = alphaOf(D, D.T(nbk, np), comp);
				const int gn = D.glob(nbk, np);
				const S raN = epot ? S(1) : S(1) / Adiag[gn];
				const S coeff = S(0.5) * (alphaP[dim] * raP + alphaN * raN);
				rv[0] -= coeff;
				rv[f + 1] += coeff;
				cols[f + 1] = gn;
				if (nonOrtho) nonOrthoMatrixFace(D, F, b, p, f, flags, 1, true, ia[f], rv);
			} else if (epot && D.potBC(b, f, p) == PB_DIRICHLET) {
				rv[0] -= alphaP[dim] * raP;
			}
		}
		if (epot) { // potential.cu:175-219 thin-wall Robin correction
			for (int tw = 0; tw < 2 * D.dims; ++tw) {
				const int twDim = tw >> 1;
				if (!D.atBound(b, tw, p) || D.ftype(b, tw) != FT_FIXED || D.potBC(b, tw, p) != PB_THIN_WALL) continue;
				const S Cw = D.potCw(b, tw);
				const S *mP = D.Minv(tP, twDim);
				const S MinvNP = std::sqrt(dotv(mP, mP, D.dims));
				for (int tDim = 0; tDim < D.dims; ++tDim) {
					if (tDim == twDim) continue;
					for (int side = 0; side < 2; ++side) {
						const int tb = tDim * 2 + side;
						if (cols[tb + 1] < 0) continue;
						int q[3] = {p[0], p[1], p[2]};
						if (D.atBound(b, tb, p)) {
							if (D.ftype(b, tb) == FT_PERIODIC) q[tDim] = side ? 0 : D.sz(b, tDim) - 1;
							else continue;
						} else {
							q[tDim] += side ? 1 : -1;
						}
						if (D.potBC(b, tw, q) != PB_THIN_WALL) continue;
						const S *tN = D.T(b, q);
						const S alphaNt = alphaOf(D, tN, tDim);
						const S *mN = D.Minv(tN, twDim);
						const S MinvNN = std::sqrt(dotv(mN, mN, D.dims));
						const S surf = Cw * S(0.5) * (alphaP[tDim] * MinvNP + alphaNt * MinvNN);
						rv[0] -= surf;
						rv[tb + 1] += surf;
					}
				}
			}
		}
		writeRow<S>(nullptr, nullptr, row[g], row[g + 1] - row[g], cols, rv, S(1), col, val);
	});
}

// pressure.cu:350-521 PISO_build_pressure_rhs (CENTRAL): HbyA per velocity component
template <typename S>
static void pressureRhs(const Dom<S> &D, const int *row, const int *col, const S *Cval, const S *Adiag,
		const S *u, const S *ustar, const S *src, int srcStatic, S dt, S nu, S *hbya, int scheme = 0) {
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		const S rDiag = S(1) / Adiag[g];
		const S det = D.det(D.T(b, p));
		S fl[6];
		if (scheme != 0) fluxes(D, b, p, u, fl);
		const int rs = row[g], re = row[g + 1];
		for (int dim = 0; dim < D.dims; ++dim) {
			const S velOld = u[(size_t)dim * D.n + g] / dt;
			S H = 0;
			for (int j = rs; j < re; ++j) {
				const int c = col[j];
				if (c != g) H += Cval[j] * ustar[(size_t)dim * D.n + c];
			}
			S Ssum = 0;
			for (int f = 0; f < 2 * D.dims; ++f) {
				if (!D.atBound(b, f, p) || D.ftype(b, f) != FT_FIXED) continue;
				const S faceNormal = (f & 1) ? S(1) : S(-1);
				const S vel = D.fixedVel(b, f, p, dim);
				const S alpha = alphaOf(D, D.faceT(b, f, p), f >> 1);
				const S flux = contraFixed(D, b, f, p, f >> 1) * faceNormal;
				Ssum -= vel * flux;
				const S slip = D.velType(b, f) == 0 ? S(0) : S(1);
				Ssum += vel * (S(1) - slip) * nu * S(2) * alpha;
			}
			Ssum /= det;
			if (src) Ssum += srcStatic ? src[dim] : src[(size_t)dim * D.n + g];
			if (scheme != 0) { // pressure.cu:474-515: the predictor's deferred correction, / det
				S corr = 0; // minus the face terms' sum, accumulated face by face
				upwindCorrection(D, b, p, fl, [&](int gg) { return u[(size_t)dim * D.n + gg]; }, corr);
				Ssum -= (-corr) / det;
			}
			hbya[(size_t)dim * D.n + g] = rDiag * (velOld - H + Ssum);
		}
	});
}

// pressure.cu:839-860 k_pressureRHSaddNonOrthoComponents: div += the pressure result's cross
// terms weighted with 1/A
template <typename S>
static void pressureNonOrtho(const Dom<S> &D, const S *Adiag, const S *pr, int flags, S *div) {
	NField<S> F;
	F.kind = NF_PRESSURE;
	F.cells = pr;
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		div[g] += nonOrthoRhs(D, F, b, p, flags, [&](int bb, const int *pp) { return S(1) / Adiag[D.glob(bb, pp)]; }, S(1));
	});
}

// pressure.cu:756-801 k_computePressureRHSdivergenceFromFlux (no face transforms)
template <typename S>
static void divergence(const Dom<S> &D, const S *field, S *div) {
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		S fl[6];
		fluxes(D, b, p, field, fl);
		S dv = 0;
		for (int d = 0; d < D.dims; ++d) dv += fl[d * 2 + 1] - fl[d * 2];
		div[g] = dv;
	});
}

// nonortho_laplace.cuh:302-381 getPressureAtWithBounds (one ghost layer)
template <typename S>
static S pressureAt(const Dom<S> &D, int b, const int *pos, const S *pr) {
	int t[3] = {pos[0], pos[1], pos[2]};
	for (int dim = 0; dim < D.dims; ++dim) {
		if (pos[dim] < 0) {
			const int f = dim * 2;
			const int ty = D.ftype(b, f);
			if (ty == FT_FIXED) { t[dim] = 0; return pr[D.glob(b, t)]; }
			if (ty == FT_CONNECTED) {
				int ob, op[3]; connectedPos(D, b, f, t, -(pos[dim] + 1), ob, op);
				return pr[D.glob(ob, op)];
			}
			t[dim] += D.sz(b, dim);
			return pr[D.glob(b, t)];
		}
		if (pos[dim] >= D.sz(b, dim)) {
			const int f = dim * 2 + 1;
			const int ty = D.ftype(b, f);
			if (ty == FT_FIXED) { t[dim] = D.sz(b, dim) - 1; return pr[D.glob(b, t)]; }
			if (ty == FT_CONNECTED) {
				int ob, op[3]; connectedPos(D, b, f, t, pos[dim] - D.sz(b, dim), ob, op);
				return pr[D.glob(ob, op)];
			}
			t[dim] -= D.sz(b, dim);
			return pr[D.glob(b, t)];
		}
	}
	return pr[D.glob(b, pos)];
}

// velocity.cuh:347-378 getPressureGradient: central differences, one-sided at prescribed
// faces, then times Minv from the left (g^T Minv)
template <typename S>
static void pressureGradient(const Dom<S> &D, int b, const int *p, const S *pr, S *grad) {
	S gr[3];
	for (int dim = 0; dim < D.dims; ++dim) {
		int t[3] = {p[0], p[1], p[2]};
		S fac = 0.5;
		if (!(p[dim] == 0 && D.isEmpty(b, dim * 2))) t[dim] = p[dim] - 1; else fac = 1;
		const S valN = pressureAt(D, b, t, pr);
		if (!(p[dim] == D.sz(b, dim) - 1 && D.isEmpty(b, dim * 2 + 1))) t[dim] = p[dim] + 1; else { t[dim] = p[dim]; fac = 1; }
		const S valP = pressureAt(D, b, t, pr);
		gr[dim] = (valP - valN) * fac;
	}
	const S *tP = D.T(b, p);
	for (int c = 0; c < D.dims; ++c) grad[c] = 0;
	for (int r = 0; r < D.dims; ++r)
		for (int c = 0; c < D.dims; ++c) grad[c] += D.Minv(tP, r)[c] * gr[r];
}

// velocity_correction.cu:27-60 PISO_update_velocity (version 1, no time step norm)
template <typename S>
static void correctVelocity(const Dom<S> &D, const S *pr, const S *hbya, const S *Adiag, S *uout) {
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		const S rDiag = S(1) / Adiag[g];
		S grad[3];
		pressureGradient(D, b, p, pr, grad);
		for (int d = 0; d < D.dims; ++d) {
			const size_t o = (size_t)d * D.n + g;
			uout[o] = -rDiag * grad[d] + hbya[o];
		}
	});
}

// potential.cu:273-323 k_computeEpotRHS with discretization.cuh:856-912 computeEpotFluxesNDLoop
template <typename S>
static void epotRhs(const Dom<S> &D, const S *field, S *div) {
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		S fl[6];
		for (int f = 0; f < 2 * D.dims; ++f) {
			const int dim = f >> 1;
			const S velC = contra(D, b, p, dim, field);
			if (D.atBound(b, f, p) && D.ftype(b, f) == FT_FIXED) {
				const int bc = D.potBC(b, f, p);
				fl[f] = (bc == PB_INSULATING || bc == PB_THIN_WALL) ? S(0) : velC;
			} else if (D.atBound(b, f, p) && D.ftype(b, f) == FT_CONNECTED) {
				int ob, op[3]; connectedPos(D, b, f, p, 0, ob, op);
				S velN = contra(D, ob, op, D.face(b, f)[2] >> 1, field);
				if (connectedSameSide(D, b, f)) velN = -velN;
				fl[f] = (velN + velC) * S(0.5);
			} else {
				int nbk, np[3]; neighbor(D, b, f, p, nbk, np);
				fl[f] = (contra(D, nbk, np, dim, field) + velC) * S(0.5);
			}
		}
		S dv = 0;
		for (int d = 0; d < D.dims; ++d) dv += fl[d * 2 + 1] - fl[d * 2];
		for (int f = 0; f < 2 * D.dims; ++f) {
			if (!D.atBound(b, f, p) || D.ftype(b, f) != FT_FIXED) continue;
			if (D.potBC(b, f, p) != PB_DIRICHLET) continue;
			const S gv = D.potValue(b, f, p);
			if (gv == S(0)) continue;
			dv -= alphaOf(D, D.T(b, p), f >> 1) * gv;
		}
		div[g] = dv;
	});
}

// potential.cu:718-880 computeCurrentDensityFaceBased; uxb holds 3 components in 2D
template <typename S>
static void currentDensity(const Dom<S> &D, const S *phi, const S *uxb, S *J) {
	forEachCell<S>(D, [&](int b, const int *p, int g) {
		const S phiP = phi[g];
		const S *tP = D.T(b, p);
		S alphaP[3] = {0, 0, 0}, cvelP[3] = {0, 0, 0};
		for (int d = 0; d < D.dims; ++d) { alphaP[d] = alphaOf(D, tP, d); cvelP[d] = contra(D, b, p, d, uxb); }
		S jf[6] = {0, 0, 0, 0, 0, 0};
		for (int f = 0; f < 2 * D.dims; ++f) {
			const int dim = f >> 1;
			const S faceSign = (f & 1) ? S(1) : S(-1);
			const bool ab = D.atBound(b, f, p);
			if (ab && D.isEmpty(b, f)) {
				const int bc = D.potBC(b, f, p);
				if (bc == PB_INSULATING || bc == PB_THIN_WALL) jf[f] = 0;
				else if (bc == PB_DIRICHLET) jf[f] = alphaP[dim] * faceSign * (phiP - D.potValue(b, f, p)) + cvelP[dim];
				else jf[f] = cvelP[dim];
				continue;
			}
			int nbk, np[3]; neighbor(D, b, f, p, nbk, np);
			S phiN = phi[D.glob(nbk, np)];
			S alphaN, cvelN;
			if (ab && D.ftype(b, f) == FT_CONNECTED) {
				const int ca = connectedChannel(D, b, f, dim);
				alphaN = alphaOf(D, D.T(nbk, np), ca);
				cvelN = contra(D, nbk, np, ca, uxb);
				if (connectedSameSide(D, b, f)) cvelN = -cvelN;
			} else {
				alphaN = alphaOf(D, D.T(nbk, np), dim);
				cvelN = contra(D, nbk, np, dim, uxb);
			}
			const S coeff = S(0.5) * (alphaP[dim] + alphaN);
			const S chi = S(0.5) * (cvelP[dim] + cvelN);
			jf[f] = -coeff * faceSign * (phiN - phiP) + chi;
		}
		S javg[3] = {0, 0, 0};
		for (int d = 0; d < D.dims; ++d) javg[d] = S(0.5) * (jf[d * 2] + jf[d * 2 + 1]);
		const S invDet = S(1) / D.det(tP);
		S out[3] = {0, 0, 0};
		for (int r = 0; r < D.dims; ++r) {
			S s = 0;
			for (int c = 0; c < D.dims; ++c) s += tP[r * D.dims + c] * javg[c];
			out[r] = s * invDet;
		}
		if (D.dims == 2) out[2] = uxb[(size_t)2 * D.n + g];
		for (int c = 0; c < 3; ++c) J[(size_t)c * D.n + g] = out[c];
	});
}

// ---------------------------------------------------------------------------------------
// Krylov solvers: the reference's stop rule ||r||_2 / sqrt(n) < tol
// (solvers/krylov/krylov.cu:292-366 initial check, :502-568 CG, :599-824 BiCGStab)

template <typename S>
static void spmv(int n, const int *row, const int *col, const S *val, const S *x, S *y) {
	#pragma omp parallel for schedule(static)
	for (int i = 0; i < n; ++i) {
		S s = 0;
		for (int j = row[i]; j < row[i + 1]; ++j) s += val[j] * x[col[j]];
		y[i] = s;
	}
}
template <typename S>
static double dotd(int n, const S *a, const S *b) {
	double s = 0;
	#pragma omp parallel for reduction(+ : s) schedule(static)
	for (int i = 0; i < n; ++i) s += double(a[i]) * double(b[i]);
	return s;
}

// returns status: 1 converged, 2 nonfinite, 3 maxit; iters/crit out
template <typename S>
static int cg(int n, const int *row, const int *col, const S *val, const S *b, S *x, double tol, int maxit, int *iters, double *critOut) {
	std::vector<S> r(n), p(n), q(n);
	spmv(n, row, col, val, x, q.data());
	for (int i = 0; i < n; ++i) r[i] = b[i] - q[i];
	const double ns = 1.0 / std::sqrt(double(n));
	double rr = dotd(n, r.data(), r.data());
	double crit = std::sqrt(rr) * ns;
	*critOut = crit; *iters = 0;
	if (!std::isfinite(crit)) return 2;
	if (crit == 0.0) return 1;
	double rho = rr, beta = 0;
	bool restart = true;
	for (int it = 1;; ++it) {
		#pragma omp parallel for schedule(static)
		for (int i = 0; i < n; ++i) p[i] = restart ? r[i] : r[i] + S(beta) * p[i];
		restart = false;
		spmv(n, row, col, val, p.data(), q.data());
		const double pq = dotd(n, p.data(), q.data());
		const double alpha = rho / pq;
		if (!std::isfinite(alpha)) { *iters = it - 1; return 2; }
		const S a = S(alpha);
		#pragma omp parallel for schedule(static)
		for (int i = 0; i < n; ++i) { x[i] += a * p[i]; r[i] -= a * q[i]; }
		rr = dotd(n, r.data(), r.data());
		crit = std::sqrt(rr) * ns;
		*critOut = crit; *iters = it;
		if (!std::isfinite(crit)) return 2;
		if (crit < tol) return 1;
		if (it >= maxit) return 3;
		beta = rr / rho;
		rho = rr;
	}
}

template <typename S>
static int bicgstab(int n, const int *row, const int *col, const S *val, const S *b, S *x, double tol, int maxit, int *iters, double *critOut) {
	std::vector<S> r(n), r0(n), p(n), v(n), s(n), t(n);
	spmv(n, row, col, val, x, v.data());
	for (int i = 0; i < n; ++i) { r[i] = b[i] - v[i]; r0[i] = r[i]; }
	const double ns = 1.0 / std::sqrt(double(n));
	double rho = dotd(n, r.data(), r.data());
	double crit = std::sqrt(rho) * ns;
	*critOut = crit; *iters = -1;
	if (!std::isfinite(crit)) return 2;
	if (crit < tol) return 1;
	double alpha = 0, omega = 0, beta = 0;
	bool restart = true;
	int it = 0;
	for (;;) {
		#pragma omp parallel for schedule(static)
		for (int i = 0; i < n; ++i) p[i] = restart ? r[i] : r[i] + S(beta) * (p[i] - S(omega) * v[i]);
		restart = false;
		spmv(n, row, col, val, p.data(), v.data());
		alpha = rho / dotd(n, r0.data(), v.data());
		if (!std::isfinite(alpha)) { *iters = it; return 2; }
		#pragma omp parallel for schedule(static)
		for (int i = 0; i < n; ++i) s[i] = r[i] - S(alpha) * v[i];
		spmv(n, row, col, val, s.data(), t.data());
		const double critS = std::sqrt(dotd(n, s.data(), s.data())) * ns;
		if (!std::isfinite(critS)) { *critOut = critS; *iters = it; return 2; }
		if (critS < tol) {
			for (int i = 0; i < n; ++i) { x[i] += S(alpha) * p[i]; r[i] = s[i]; }
			*critOut = critS; *iters = it; return 1;
		}
		omega = dotd(n, t.data(), s.data()) / dotd(n, t.data(), t.data());
		if (!std::isfinite(omega)) { *critOut = critS; *iters = it; return 2; }
		#pragma omp parallel for schedule(static)
		for (int i = 0; i < n; ++i) { x[i] += S(alpha) * p[i] + S(omega) * s[i]; r[i] = s[i] - S(omega) * t[i]; }
		const double rhoNew = dotd(n, r0.data(), r.data());
		crit = std::sqrt(dotd(n, r.data(), r.data())) * ns;
		*critOut = crit;
		if (!std::isfinite(crit)) { *iters = it; return 2; }
		if (crit < tol) { *iters = it + 1; return 1; }
		++it;
		*iters = it - 1;
		beta = (rhoNew / rho) * (alpha / omega);
		rho = rhoNew;
		if (!std::isfinite(beta)) return 2;
		if (it >= maxit) return 3;
	}
}

} // namespace orc

// ---------------------------------------------------------------------------------------
// extern "C" surface (ctypes). Suffix _d: double, _f: float.
#define ORC_DOM(S) orc::Dom<S> D(desc, Tc, Tf, fvel, fpot, fcw, fmask)
#define ORC_DOM_ARGS(S) const int32_t *desc, const S *Tc, const S *Tf, const S *fvel, const S *fpot, const S *fcw, const int8_t *fmask

#define ORC_INSTANTIATE(S, SUF)                                                                                          \
extern "C" void orc_row_pointers##SUF(ORC_DOM_ARGS(S), int *row) { ORC_DOM(S); orc::rowPointers(D, row); }              \
extern "C" void orc_adv_matrix##SUF(ORC_DOM_ARGS(S), const S *u, double dt, double nu, const int *row, int *col, S *val, S *Adiag, \
		int scheme, int flags) {                                                                                           \
	ORC_DOM(S); orc::advMatrix<S>(D, u, S(dt), S(nu), row, col, val, Adiag, nullptr, scheme, flags); }                    \
extern "C" void orc_scalar_matrix##SUF(ORC_DOM_ARGS(S), const S *u, double dt, double nu, const int8_t *types,            \
		const int *row, int *col, S *val, S *Adiag, int scheme, int flags) {                                              \
	ORC_DOM(S); orc::advMatrix<S>(D, u, S(dt), S(nu), row, col, val, Adiag, types, scheme, flags); }                       \
extern "C" void orc_scalar_rhs##SUF(ORC_DOM_ARGS(S), const S *phi, double dt, double nu, const int8_t *types,            \
		const S *values, const int64_t *offsets, const int8_t *statics, S *rhs, const S *u, int scheme, int flags,        \
		const S *phires) {                                                                                                 \
	ORC_DOM(S); orc::scalarRhs<S>(D, phi, S(dt), S(nu), types, values, offsets, statics, rhs, u, scheme, flags, phires); } \
extern "C" void orc_adv_rhs##SUF(ORC_DOM_ARGS(S), const S *u, const S *src, int srcStatic, double dt, double nu, S *rhs, \
		int scheme, int flags, const S *ures) {                                                                            \
	ORC_DOM(S); orc::advRhs<S>(D, u, src, srcStatic, S(dt), S(nu), rhs, scheme, flags, ures); }                          \
extern "C" void orc_laplace_matrix##SUF(ORC_DOM_ARGS(S), const S *Adiag, int epot, const int *row, int *col, S *val,   \
		int flags) {                                                                                                       \
	ORC_DOM(S); orc::laplaceMatrix<S>(D, Adiag, epot != 0, row, col, val, flags); }                                      \
extern "C" void orc_pressure_nonortho##SUF(ORC_DOM_ARGS(S), const S *Adiag, const S *pr, int flags, S *div) {            \
	ORC_DOM(S); orc::pressureNonOrtho<S>(D, Adiag, pr, flags, div); }                                                     \
extern "C" void orc_pressure_rhs##SUF(ORC_DOM_ARGS(S), const int *row, const int *col, const S *Cval, const S *Adiag,   \
		const S *u, const S *ustar, const S *src, int srcStatic, double dt, double nu, S *hbya, int scheme) {           \
	ORC_DOM(S); orc::pressureRhs<S>(D, row, col, Cval, Adiag, u, ustar, src, srcStatic, S(dt), S(nu), hbya, scheme); } \
extern "C" void orc_divergence##SUF(ORC_DOM_ARGS(S), const S *field, S *div) { ORC_DOM(S); orc::divergence<S>(D, field, div); } \
extern "C" void orc_correct_velocity##SUF(ORC_DOM_ARGS(S), const S *pr, const S *hbya, const S *Adiag, S *uout) {       \
	ORC_DOM(S); orc::correctVelocity<S>(D, pr, hbya, Adiag, uout); }                                                     \
extern "C" void orc_epot_rhs##SUF(ORC_DOM_ARGS(S), const S *field, S *div) { ORC_DOM(S); orc::epotRhs<S>(D, field, div); } \
extern "C" void orc_current_density##SUF(ORC_DOM_ARGS(S), const S *phi, const S *uxb, S *J) {                            \
	ORC_DOM(S); orc::currentDensity<S>(D, phi, uxb, J); }                                                                \
extern "C" int orc_cg##SUF(int n, const int *row, const int *col, const S *val, const S *b, S *x, double tol, int maxit, int *iters, double *crit) { \
	return orc::cg<S>(n, row, col, val, b, x, tol, maxit, iters, crit); }                                                \
extern "C" int orc_bicgstab##SUF(int n, const int *row, const int *col, const S *val, const S *b, S *x, double tol, int maxit, int *iters, double *crit) { \
	return orc::bicgstab<S>(n, row, col, val, b, x, tol, maxit, iters, crit); }                                          \
extern "C" void orc_spmv##SUF(int n, const int *row, const int *col, const S *val, const S *x, S *y) { orc::spmv<S>(n, row, col, val, x, y); }

ORC_INSTANTIATE(double, _d)
ORC_INSTANTIATE(float, _f)

// grid/grid_gen.cu:299-354 k_CoordsToTransforms. coords: [d][vz][vy][vx] vertex layout of a
// block's vertexCoordinates tensor; out: [cells][2d^2+1] = {M, Minv, det}, M[i][k] = dx_i/dxi_k
template <typename S>
static void cellTransforms(int dims, int nx, int ny, int nz, const S *coords, S *out) {
	const int vx = nx + 1, vy = dims > 1 ? ny + 1 : 1, vz = dims > 2 ? nz + 1 : 1;
	const int cy = dims > 1 ? ny : 1, cz = dims > 2 ? nz : 1;
	const int TS = 2 * dims * dims + 1;
	const size_t vstride = (size_t)vx * vy * vz;
	for (int z = 0; z < cz; ++z)
		for (int y = 0; y < cy; ++y)
			for (int x = 0; x < nx; ++x) {
				S fc[6][3] = {};
				const int nv = 1 << dims;
				for (int v = 0; v < nv; ++v) {
					const int px = x + (v & 1), py = y + ((v & 2) != 0), pz = z + ((v & 4) != 0);
					S c[3];
					for (int k = 0; k < dims; ++k) c[k] = coords[k * vstride + ((size_t)pz * vy + py) * vx + px];
					for (int fi = 0; fi < dims; ++fi) {
						const int up = (v & (1 << fi)) != 0;
						for (int k = 0; k < dims; ++k) fc[fi * 2 + up][k] += c[k];
					}
				}
				const S norm = S(1) / S(1 << (dims - 1));
				for (int f = 0; f < 2 * dims; ++f) for (int k = 0; k < dims; ++k) fc[f][k] *= norm;
				S M[3][3] = {};
				for (int i = 0; i < dims; ++i) for (int k = 0; k < dims; ++k) M[i][k] = fc[k * 2 + 1][i] - fc[k * 2][i];
				S *o = out + (((size_t)z * cy + y) * nx + x) * TS;
				S det, Mi[3][3] = {};
				if (dims == 1) { det = M[0][0]; Mi[0][0] = S(1) / det; }
				else if (dims == 2) {
					det = M[0][0] * M[1][1] - M[1][0] * M[0][1];
					const S inv = S(1) / det;
					Mi[0][0] = M[1][1] * inv; Mi[0][1] = -M[0][1] * inv; Mi[1][0] = -M[1][0] * inv; Mi[1][1] = M[0][0] * inv;
				} else {
					det = M[0][0] * (M[1][1] * M[2][2] - M[2][1] * M[1][2]) - M[0][1] * (M[1][0] * M[2][2] - M[2][0] * M[1][2]) + M[0][2] * (M[1][0] * M[2][1] - M[2][0] * M[1][1]);
					const S inv = S(1) / det;
					Mi[0][0] = (M[1][1] * M[2][2] - M[2][1] * M[1][2]) * inv;
					Mi[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * inv;
					Mi[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * inv;
					Mi[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) * inv;
					Mi[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * inv;
					Mi[1][2] = (M[1][0] * M[0][2] - M[0][0] * M[1][2]) * inv;
					Mi[2][0] = (M[1][0] * M[2][1] - M[2][0] * M[1][1]) * inv;
					Mi[2][1] = (M[2][0] * M[0][1] - M[0][0] * M[2][1]) * inv;
					Mi[2][2] = (M[0][0] * M[1][1] - M[1][0] * M[0][1]) * inv;
				}
				for (int i = 0; i < dims; ++i) for (int k = 0; k < dims; ++k) { o[i * dims + k] = M[i][k]; o[dims * dims + i * dims + k] = Mi[i][k]; }
				o[2 * dims * dims] = det;
			}
}

// grid/grid_gen.cu:398-490 k_CoordsToFaceTransforms, sliced at one block face as
// Block::GetFaceTransformBoundarySlice does (domain/block.cpp:790-816).
// out: [faceCells][2d^2+1], face cells ordered x-fastest over the face's cell grid.
template <typename S>
static void faceTransformsAtBoundary(int dims, int nx, int ny, int nz, const S *coords, int face, S *out) {
	const int vsz[3] = {nx + 1, dims > 1 ? ny + 1 : 1, dims > 2 ? nz + 1 : 1};
	const int csz[3] = {nx, dims > 1 ? ny : 1, dims > 2 ? nz : 1};
	const int TS = 2 * dims * dims + 1;
	const size_t vstride = (size_t)vsz[0] * vsz[1] * vsz[2];
	const int dim = face >> 1;
	int fsz[3] = {csz[0], csz[1], csz[2]};
	fsz[dim] = 1;
	auto vert = [&](const int *vp, int k) { return coords[k * vstride + ((size_t)vp[2] * vsz[1] + vp[1]) * vsz[0] + vp[0]]; };
	const int numFaceVertices = 1 << (dims - 1);
	const int numEdgeVertices = dims > 1 ? 1 << (dims - 2) : 1;
	for (int fz = 0; fz < fsz[2]; ++fz)
		for (int fy = 0; fy < fsz[1]; ++fy)
			for (int fx = 0; fx < fsz[0]; ++fx) {
				int pos[3] = {fx, fy, fz};
				pos[dim] = (face & 1) ? csz[dim] : 0; // vertex index of the face along the normal
				S t[3][3] = {};
				S normWeight = 0.5;
				for (int up = 0; up < 2; ++up) {
					const int faceSign = up * 2 - 1;
					const bool atB = up ? pos[dim] == vsz[dim] - 1 : pos[dim] == 0;
					int fp[3] = {pos[0], pos[1], pos[2]};
					if (!atB) fp[dim] += faceSign; else normWeight = 1.0;
					for (int v = 0; v < numFaceVertices; ++v) {
						int vp[3] = {fp[0], fp[1], fp[2]};
						for (int i = 1; i < dims; ++i) vp[(dim + i) % dims] += (v & i) != 0;
						for (int k = 0; k < dims; ++k) t[k][dim] += vert(vp, k) * S(faceSign);
					}
				}
				normWeight /= S(numFaceVertices);
				for (int k = 0; k < dims; ++k) t[k][dim] *= normWeight;
				const S tNorm = S(1) / S(numEdgeVertices);
				for (int kk = 1; kk < dims; ++kk) {
					const int tDim = (dim + kk) % dims;
					for (int v = 0; v < numFaceVertices; ++v) {
						int vp[3] = {pos[0], pos[1], pos[2]};
						for (int i = 1; i < dims; ++i) vp[(dim + i) % dims] += (v & i) != 0;
						const S ts = (v & kk) ? S(1) : S(-1);
						for (int k = 0; k < dims; ++k) t[k][tDim] += vert(vp, k) * ts;
					}
					for (int k = 0; k < dims; ++k) t[k][tDim] *= tNorm;
				}
				S *o = out + (((size_t)fz * fsz[1] + fy) * fsz[0] + fx) * TS;
				S det, Mi[3][3] = {};
				S (&M)[3][3] = t;
				if (dims == 1) { det = M[0][0]; Mi[0][0] = S(1) / det; }
				else if (dims == 2) {
					det = M[0][0] * M[1][1] - M[1][0] * M[0][1];
					const S inv = S(1) / det;
					Mi[0][0] = M[1][1] * inv; Mi[0][1] = -M[0][1] * inv; Mi[1][0] = -M[1][0] * inv; Mi[1][1] = M[0][0] * inv;
				} else {
					det = M[0][0] * (M[1][1] * M[2][2] - M[2][1] * M[1][2]) - M[0][1] * (M[1][0] * M[2][2] - M[2][0] * M[1][2]) + M[0][2] * (M[1][0] * M[2][1] - M[2][0] * M[1][1]);
					const S inv = S(1) / det;
					Mi[0][0] = (M[1][1] * M[2][2] - M[2][1] * M[1][2]) * inv;
					Mi[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * inv;
					Mi[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * inv;
					Mi[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) * inv;
					Mi[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * inv;
					Mi[1][2] = (M[1][0] * M[0][2] - M[0][0] * M[1][2]) * inv;
					Mi[2][0] = (M[1][0] * M[2][1] - M[2][0] * M[1][1]) * inv;
					Mi[2][1] = (M[2][0] * M[0][1] - M[0][0] * M[2][1]) * inv;
					Mi[2][2] = (M[0][0] * M[1][1] - M[1][0] * M[0][1]) * inv;
				}
				for (int i = 0; i < dims; ++i) for (int k = 0; k < dims; ++k) { o[i * dims + k] = M[i][k]; o[dims * dims + i * dims + k] = Mi[i][k]; }
				o[2 * dims * dims] = det;
			}
}

extern "C" void orc_cell_transforms_d(int dims, int nx, int ny, int nz, const double *coords, double *out) { cellTransforms<double>(dims, nx, ny, nz, coords, out); }
extern "C" void orc_cell_transforms_f(int dims, int nx, int ny, int nz, const float *coords, float *out) { cellTransforms<float>(dims, nx, ny, nz, coords, out); }
extern "C" void orc_face_transforms_d(int dims, int nx, int ny, int nz, const double *coords, int face, double *out) { faceTransformsAtBoundary<double>(dims, nx, ny, nz, coords, face, out); }
extern "C" void orc_face_transforms_f(int dims, int nx, int ny, int nz, const float *coords, int face, float *out) { faceTransformsAtBoundary<float>(dims, nx, ny, nz, coords, face, out); }
