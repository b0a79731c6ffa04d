// Device-side topology of the phipict_b200 PISO step.
//
// A batch is a concatenation of instances; each instance is a multi-block structured grid
// whose blocks are stored x-fastest. Per-cell kernels run one CTA per tile of PHB_TILE
// cells of one block, so a CTA never straddles a block (nor an instance): the block record
// is staged once into shared memory and every per-instance reduction is a sum over a
// contiguous range of CTAs.
//
// Neighbour resolution across block faces follows phiPICT's device topology
// (piso/device/topology.cuh:168-246): a periodic face wraps to the opposite side, a
// connected face maps the position into the other block through the connection axes
// written by ConnectBlocks (domain/boundaries.cpp:857-891), a fixed face is prescribed.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/phipict_b200.h"

namespace phb {

enum FaceType { FT_FIXED = 0, FT_PERIODIC = 1, FT_CONNECTED = 2 };
enum PotBC { PB_INSULATING = 0, PB_OPEN = 1, PB_DIRICHLET = 2, PB_THIN_WALL = 3 };

// block record fields
enum {
	B_NX = 0, B_NY = 1, B_NZ = 2, B_CELLOFF = 3, B_METOFF = 4, B_INST = 5, B_INSTOFF = 6, B_INSTN = 7,
	B_FACE = 8, /* 6 faces x {type, other, ax0, ax1, ax2, fixedId} */
	B_TILESTART = 44
};
// fixed record fields
enum {
	F_BLOCK = 0, F_FACE = 1, F_VELSTATIC = 2, F_VELTYPE = 3, F_POTTYPE = 4, F_POTMASK = 5, F_POTVAL = 6,
	F_VELOFF = 7, F_FACECELLS = 8, F_TOFF = 9
};
// instance record fields
enum { I_CELLOFF = 0, I_NCELLS = 1, I_TILESTART = 2, I_TILECOUNT = 3, I_BLOCKSTART = 4, I_BLOCKCOUNT = 5 };

template <int D> struct Tr { static constexpr int TS = 2 * D * D + 1; static constexpr int MINV = D * D; static constexpr int DET = 2 * D * D; };

// Read-only view of the domain descriptor, usable in device code.
template <typename S, int D>
struct Dom {
	const int32_t *blocks, *tiles, *fixed, *insts;
	const S *met, *fmet, *fvel, *fpot, *fcw;
	const int8_t *fmask;
	const double *dt, *nu;
	int64_t ms, fms, ncells;
	int nblocks, ninst, ntiles;
	int scheme = 0; // AdvectionScheme: 0 CENTRAL, 1 LINEAR_UPWIND
	int nonortho = 0; // non-orthogonal flag bits of the matrix and right-hand-side builders
	// set by a launcher whose vector and stencil operands all start on 16-byte boundaries and
	// whose ncells is a multiple of 4: 4-cell groups at aligned indices may use vector loads
	int vec4 = 0;
	// set by a launcher when the metric rows start on 16-byte boundaries (array and stride)
	int metal = 0;

	Dom() = default;
	__host__ Dom(const phb_domain &d)
		: blocks(d.blocks), tiles(d.tiles), fixed(d.fixed), insts(d.insts),
		  met((const S *)d.metrics), fmet((const S *)d.face_metrics), fvel((const S *)d.fvel),
		  fpot((const S *)d.fpot), fcw((const S *)d.fcw), fmask(d.fmask), dt(d.dt), nu(d.nu),
		  ms(d.metric_stride), fms(d.face_metric_stride), ncells(d.ncells), nblocks(d.nblocks),
		  ninst(d.ninst), ntiles(d.ntiles), scheme(d.scheme), nonortho(d.nonortho) {}

	__device__ __forceinline__ const int32_t *blk(int b) const { return blocks + b * PHB_BREC; }
	__device__ __forceinline__ const int32_t *fix(int k) const { return fixed + k * PHB_FREC; }
	__device__ __forceinline__ S m(int k, int64_t idx) const { return __ldg(met + k * ms + idx); }
	__device__ __forceinline__ S fm(int k, int64_t idx) const { return __ldg(fmet + k * fms + idx); }
};

// A cell position inside a block, with its state and metric indices.
struct Cell {
	const int32_t *B; // block record
	int b;
	int p[3];
	int g;  // global cell (state index)
	int mi; // metric index
};

__device__ __forceinline__ int bsz(const int32_t *B, int a) { return B[B_NX + a]; }
__device__ __forceinline__ int fType(const int32_t *B, int f) { return B[B_FACE + f * 6]; }
__device__ __forceinline__ const int32_t *fRec(const int32_t *B, int f) { return B + B_FACE + f * 6; }
__device__ __forceinline__ bool atBound(const int32_t *B, int f, const int *p) {
	const int ax = f >> 1;
	return (f & 1) ? p[ax] == B[B_NX + ax] - 1 : p[ax] == 0;
}
__device__ __forceinline__ int flat(const int32_t *B, const int *p) { return p[0] + B[B_NX] * (p[1] + B[B_NY] * p[2]); }
// vector component k of state cell g in block B: [inst][comp][cells] layout
template <int D>
__device__ __forceinline__ int64_t vidx(const int32_t *B, int64_t g, int k) {
	return g + (int64_t)(D - 1) * B[B_INSTOFF] + (int64_t)k * B[B_INSTN];
}

__device__ __forceinline__ int posMod(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

// computeConnectedPos (topology.cuh:168-189): position in the other block across face f.
template <typename S, int D>
__device__ __forceinline__ void connectedPos(const Dom<S, D> &dom, const int32_t *B, int f, const int *pos, int borderOffset, int &ob, int *op) {
	const int32_t *fr = fRec(B, f);
	ob = fr[1];
	const int32_t *OB = dom.blk(ob);
	const int boundaryDim = f >> 1;
	op[0] = pos[0]; op[1] = pos[1]; op[2] = pos[2];
	int ca = fr[2] >> 1;
	op[ca] = (fr[2] & 1) ? OB[B_NX + ca] - 1 - borderOffset : borderOffset;
	{
		const int axis = (boundaryDim + 1) % D;
		ca = fr[3] >> 1;
		op[ca] = (fr[3] & 1) ? OB[B_NX + ca] - 1 - pos[axis] : pos[axis];
	}
	if (D > 2) {
		const int axis = (boundaryDim + 2) % D;
		ca = fr[4] >> 1;
		op[ca] = (fr[4] & 1) ? OB[B_NX + ca] - 1 - pos[axis] : pos[axis];
	}
}
// component of the connected block that component w of this block maps to (topology.cuh:193-203)
template <int D>
__device__ __forceinline__ int connectedChannel(const int32_t *B, int f, int w) {
	return fRec(B, f)[2 + posMod(w - (f >> 1), D)] >> 1;
}
__device__ __forceinline__ bool connectedSameSide(const int32_t *B, int f) {
	return ((fRec(B, f)[2] & 1) != 0) == ((f & 1) != 0);
}

// Neighbour across a non-prescribed face f (interior, periodic or connected).
struct Nbr {
	const int32_t *B;
	int p[3];
	int64_t g;
	int64_t mi;
	int comp;      // component of the neighbour block that this block's axis f>>1 maps to
	bool flip;     // connected same-side faces invert the normal flux
};
template <typename S, int D>
__device__ __forceinline__ Nbr neighbor(const Dom<S, D> &dom, const Cell &c, int f) {
	Nbr n;
	const int ax = f >> 1;
	n.comp = ax;
	n.flip = false;
	if (atBound(c.B, f, c.p)) {
		if (fType(c.B, f) == FT_CONNECTED) {
			int ob;
			connectedPos<S, D>(dom, c.B, f, c.p, 0, ob, n.p);
			n.B = dom.blk(ob);
			n.comp = fRec(c.B, f)[2] >> 1;
			n.flip = connectedSameSide(c.B, f);
			const int l = flat(n.B, n.p);
			n.g = n.B[B_CELLOFF] + l;
			n.mi = n.B[B_METOFF] + l;
			return n;
		}
		n.B = c.B;
		n.p[0] = c.p[0]; n.p[1] = c.p[1]; n.p[2] = c.p[2];
		n.p[ax] = (f & 1) ? 0 : c.B[B_NX + ax] - 1;
	} else {
		n.B = c.B;
		n.p[0] = c.p[0]; n.p[1] = c.p[1]; n.p[2] = c.p[2];
		n.p[ax] += (f & 1) ? 1 : -1;
	}
	const int l = flat(n.B, n.p);
	n.g = n.B[B_CELLOFF] + l;
	n.mi = n.B[B_METOFF] + l;
	return n;
}

// Index of the neighbour state cell across face f, or -1 for a prescribed face.
template <typename S, int D>
__device__ __forceinline__ int64_t neighborIndex(const Dom<S, D> &dom, const Cell &c, int f) {
	const int ax = f >> 1;
	if (!atBound(c.B, f, c.p)) {
		int64_t step = 1;
		if (ax >= 1) step *= c.B[B_NX];
		if (ax >= 2) step *= c.B[B_NY];
		return (f & 1) ? c.g + step : c.g - step;
	}
	const int t = fType(c.B, f);
	if (t == FT_FIXED) return -1;
	return neighbor<S, D>(dom, c, f).g;
}

// metric helpers -----------------------------------------------------------------------
// getLaplaceCoefficientOrthogonal (discretization.cuh:360-375): det * |Minv[c]|^2
template <typename S, int D>
__device__ __forceinline__ S alphaAt(const Dom<S, D> &dom, int64_t mi, int c) {
	S s = 0;
#pragma unroll
	for (int j = 0; j < D; ++j) { const S v = dom.m(Tr<D>::MINV + c * D + j, mi); s += v * v; }
	return dom.m(Tr<D>::DET, mi) * s;
}
template <typename S, int D>
__device__ __forceinline__ S detAt(const Dom<S, D> &dom, int64_t mi) { return dom.m(Tr<D>::DET, mi); }
// getContravariantComponent (velocity.cuh:188-199): det * Minv[c] . v, v read from a
// vector field in [inst][comp][cells] layout
template <typename S, int D>
__device__ __forceinline__ S contraAt(const Dom<S, D> &dom, const int32_t *B, int64_t g, int64_t mi, int c, const S *field) {
	S s = 0;
#pragma unroll
	for (int j = 0; j < D; ++j) s += dom.m(Tr<D>::MINV + c * D + j, mi) * field[vidx<D>(B, g, j)];
	return dom.m(Tr<D>::DET, mi) * s;
}

// det * Minv[c] . v for a vector v given by value
template <typename S, int D>
__device__ __forceinline__ S contraVec(const Dom<S, D> &dom, int64_t mi, int c, const S *v) {
	S s = 0;
#pragma unroll
	for (int j = 0; j < D; ++j) s += dom.m(Tr<D>::MINV + c * D + j, mi) * v[j];
	return dom.m(Tr<D>::DET, mi) * s;
}
// [inst][3][cells] index (u x e_b and current density always have 3 components)
__device__ __forceinline__ int64_t vidx3(const int32_t *B, int64_t g, int k) { return g + 2 * (int64_t)B[B_INSTOFF] + (int64_t)k * B[B_INSTN]; }

// fixed face helpers (block_data.cuh:137-205, topology.cuh:46-66) --------------------
__device__ __forceinline__ int faceCell(const int32_t *B, int f, const int *p) {
	const int ax = f >> 1;
	int s0 = B[B_NX], s1 = B[B_NY];
	int q0 = p[0], q1 = p[1], q2 = p[2];
	if (ax == 0) { s0 = 1; q0 = 0; }
	if (ax == 1) { s1 = 1; q1 = 0; }
	if (ax == 2) { q2 = 0; }
	return q0 + s0 * (q1 + s1 * q2);
}
template <typename S, int D>
__device__ __forceinline__ S fixedVel(const Dom<S, D> &dom, const int32_t *FR, int fc, int k) {
	if (FR[F_VELSTATIC]) return dom.fvel[FR[F_VELOFF] + k];
	return dom.fvel[FR[F_VELOFF] + k * FR[F_FACECELLS] + fc];
}
__device__ __forceinline__ int potBC(const int8_t *fmask, const int32_t *FR, int fc) {
	return FR[F_POTMASK] < 0 ? FR[F_POTTYPE] : (int)fmask[FR[F_POTMASK] + fc];
}
template <typename S, int D>
__device__ __forceinline__ S potValue(const Dom<S, D> &dom, const int32_t *FR, int fc) {
	return FR[F_POTVAL] < 0 ? S(0) : dom.fpot[FR[F_POTVAL] + fc];
}
// contravariant component c of the boundary velocity with the face metrics
// (velocity.cuh:216-237 getContravariantComponentBoundaryFixed; Neumann faces carry 0)
template <typename S, int D>
__device__ __forceinline__ S contraFixed(const Dom<S, D> &dom, const int32_t *FR, int fc, int c) {
	if (FR[F_VELTYPE] != 0) return S(0);
	const int64_t fi = FR[F_TOFF] + fc;
	S s = 0;
#pragma unroll
	for (int j = 0; j < D; ++j) s += dom.fm(Tr<D>::MINV + c * D + j, fi) * fixedVel(dom, FR, fc, j);
	return dom.fm(Tr<D>::DET, fi) * s;
}
template <typename S, int D>
__device__ __forceinline__ S alphaFixed(const Dom<S, D> &dom, const int32_t *FR, int fc, int c) {
	const int64_t fi = FR[F_TOFF] + fc;
	S s = 0;
#pragma unroll
	for (int j = 0; j < D; ++j) { const S v = dom.fm(Tr<D>::MINV + c * D + j, fi); s += v * v; }
	return dom.fm(Tr<D>::DET, fi) * s;
}

// cells each thread handles per tile: a tile is PHB_TILE_CELLS consecutive cells of one
// block, thread t takes cells t, t+PHB_TILE, ... (coalesced)
constexpr int CPT = PHB_TILE_CELLS / PHB_TILE;

// Stage the CTA's block record into shared memory; l0 = first local cell of the tile,
// nc = cells of the block.
template <typename S, int D>
__device__ __forceinline__ void loadTile(const Dom<S, D> &dom, int32_t *sB, int &l0, int &nc) {
	const int tile = blockIdx.x;
	const int b = __ldg(dom.tiles + 2 * tile);
	l0 = __ldg(dom.tiles + 2 * tile + 1);
	if (threadIdx.x < PHB_BREC) sB[threadIdx.x] = __ldg(dom.blocks + b * PHB_BREC + threadIdx.x);
	__syncthreads();
	nc = sB[B_NX] * sB[B_NY] * (D > 2 ? sB[B_NZ] : 1);
}

// The j-th cell of this thread in the tile; false past the end of the block.
template <int D>
__device__ __forceinline__ bool cellAt(const int32_t *sB, int l0, int nc, int j, Cell &c) {
	const int l = l0 + threadIdx.x + j * PHB_TILE;
	if (l >= nc || l >= l0 + PHB_TILE_CELLS) return false;
	const int nx = sB[B_NX], ny = sB[B_NY];
	c.B = sB;
	c.p[0] = l % nx;
	c.p[1] = (l / nx) % ny;
	c.p[2] = D > 2 ? l / (nx * ny) : 0;
	c.g = sB[B_CELLOFF] + l;
	c.mi = sB[B_METOFF] + l;
	return true;
}

// Four consecutive cells of a tile taken by one thread (cells l0 + 4 t + i, i < n): the
// coordinates are computed once per group, and a group inside one row away from the y and z
// faces of its block has its stencil neighbours at the fixed strides 1, nx and nx*ny (only a
// row end needs the neighbour across the x face), so that four cells' loads issue together
// (as 16-byte vectors when aligned) instead of one neighbour search per cell and face.
static_assert(PHB_TILE_CELLS == 4 * PHB_TILE, "a quad is four cells per thread");
struct Quad {
	const int32_t *B; // block record
	int64_t g;        // flat index of the first cell
	int l;            // block-local index of the first cell
	int n;            // valid cells, 0..4
	int p[3];         // coordinates of the first cell
	int sy, sz;       // neighbour strides in y and z
	bool fast;        // four valid cells in one row, none on a y or z face of the block: the
	                  // neighbours are at fixed strides except across an x face at a row end
	bool al;          // four valid cells at a 4-aligned index of every operand: vector loads
	bool alY, alZ;    // al, and the y (z) neighbour groups aligned too
	bool fastW;       // as fast, but also on a y or z face of the block where that face is
	                  // prescribed (a wall): the neighbour across it is absent
	unsigned char miss; // fastW quads: bit 0/1/2/3 set when the -y/+y/-z/+z neighbour is absent
};

// K: right-hand sides per instance ([inst][K][cells] layout; their offsets must keep the
// alignment for vector access).
template <int D, int K = 1>
__device__ __forceinline__ void quadAt(int vec4, const int32_t *sB, int l0, int nc, Quad &q) {
	const int l = l0 + 4 * (int)threadIdx.x;
	const int nx = sB[B_NX], ny = sB[B_NY];
	q.B = sB;
	q.l = l;
	q.n = max(0, min(4, nc - l));
	q.g = (int64_t)sB[B_CELLOFF] + l;
	const int row = l / nx;
	q.p[0] = l - row * nx;
	q.p[1] = D > 2 ? row % ny : row;
	q.p[2] = D > 2 ? row / ny : 0;
	q.sy = nx;
	q.sz = nx * ny;
	bool fast = q.n == 4 && q.p[0] + 3 <= nx - 1 && q.p[1] >= 1 && q.p[1] <= ny - 2;
	if (D > 2) fast = fast && q.p[2] >= 1 && q.p[2] <= sB[B_NZ] - 2;
	q.fast = fast;
	// a row on a prescribed y or z face keeps the fixed strides: its neighbour across that face
	// is absent, as a per-cell resolution finds it (neighborIndex returns -1 there)
	bool inner = q.n == 4 && q.p[0] + 3 <= nx - 1;
	int miss = 0;
	if (q.p[1] == 0) { if (fType(sB, 2) == FT_FIXED) miss |= 1; else inner = false; }
	if (q.p[1] == ny - 1) { if (fType(sB, 3) == FT_FIXED) miss |= 2; else inner = false; }
	if (D > 2) {
		if (q.p[2] == 0) { if (fType(sB, 4) == FT_FIXED) miss |= 4; else inner = false; }
		if (q.p[2] == sB[B_NZ] - 1) { if (fType(sB, 5) == FT_FIXED) miss |= 8; else inner = false; }
	}
	q.fastW = inner;
	q.miss = (unsigned char)miss;
	bool al = vec4 && q.n == 4 && (q.g & 3) == 0;
	if (K > 1) al = al && ((sB[B_INSTOFF] | sB[B_INSTN]) & 3) == 0;
	q.al = al;
	q.alY = al && (nx & 3) == 0;
	q.alZ = al && (q.sz & 3) == 0;
}

// Vector loads of the quad's four cell transforms (metric index mi0 of its first cell).
template <typename S, int D>
__device__ __forceinline__ bool metAligned(const Dom<S, D> &dom, const Quad &q, int64_t mi0) {
	return dom.metal && q.n == 4 && (mi0 & 3) == 0;
}

// The i-th cell of a quad (i < q.n) as a Cell.
template <int D>
__device__ __forceinline__ void quadCell(const Quad &q, int i, Cell &c) {
	const int nx = q.B[B_NX], ny = q.B[B_NY];
	c.B = q.B;
	c.p[0] = q.p[0] + i;
	c.p[1] = q.p[1];
	c.p[2] = q.p[2];
	while (c.p[0] >= nx) {
		c.p[0] -= nx;
		if (++c.p[1] == ny && D > 2) { c.p[1] = 0; ++c.p[2]; }
	}
	c.g = (int)(q.g + i);
	c.mi = q.B[B_METOFF] + q.l + i;
}

// Four consecutive values: one 16-byte vector load (two for double) when `al`, else scalar
// loads of the first n (zeros after).
template <typename T>
__device__ __forceinline__ void ld4(const T *p, int n, bool al, T (&v)[4]) {
	if (al) {
		if constexpr (sizeof(T) == 4) {
			const float4 f = *reinterpret_cast<const float4 *>(p);
			v[0] = f.x; v[1] = f.y; v[2] = f.z; v[3] = f.w;
		} else {
			const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
			v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
		}
		return;
	}
#pragma unroll
	for (int i = 0; i < 4; ++i) v[i] = i < n ? p[i] : T(0);
}
template <typename T>
__device__ __forceinline__ void st4(T *p, int n, bool al, const T (&v)[4]) {
	if (al) {
		if constexpr (sizeof(T) == 4) {
			*reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
		} else {
			reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
			reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
		}
		return;
	}
#pragma unroll
	for (int i = 0; i < 4; ++i)
		if (i < n) p[i] = v[i];
}

// Passive-scalar data of a launch (phb_scalar), passed by value.
struct ScalarView {
	int channels, nuCount;
	const double *nu;
	const int8_t *types;
	const void *values;
	const int64_t *offsets;
	const int8_t *statics;
};
__host__ inline ScalarView scalarView(const phb_scalar *sc) {
	if (!sc) return ScalarView{0, 0, nullptr, nullptr, nullptr, nullptr, nullptr};
	return ScalarView{sc->channels, sc->nu_count, sc->nu, sc->types, sc->values, sc->offsets, sc->statics};
}
// getViscosity with forPassiveScalar (discretization.cuh:1141-1151): the scalar diffusivity of
// channel c, or the velocity viscosity of the instance without one
__device__ __forceinline__ double scalarNu(const ScalarView &sv, int c, double velocityNu) {
	if (sv.nuCount <= 0) return velocityNu;
	return sv.nu[sv.nuCount == 1 ? 0 : c];
}
// fixed-face scalar value of channel c at face cell fc (getFixedBoundaryData, PASSIVE_SCALAR)
template <typename S>
__device__ __forceinline__ S scalarFixed(const ScalarView &sv, const int32_t *FR, int fid, int c, int fc) {
	const S *v = (const S *)sv.values + sv.offsets[fid];
	return sv.statics[fid] ? v[c] : v[(int64_t)c * FR[F_FACECELLS] + fc];
}
// [inst][channels][cells] index of channel c of cell g
__device__ __forceinline__ int64_t sidx(const int32_t *B, int64_t g, int c, int channels) {
	return g + (int64_t)(channels - 1) * B[B_INSTOFF] + (int64_t)c * B[B_INSTN];
}

} // namespace phb
