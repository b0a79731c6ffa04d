// Per-cell assembly kernels of the PISO/MHD step.
//
// One thread per cell, one CTA per tile of one block (phb_device.cuh). Matrices are
// written as stencils value[slot][cell] (slot 0 diagonal, slot f+1 face f), which keeps
// every store coalesced and needs no column indices; the CSR view phiPICT exposes is a
// gather over the same values (csr.cu). Metrics are SoA so that each of the 2d^2+1
// metric loads of a warp is one coalesced transaction.
//
// The arithmetic of every kernel follows the reference kernel named in its comment
// (paths relative to the phiPICT source tree).
#include "phb_device.cuh"
#include "phb_launch.cuh"
#include "phb_nonortho.cuh"
#include "phb_upwind.cuh"
#include <initializer_list>

namespace phb {

// PISO_build_matrix (piso/advection.cu:27-305): implicit Euler advection-diffusion row
// divided by the cell determinant; Adiag = its diagonal. SCALAR: the matrix of passive-scalar
// channel `channel` (forPassiveScalar): its diffusivity, and the wall diffusion term of a fixed
// face taken from the scalar's face type instead of the velocity's (advection.cu:254-266).
// NO: with the non-orthogonal cross terms of dom.nonortho (advection.cu:176-240), the
// velocity matrix weighting them with the viscosity, the scalar matrix scaling them by its
// diffusivity (advection.cu:181-195).
template <typename S, int D, bool SCALAR = false, bool NO = false>
__global__ void __launch_bounds__(PHB_TILE) kAdvectionMatrix(Dom<S, D> dom, const S *__restrict__ u, S *__restrict__ C,
		S *__restrict__ Adiag, float *__restrict__ Clo, ScalarView sv = {}, int channel = 0) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	const int inst = c.B[B_INST];
	const S dt = S(dom.dt[inst]);
	const S nu = SCALAR ? S(scalarNu(sv, channel, dom.nu[inst])) : S(dom.nu[inst]);
	BPos bp;
	S ia[2 * D][2];
	NField<S> F;
	if constexpr (NO) {
		bp = BPos{__ldg(dom.tiles + 2 * blockIdx.x), {c.p[0], c.p[1], c.p[2]}};
		nonOrthoInterp<S, D>(dom, bp, [&](int64_t) { return SCALAR ? S(1) : nu; }, ia);
		F = NField<S>{SCALAR ? NF_SCALAR : NF_VELOCITY, SCALAR ? channel : 0, nullptr, sv};
	}
	S fl[2 * D];
	faceFluxes<S, D>(dom, c, u, fl);
	const S det = detAt<S, D>(dom, c.mi);
	S diag = det / dt;
	S alphaP[D];
#pragma unroll
	for (int d = 0; d < D; ++d) alphaP[d] = alphaAt<S, D>(dom, c.mi, d);
	S rv[2 * D + 1];
#pragma unroll
	for (int s = 0; s < 2 * D + 1; ++s) rv[s] = 0;
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		const int dim = f >> 1;
		const S faceSign = (f & 1) ? S(1) : S(-1);
		if (!atBound(c.B, f, c.p) || fType(c.B, f) != FT_FIXED) {
			const S fout = faceSign * fl[f];
			if (dom.scheme != 0 && farUpwind(c.B, c.p, f, fout >= S(0))) {
				// first-order upwind implicitly (advection.cu:131-139)
				if (fout >= S(0)) diag += fout;
				else rv[f + 1] += fout;
			} else {
				const S half = S(0.5) * fout;
				diag += half;
				rv[f + 1] += half;
			}
			const Nbr n = neighbor<S, D>(dom, c, f);
			const S alphaN = alphaAt<S, D>(dom, n.mi, n.comp);
			const S coeff = (alphaP[dim] * nu + alphaN * nu) * S(0.5);
			diag += coeff;
			rv[f + 1] -= coeff;
			if constexpr (NO) {
				const S a[2] = {ia[f][0] * (SCALAR ? nu : S(1)), ia[f][1] * (SCALAR ? nu : S(1))};
				rv[0] = diag;
				nonOrthoMatrixFace<S, D>(dom, F, bp, f, dom.nonortho, -1, false, a, rv, innerCell<D>(c.B, c.p));
				diag = rv[0];
			}
		} else {
			const int fid = fRec(c.B, f)[5];
			const int32_t *FR = dom.fix(fid);
			const int type = SCALAR ? int(sv.types[(int64_t)fid * sv.channels + channel]) : FR[F_VELTYPE];
			const S slip = type == 0 ? S(0) : S(1);
			diag += (S(1) - slip) * S(2) * nu * alphaP[dim];
		}
	}
	rv[0] = diag;
	if constexpr (NO) {
		// a share that falls on a fixed face has no column (the reference drops it)
#pragma unroll
		for (int f = 0; f < 2 * D; ++f)
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) rv[f + 1] = 0;
	}
	const int64_t N = dom.ncells;
#pragma unroll
	for (int s = 0; s < 2 * D + 1; ++s) {
		const S v = rv[s] / det;
		C[s * N + c.g] = v;
		if (Clo) Clo[s * N + c.g] = float(v);
	}
	Adiag[c.g] = rv[0] / det;
	}
}

// boundary source of the momentum equation at fixed faces (advection.cu:834-866, the same
// terms as pressure.cu:404-432): -u_b F_b + 2 nu alpha u_b (no-slip faces)
template <typename S, int D>
__device__ __forceinline__ S boundarySource(const Dom<S, D> &dom, const Cell &c, int dim, S nu) {
	S r = 0;
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		if (!atBound(c.B, f, c.p) || fType(c.B, f) != FT_FIXED) continue;
		const S faceNormal = (f & 1) ? S(1) : S(-1);
		const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
		const int fc = faceCell(c.B, f, c.p);
		const S vel = fixedVel<S, D>(dom, FR, fc, dim);
		const S alpha = alphaFixed<S, D>(dom, FR, fc, f >> 1);
		const S flux = contraFixed<S, D>(dom, FR, fc, f >> 1) * faceNormal;
		r -= vel * flux;
		const S slip = FR[F_VELTYPE] == 0 ? S(0) : S(1);
		r += vel * (S(1) - slip) * nu * S(2) * alpha;
	}
	return r;
}
template <typename S, int D>
__device__ __forceinline__ S sourceAt(const Cell &c, const S *__restrict__ src, int mode, int dim) {
	if (mode == 1) return src[c.B[B_INST] * D + dim];
	if (mode == 2) return src[vidx<D>(c.B, c.g, dim)];
	return S(0);
}

// kPISO_build_advection_RHS (advection.cu:800-954), no pressure gradient. A thread takes four
// consecutive cells (Quad): their transforms, velocities and sources load as vectors; the
// fixed-face sources and the LINEAR_UPWIND correction are added per cell where they apply.
template <typename S, int D, bool UPW>
__global__ void __launch_bounds__(PHB_TILE, sizeof(S) == 8 ? 2 : 3) kAdvectionRhs(Dom<S, D> dom, const S *__restrict__ u, const S *__restrict__ src,
		int srcMode, S *__restrict__ rhs) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	Quad q;
	quadAt<D, D>(dom.vec4, sB, l0, nc, q);
	if (q.n == 0) return;
	const int inst = sB[B_INST];
	const S dt = S(dom.dt[inst]);
	const S nu = S(dom.nu[inst]);
	const int64_t mi0 = sB[B_METOFF] + q.l;
	S det[4];
	ld4(dom.met + Tr<D>::DET * dom.ms + mi0, q.n, metAligned(dom, q, mi0), det);
	// cells with a fixed face, or every cell with LINEAR_UPWIND, take the per-cell terms
	const bool perCell = UPW || !q.fast || q.p[0] == 0 || q.p[0] + 3 == sB[B_NX] - 1;
#pragma unroll
	for (int dim = 0; dim < D; ++dim) {
		const int64_t o = vidx<D>(q.B, q.g, dim);
		S uv[4], r[4];
		ld4(u + o, q.n, q.al, uv);
#pragma unroll
		for (int i = 0; i < 4; ++i) r[i] = det[i] * uv[i] / dt;
		if (perCell) {
#pragma unroll
			for (int i = 0; i < 4; ++i) {
				if (i >= q.n) break;
				Cell c;
				quadCell<D>(q, i, c);
				r[i] += boundarySource<S, D>(dom, c, dim, nu);
				if constexpr (UPW) {
					S fl[2 * D];
					faceFluxes<S, D>(dom, c, u, fl);
					upwindCorrection<S, D>(c, fl, [&](int64_t g) { return u[vidx<D>(c.B, g, dim)]; }, r[i]);
				}
			}
		}
		S sv[4] = {0, 0, 0, 0};
		if (srcMode == 1) {
			const S v = src[inst * D + dim];
#pragma unroll
			for (int i = 0; i < 4; ++i) sv[i] = v;
		} else if (srcMode == 2) {
			ld4(src + o, q.n, q.al, sv);
		}
#pragma unroll
		for (int i = 0; i < 4; ++i) r[i] = r[i] / det[i] + sv[i];
		st4(rhs + o, q.n, q.al, r);
	}
}

// kPISO_build_scalar_advection_RHS (advection.cu:545-698), CENTRAL, orthogonal:
// det phi / dt plus, at fixed faces, Dirichlet: -phi_b F + 2 nu alpha phi_b (ghost cell);
// Neumann: -phi_P F + nu |S_f| dphi/dn; all divided by det.
template <typename S, int D>
__global__ void __launch_bounds__(PHB_TILE) kScalarRhs(Dom<S, D> dom, const S *__restrict__ phi, const S *__restrict__ u,
		ScalarView sv, S *__restrict__ rhs) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	const int inst = c.B[B_INST];
	const S dt = S(dom.dt[inst]);
	const double nuVel = dom.nu[inst];
	const S det = detAt<S, D>(dom, c.mi);
	S fl[2 * D];
	if (dom.scheme != 0) faceFluxes<S, D>(dom, c, u, fl);
	for (int ch = 0; ch < sv.channels; ++ch) {
		const int64_t o = sidx(c.B, c.g, ch, sv.channels);
		const S phiP = phi[o];
		const S nu = S(scalarNu(sv, ch, nuVel));
		S r = det * phiP / dt;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			if (!atBound(c.B, f, c.p) || fType(c.B, f) != FT_FIXED) continue;
			const S faceNormal = (f & 1) ? S(1) : S(-1);
			const int fid = fRec(c.B, f)[5];
			const int32_t *FR = dom.fix(fid);
			const int fc = faceCell(c.B, f, c.p);
			const S value = scalarFixed<S>(sv, FR, fid, ch, fc);
			const S flux = contraFixed<S, D>(dom, FR, fc, f >> 1) * faceNormal;
			if (sv.types[(int64_t)fid * sv.channels + ch] == 0) {
				r -= value * flux;
				r += value * nu * S(2) * alphaFixed<S, D>(dom, FR, fc, f >> 1);
			} else {
				// getFaceAreaOrthogonalBoundary (discretization.cuh:618-634): det_f |Minv_f[dim]|
				const int64_t fi = FR[F_TOFF] + fc;
				S m2 = 0;
#pragma unroll
				for (int j = 0; j < D; ++j) { const S v = dom.fm(Tr<D>::MINV + (f >> 1) * D + j, fi); m2 += v * v; }
				const S area = dom.fm(Tr<D>::DET, fi) * sqrt(m2);
				r -= phiP * flux;
				r += value * nu * area;
			}
		}
		if (dom.scheme != 0) upwindCorrection<S, D>(c, fl, [&](int64_t g) { return phi[sidx(c.B, g, ch, sv.channels)]; }, r);
		rhs[o] = r / det;
	}
	}
}

// PISO_build_pressure_matrix (pressure.cu:26-191) with raP = 1/A, and
// PISO_build_epot_matrix (mhd/potential.cu:30-233) with raP = 1 plus the Dirichlet ghost
// diagonal and the thin-wall Robin correction.
// NO (pressure only): with the non-orthogonal cross terms of dom.nonortho, weighted with 1/A
// (pressure.cu:103-156).
template <typename S, int D, bool EPOT, bool NO = false>
__global__ void __launch_bounds__(PHB_TILE) kLaplaceMatrix(Dom<S, D> dom, const S *__restrict__ Adiag, S *__restrict__ P,
		float *__restrict__ Plo) {
	static_assert(!(EPOT && NO), "the potential matrix has no non-orthogonal terms here");
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	S alphaP[D];
#pragma unroll
	for (int d = 0; d < D; ++d) alphaP[d] = alphaAt<S, D>(dom, c.mi, d);
	const S raP = EPOT ? S(1) : S(1) / Adiag[c.g];
	BPos bp;
	S ia[2 * D][2];
	if constexpr (NO) {
		bp = BPos{__ldg(dom.tiles + 2 * blockIdx.x), {c.p[0], c.p[1], c.p[2]}};
		nonOrthoInterp<S, D>(dom, bp, [&](int64_t g) { return S(1) / Adiag[g]; }, ia);
	}
	S rv[2 * D + 1];
	bool has[2 * D + 1];
#pragma unroll
	for (int s = 0; s < 2 * D + 1; ++s) { rv[s] = 0; has[s] = false; }
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		const int dim = f >> 1;
		const bool ab = atBound(c.B, f, c.p);
		if (!(ab && fType(c.B, f) == FT_FIXED)) {
			const Nbr n = neighbor<S, D>(dom, c, f);
			const S alphaN = alphaAt<S, D>(dom, n.mi, n.comp);
			const S raN = EPOT ? S(1) : S(1) / Adiag[n.g];
			const S coeff = S(0.5) * (alphaP[dim] * raP + alphaN * raN);
			rv[0] -= coeff;
			rv[f + 1] += coeff;
			has[f + 1] = true;
			if constexpr (NO) {
				const NField<S> F{NF_MARK, 0, nullptr, ScalarView{}};
				nonOrthoMatrixFace<S, D>(dom, F, bp, f, dom.nonortho, 1, true, ia[f], rv, innerCell<D>(c.B, c.p));
			}
		} else if (EPOT) {
			const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
			if (potBC(dom.fmask, FR, faceCell(c.B, f, c.p)) == PB_DIRICHLET) rv[0] -= alphaP[dim] * raP;
		}
	}
	if (EPOT) {
		// potential.cu:175-219: C_w * surface Laplacian along thin conducting walls
#pragma unroll
		for (int tw = 0; tw < 2 * D; ++tw) {
			const int twDim = tw >> 1;
			if (!atBound(c.B, tw, c.p) || fType(c.B, tw) != FT_FIXED) continue;
			const int32_t *FR = dom.fix(fRec(c.B, tw)[5]);
			if (potBC(dom.fmask, FR, faceCell(c.B, tw, c.p)) != PB_THIN_WALL) continue;
			const S Cw = dom.fcw[fRec(c.B, tw)[5]];
			S nP = 0;
#pragma unroll
			for (int j = 0; j < D; ++j) { const S v = dom.m(Tr<D>::MINV + twDim * D + j, c.mi); nP += v * v; }
			const S MinvNP = sqrt(nP);
#pragma unroll
			for (int tDim = 0; tDim < D; ++tDim) {
				if (tDim == twDim) continue;
#pragma unroll
				for (int side = 0; side < 2; ++side) {
					const int tb = tDim * 2 + side;
					if (!has[tb + 1]) continue;
					int q[3] = {c.p[0], c.p[1], c.p[2]};
					if (atBound(c.B, tb, c.p)) {
						if (fType(c.B, tb) == FT_PERIODIC) q[tDim] = side ? 0 : c.B[B_NX + tDim] - 1;
						else continue;
					} else {
						q[tDim] += side ? 1 : -1;
					}
					if (potBC(dom.fmask, FR, faceCell(c.B, tw, q)) != PB_THIN_WALL) continue;
					const int64_t qm = c.B[B_METOFF] + flat(c.B, q);
					const S alphaNt = alphaAt<S, D>(dom, qm, tDim);
					S nN = 0;
#pragma unroll
					for (int j = 0; j < D; ++j) { const S v = dom.m(Tr<D>::MINV + twDim * D + j, qm); nN += v * v; }
					const S MinvNN = sqrt(nN);
					const S surf = Cw * S(0.5) * (alphaP[tDim] * MinvNP + alphaNt * MinvNN);
					rv[0] -= surf;
					rv[tb + 1] += surf;
				}
			}
		}
	}
	if constexpr (NO) {
#pragma unroll
		for (int f = 0; f < 2 * D; ++f)
			if (!has[f + 1]) rv[f + 1] = 0;
	}
	const int64_t N = dom.ncells;
#pragma unroll
	for (int s = 0; s < 2 * D + 1; ++s) {
		P[s * N + c.g] = rv[s];
		if (Plo) Plo[s * N + c.g] = float(rv[s]);
	}
	}
}

// The cold paths of kPressureRhs: H of cell i of a quad off the fast path, resolving each
// face ...
template <typename S, int D>
struct CompSums {
	S v[D];
};
template <typename S, int D>
__device__ __forceinline__ CompSums<S, D> hbyaSlowH(const Dom<S, D> &dom, const Quad &q, int i, const S *__restrict__ C,
		const S *__restrict__ ustar) {
	const int64_t N = dom.ncells;
	const int64_t cs = (int64_t)q.B[B_INSTN];
	Cell c;
	quadCell<D>(q, i, c);
	const int64_t comp = vidx<D>(c.B, c.g, 0) - c.g;
	CompSums<S, D> h;
#pragma unroll
	for (int d = 0; d < D; ++d) h.v[d] = 0;
	for (int f = 0; f < 2 * D; ++f) {
		const int64_t n = neighborIndex<S, D>(dom, c, f);
		if (n < 0 || n == c.g) continue;
		const S cvf = C[(f + 1) * N + c.g];
#pragma unroll
		for (int d = 0; d < D; ++d) h.v[d] = fma(cvf, ustar[n + comp + d * cs], h.v[d]);
	}
	return h;
}
// ... and the source of cell i with its fixed faces and the deferred LINEAR_UPWIND correction
template <typename S, int D, bool UPW>
__device__ __forceinline__ S hbyaCellSource(const Dom<S, D> &dom, const Quad &q, int i, int dim, S nu, S det, S src, const S *__restrict__ u) {
	Cell c;
	quadCell<D>(q, i, c);
	S Ssum = boundarySource<S, D>(dom, c, dim, nu);
	Ssum /= det;
	Ssum += src;
	if constexpr (UPW) {
		// HbyA repeats the predictor's deferred correction (pressure.cu:474-515)
		S fl[2 * D];
		faceFluxes<S, D>(dom, c, u, fl);
		S corr = 0;
		upwindCorrection<S, D>(c, fl, [&](int64_t g) { return u[vidx<D>(c.B, g, dim)]; }, corr);
		Ssum += corr / det;
	}
	return Ssum;
}

// Out-of-line calls of the two: in 3D the inlined cold paths make the kernel large enough to
// stall on instruction fetch (measured: HbyA on 256^3 at 0.38 of HBM out of line against 0.34
// inline), in 2D inlining is faster (0.66 against 0.55 on 4096^2).
template <typename S, int D>
__device__ __noinline__ CompSums<S, D> hbyaSlowHCall(const Dom<S, D> &dom, const Quad &q, int i, const S *__restrict__ C,
		const S *__restrict__ ustar) {
	return hbyaSlowH<S, D>(dom, q, i, C, ustar);
}
template <typename S, int D, bool UPW>
__device__ __noinline__ S hbyaCellSourceCall(const Dom<S, D> &dom, const Quad &q, int i, int dim, S nu, S det, S src,
		const S *__restrict__ u) {
	return hbyaCellSource<S, D, UPW>(dom, q, i, dim, nu, det, src, u);
}

// PISO_build_pressure_rhs (pressure.cu:350-521): HbyA = (u/dt - H(u*) + S)/A per component,
// four consecutive cells per thread. H sums the stencil's face slots in face order for every
// component at once, so that a slot's four values are loaded once and dropped.
template <typename S, int D, bool UPW>
__global__ void __launch_bounds__(PHB_TILE, sizeof(S) == 8 ? 2 : 3) kPressureRhs(Dom<S, D> dom, const S *__restrict__ C, const S *__restrict__ Adiag,
		const S *__restrict__ u, const S *__restrict__ ustar, const S *__restrict__ src, int srcMode, S *__restrict__ hbya) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	Quad q;
	quadAt<D, D>(dom.vec4, sB, l0, nc, q);
	if (q.n == 0) return;
	const int inst = sB[B_INST];
	const S dt = S(dom.dt[inst]);
	const S nu = S(dom.nu[inst]);
	const int64_t N = dom.ncells;
	const int64_t o0 = vidx<D>(q.B, q.g, 0);
	const int64_t cs = (int64_t)q.B[B_INSTN]; // component stride
	S H[D][4];
#pragma unroll
	for (int d = 0; d < D; ++d)
#pragma unroll
		for (int i = 0; i < 4; ++i) H[d][i] = 0;
	if (q.fast) {
		int64_t gW = q.g - 1, gE = q.g + 4;
		if (q.p[0] == 0 || q.p[0] + 3 == q.B[B_NX] - 1) {
			Cell c;
			c.B = q.B;
			c.p[1] = q.p[1];
			c.p[2] = q.p[2];
			if (q.p[0] == 0) {
				c.p[0] = 0;
				c.g = (int)q.g;
				gW = neighborIndex<S, D>(dom, c, 0);
			}
			if (q.p[0] + 3 == q.B[B_NX] - 1) {
				c.p[0] = q.p[0] + 3;
				c.g = (int)(q.g + 3);
				gE = neighborIndex<S, D>(dom, c, 1);
			}
		}
		const int64_t comp = o0 - q.g;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			S cv[4];
			ld4(C + (f + 1) * N + q.g, 4, q.al, cv);
#pragma unroll
			for (int d = 0; d < D; ++d) {
				if (f < 2) {
					S own[4];
					ld4(ustar + o0 + d * cs, 4, q.al, own);
					if (f == 0) {
						if (gW >= 0) H[d][0] = fma(cv[0], ustar[gW + comp + d * cs], H[d][0]);
#pragma unroll
						for (int i = 1; i < 4; ++i) H[d][i] = fma(cv[i], own[i - 1], H[d][i]);
					} else {
#pragma unroll
						for (int i = 0; i < 3; ++i) H[d][i] = fma(cv[i], own[i + 1], H[d][i]);
						if (gE >= 0) H[d][3] = fma(cv[3], ustar[gE + comp + d * cs], H[d][3]);
					}
				} else {
					const int64_t off = f == 2 ? -(int64_t)q.sy : f == 3 ? (int64_t)q.sy : f == 4 ? -(int64_t)q.sz : (int64_t)q.sz;
					S v[4];
					ld4(ustar + o0 + d * cs + off, 4, f < 4 ? q.alY : q.alZ, v);
#pragma unroll
					for (int i = 0; i < 4; ++i) H[d][i] = fma(cv[i], v[i], H[d][i]);
				}
			}
		}
	} else {
#pragma unroll
		for (int i = 0; i < 4; ++i) {
			if (i >= q.n) break;
			const CompSums<S, D> h = D > 2 ? hbyaSlowHCall<S, D>(dom, q, i, C, ustar) : hbyaSlowH<S, D>(dom, q, i, C, ustar);
#pragma unroll
			for (int d = 0; d < D; ++d) H[d][i] = h.v[d];
		}
	}
	const int64_t mi0 = sB[B_METOFF] + q.l;
	S a[4], det[4];
	ld4(Adiag + q.g, q.n, q.al, a);
	ld4(dom.met + Tr<D>::DET * dom.ms + mi0, q.n, metAligned(dom, q, mi0), det);
	const bool perCell = UPW || !q.fast || q.p[0] == 0 || q.p[0] + 3 == sB[B_NX] - 1;
#pragma unroll
	for (int dim = 0; dim < D; ++dim) {
		const int64_t o = o0 + dim * cs;
		S uv[4], sv[4] = {0, 0, 0, 0};
		ld4(u + o, q.n, q.al, uv);
		if (srcMode == 1) {
			const S v = src[inst * D + dim];
#pragma unroll
			for (int i = 0; i < 4; ++i) sv[i] = v;
		} else if (srcMode == 2) {
			ld4(src + o, q.n, q.al, sv);
		}
		S out[4];
#pragma unroll
		for (int i = 0; i < 4; ++i) {
			S Ssum = 0;
			if (perCell && i < q.n) {
				Ssum = D > 2 ? hbyaCellSourceCall<S, D, UPW>(dom, q, i, dim, nu, det[i], sv[i], u)
				             : hbyaCellSource<S, D, UPW>(dom, q, i, dim, nu, det[i], sv[i], u);
			} else {
				Ssum /= det[i];
				Ssum += sv[i];
			}
			out[i] = (S(1) / a[i]) * (uv[i] / dt - H[dim][i] + Ssum);
		}
		st4(hbya + o, q.n, q.al, out);
	}
}

// k_computePressureRHSdivergenceFromFlux (pressure.cu:756-801), no face transforms
template <typename S, int D>
__global__ void __launch_bounds__(PHB_TILE) kDivergence(Dom<S, D> dom, const S *__restrict__ field, S *__restrict__ div) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	S fl[2 * D];
	faceFluxes<S, D>(dom, c, field, fl);
	S dv = 0;
#pragma unroll
	for (int d = 0; d < D; ++d) dv += fl[d * 2 + 1] - fl[d * 2];
	div[c.g] = dv;
	}
}

// getPressureAtWithBounds for the +-1 neighbours (nonortho_laplace.cuh:302-381)
template <typename S, int D>
__device__ __forceinline__ S scalarAcross(const Dom<S, D> &dom, const Cell &c, int f, const S *__restrict__ p) {
	if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) return p[c.g];
	return p[neighbor<S, D>(dom, c, f).g];
}

// PISO_update_velocity, version 1 (velocity_correction.cu:27-60) with the finite
// difference gradient of getPressureGradient (piso/device/velocity.cuh:347-378)
template <typename S, int D>
__global__ void __launch_bounds__(PHB_TILE) kCorrectVelocity(Dom<S, D> dom, const S *__restrict__ p, const S *__restrict__ hbya,
		const S *__restrict__ Adiag, S *__restrict__ u) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	const S rDiag = S(1) / Adiag[c.g];
	S gr[D];
#pragma unroll
	for (int dim = 0; dim < D; ++dim) {
		S fac = 0.5;
		const bool lowFixed = c.p[dim] == 0 && fType(c.B, dim * 2) == FT_FIXED;
		const bool upFixed = c.p[dim] == c.B[B_NX + dim] - 1 && fType(c.B, dim * 2 + 1) == FT_FIXED;
		if (lowFixed || upFixed) fac = 1;
		const S valN = lowFixed ? p[c.g] : scalarAcross<S, D>(dom, c, dim * 2, p);
		const S valP = upFixed ? p[c.g] : scalarAcross<S, D>(dom, c, dim * 2 + 1, p);
		gr[dim] = (valP - valN) * fac;
	}
	S grad[D];
#pragma unroll
	for (int k = 0; k < D; ++k) grad[k] = 0;
#pragma unroll
	for (int r = 0; r < D; ++r)
#pragma unroll
		for (int k = 0; k < D; ++k) grad[k] += dom.m(Tr<D>::MINV + r * D + k, c.mi) * gr[r];
#pragma unroll
	for (int d = 0; d < D; ++d) {
		const int64_t o = vidx<D>(c.B, c.g, d);
		u[o] = -rDiag * grad[d] + hbya[o];
	}
	}
}

// u x e_b at a cell (simulation/mhd.py:276-355): 2D velocities are lifted to 3D
template <typename S, int D>
__device__ __forceinline__ void uCrossB(const int32_t *B, int64_t g, const S *__restrict__ u, const double *eb, S *out) {
	const S u0 = u[vidx<D>(B, g, 0)], u1 = u[vidx<D>(B, g, 1)];
	const S u2 = D > 2 ? u[vidx<D>(B, g, D > 2 ? 2 : 0)] : S(0);
	const S e0 = S(eb[0]), e1 = S(eb[1]), e2 = S(eb[2]);
	out[0] = u1 * e2 - u2 * e1;
	out[1] = u2 * e0 - u0 * e2;
	out[2] = u0 * e1 - u1 * e0;
}

// u x e_b fused with k_computeEpotRHS (mhd/potential.cu:273-323) and its face fluxes
// computeEpotFluxesNDLoop (discretization.cuh:856-912)
template <typename S, int D>
__global__ void __launch_bounds__(PHB_TILE) kUxbEpotRhs(Dom<S, D> dom, const S *__restrict__ u, const double *__restrict__ eb,
		S *__restrict__ uxb, S *__restrict__ rhs) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	const double *e = eb + 3 * c.B[B_INST];
	S x[3];
	uCrossB<S, D>(c.B, c.g, u, e, x);
#pragma unroll
	for (int k = 0; k < 3; ++k) uxb[vidx3(c.B, c.g, k)] = x[k];
	S fl[2 * D];
#pragma unroll
	for (int dim = 0; dim < D; ++dim) {
		const S velC = contraVec<S, D>(dom, c.mi, dim, x);
#pragma unroll
		for (int up = 0; up < 2; ++up) {
			const int f = dim * 2 + up;
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) {
				const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
				const int bc = potBC(dom.fmask, FR, faceCell(c.B, f, c.p));
				fl[f] = (bc == PB_INSULATING || bc == PB_THIN_WALL) ? S(0) : velC;
			} else {
				const Nbr n = neighbor<S, D>(dom, c, f);
				S xn[3];
				uCrossB<S, D>(n.B, n.g, u, e, xn);
				S velN = contraVec<S, D>(dom, n.mi, n.comp, xn);
				if (n.flip) velN = -velN;
				fl[f] = (velN + velC) * S(0.5);
			}
		}
	}
	S dv = 0;
#pragma unroll
	for (int d = 0; d < D; ++d) dv += fl[d * 2 + 1] - fl[d * 2];
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		if (!atBound(c.B, f, c.p) || fType(c.B, f) != FT_FIXED) continue;
		const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
		const int fc = faceCell(c.B, f, c.p);
		if (potBC(dom.fmask, FR, fc) != PB_DIRICHLET) continue;
		const S gv = potValue<S, D>(dom, FR, fc);
		if (gv == S(0)) continue;
		dv -= alphaAt<S, D>(dom, c.mi, f >> 1) * gv;
	}
	rhs[c.g] = dv;
	}
}

// k_computeEpotRHS (mhd/potential.cu:273-323) of a given in-plane field [inst][dims][cells]
template <typename S, int D>
__global__ void __launch_bounds__(PHB_TILE) kEpotRhs(Dom<S, D> dom, const S *__restrict__ field, S *__restrict__ rhs) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	S fl[2 * D];
#pragma unroll
	for (int dim = 0; dim < D; ++dim) {
		const S velC = contraAt<S, D>(dom, c.B, c.g, c.mi, dim, field);
#pragma unroll
		for (int up = 0; up < 2; ++up) {
			const int f = dim * 2 + up;
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) {
				const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
				const int bc = potBC(dom.fmask, FR, faceCell(c.B, f, c.p));
				fl[f] = (bc == PB_INSULATING || bc == PB_THIN_WALL) ? S(0) : velC;
			} else {
				const Nbr n = neighbor<S, D>(dom, c, f);
				S velN = contraAt<S, D>(dom, n.B, n.g, n.mi, n.comp, field);
				if (n.flip) velN = -velN;
				fl[f] = (velN + velC) * S(0.5);
			}
		}
	}
	S dv = 0;
#pragma unroll
	for (int d = 0; d < D; ++d) dv += fl[d * 2 + 1] - fl[d * 2];
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		if (!atBound(c.B, f, c.p) || fType(c.B, f) != FT_FIXED) continue;
		const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
		const int fc = faceCell(c.B, f, c.p);
		if (potBC(dom.fmask, FR, fc) != PB_DIRICHLET) continue;
		const S gv = potValue<S, D>(dom, FR, fc);
		if (gv == S(0)) continue;
		dv -= alphaAt<S, D>(dom, c.mi, f >> 1) * gv;
	}
	rhs[c.g] = dv;
	}
}

// computeCurrentDensityFaceBased (mhd/potential.cu:718-880) fused with the Lorentz force
// F_L = N (J x e_b) of simulation/mhd.py:543-595 added to the velocity source
template <typename S, int D>
__global__ void __launch_bounds__(PHB_TILE) kCurrentLorentz(Dom<S, D> dom, const S *__restrict__ phi, const S *__restrict__ uxb,
		const double *__restrict__ eb, const double *__restrict__ stuart, S *__restrict__ Jout, S *__restrict__ src, int accumulate) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	const int inst = c.B[B_INST];
	const S phiP = phi[c.g];
	S alphaP[D], cvelP[D];
	S xP[D];
#pragma unroll
	for (int k = 0; k < D; ++k) xP[k] = uxb[vidx3(c.B, c.g, k)];
#pragma unroll
	for (int d = 0; d < D; ++d) { alphaP[d] = alphaAt<S, D>(dom, c.mi, d); cvelP[d] = contraVec<S, D>(dom, c.mi, d, xP); }
	S jf[2 * D];
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		const int dim = f >> 1;
		const S faceSign = (f & 1) ? S(1) : S(-1);
		const bool ab = atBound(c.B, f, c.p);
		if (ab && fType(c.B, f) == FT_FIXED) {
			const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
			const int fc = faceCell(c.B, f, c.p);
			const int bc = potBC(dom.fmask, FR, fc);
			if (bc == PB_INSULATING || bc == PB_THIN_WALL) jf[f] = 0;
			else if (bc == PB_DIRICHLET) jf[f] = alphaP[dim] * faceSign * (phiP - potValue<S, D>(dom, FR, fc)) + cvelP[dim];
			else jf[f] = cvelP[dim];
			continue;
		}
		const Nbr n = neighbor<S, D>(dom, c, f);
		const S phiN = phi[n.g];
		const S alphaN = alphaAt<S, D>(dom, n.mi, n.comp);
		S xN[D];
#pragma unroll
		for (int k = 0; k < D; ++k) xN[k] = uxb[vidx3(n.B, n.g, k)];
		S cvelN = contraVec<S, D>(dom, n.mi, n.comp, xN);
		if (n.flip) cvelN = -cvelN;
		const S coeff = S(0.5) * (alphaP[dim] + alphaN);
		const S chi = S(0.5) * (cvelP[dim] + cvelN);
		jf[f] = -coeff * faceSign * (phiN - phiP) + chi;
	}
	S javg[D];
#pragma unroll
	for (int d = 0; d < D; ++d) javg[d] = S(0.5) * (jf[d * 2] + jf[d * 2 + 1]);
	const S invDet = S(1) / detAt<S, D>(dom, c.mi);
	S J[3] = {0, 0, 0};
#pragma unroll
	for (int r = 0; r < D; ++r) {
		S s = 0;
#pragma unroll
		for (int k = 0; k < D; ++k) s += dom.m(r * D + k, c.mi) * javg[k];
		J[r] = s * invDet;
	}
	if (D == 2) J[2] = uxb[vidx3(c.B, c.g, 2)];
	if (Jout) {
#pragma unroll
		for (int k = 0; k < 3; ++k) Jout[vidx3(c.B, c.g, k)] = J[k];
	}
	if (src) {
		const double *e = eb + 3 * inst;
		const S N = S(stuart[inst]);
		const S e0 = S(e[0]), e1 = S(e[1]), e2 = S(e[2]);
		const S F[3] = {J[1] * e2 - J[2] * e1, J[2] * e0 - J[0] * e2, J[0] * e1 - J[1] * e0};
#pragma unroll
		for (int d = 0; d < D; ++d) {
			const int64_t o = vidx<D>(c.B, c.g, d);
			const S v = N * F[d];
			src[o] = accumulate ? v + src[o] : v;
		}
	}
	}
}

// The explicit non-orthogonal terms of a result field applied to a right-hand side
// (nonortho_rhs.cuh:27-180): the velocity (advection.cu:936-937) and scalar
// (advection.cu:684-689) right-hand sides lose S / det (the scalar's times its diffusivity),
// the pressure divergence gains S weighted with 1/A (pressure.cu:839-860).
template <typename S, int D, int KIND>
__global__ void __launch_bounds__(PHB_TILE) kNonOrthoRhs(Dom<S, D> dom, const S *__restrict__ field, ScalarView sv,
		const S *__restrict__ Adiag, S *__restrict__ rhs) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	const int blk = __ldg(dom.tiles + 2 * blockIdx.x);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	const BPos bp{blk, {c.p[0], c.p[1], c.p[2]}};
	const int inst = c.B[B_INST];
	if (innerCell<D>(c.B, c.p)) {
		// away from the block's faces: all components at once from the fixed strides
		if constexpr (KIND == PHB_NONORTHO_PRESSURE) {
			S o[1];
			nonOrthoRhsInner<S, D, 1>(dom, field, 0, 0, c.B, c.p, dom.nonortho, [&](int64_t g) { return S(1) / Adiag[g]; }, o);
			rhs[c.g] += o[0];
		} else if constexpr (KIND == PHB_NONORTHO_VELOCITY) {
			const S nu = S(dom.nu[inst]);
			const S det = detAt<S, D>(dom, c.mi);
			S o[D];
			nonOrthoRhsInner<S, D, D>(dom, field, vidx<D>(c.B, 0, 0), c.B[B_INSTN], c.B, c.p, dom.nonortho,
				[&](int64_t) { return nu; }, o);
#pragma unroll
			for (int w = 0; w < D; ++w) rhs[vidx<D>(c.B, c.g, w)] -= o[w] / det;
		} else {
			const S det = detAt<S, D>(dom, c.mi);
			for (int ch = 0; ch < sv.channels; ++ch) {
				S o[1];
				nonOrthoRhsInner<S, D, 1>(dom, field, sidx(c.B, 0, ch, sv.channels), 0, c.B, c.p, dom.nonortho,
					[&](int64_t) { return S(1); }, o);
				const S nuc = S(scalarNu(sv, ch, dom.nu[inst]));
				rhs[sidx(c.B, c.g, ch, sv.channels)] -= o[0] * nuc / det;
			}
		}
		continue;
	}
	if constexpr (KIND == PHB_NONORTHO_PRESSURE) {
		const NField<S> F{NF_PRESSURE, 0, field, sv};
		S o[1];
		nonOrthoRhs<S, D, 1>(dom, F, bp, dom.nonortho, [&](int64_t g) { return S(1) / Adiag[g]; }, S(1), o);
		rhs[c.g] += o[0];
	} else if constexpr (KIND == PHB_NONORTHO_VELOCITY) {
		// one walk per corner for all components (they share the faces' velocity type)
		const S nu = S(dom.nu[inst]);
		const S det = detAt<S, D>(dom, c.mi);
		const NField<S> F{NF_VELOCITY, 0, field, sv};
		S o[D];
		nonOrthoRhs<S, D, D>(dom, F, bp, dom.nonortho, [&](int64_t) { return nu; }, nu, o);
#pragma unroll
		for (int w = 0; w < D; ++w) rhs[vidx<D>(c.B, c.g, w)] -= o[w] / det;
	} else {
		const S det = detAt<S, D>(dom, c.mi);
		for (int ch = 0; ch < sv.channels; ++ch) {
			const S nuc = S(scalarNu(sv, ch, dom.nu[inst]));
			const NField<S> F{NF_SCALAR, ch, field, sv};
			S o[1];
			nonOrthoRhs<S, D, 1>(dom, F, bp, dom.nonortho, [&](int64_t) { return S(1); }, S(1), o);
			rhs[sidx(c.B, c.g, ch, sv.channels)] -= o[0] * nuc / det;
		}
	}
	}
}

} // namespace phb

using namespace phb;

#define PHB_DISPATCH(DOM, ...)                                                                     \
	do {                                                                                           \
		if ((DOM)->dims == 2 && (DOM)->dtype == PHB_F64) { using S = double; constexpr int D = 2; __VA_ARGS__; } \
		else if ((DOM)->dims == 3 && (DOM)->dtype == PHB_F64) { using S = double; constexpr int D = 3; __VA_ARGS__; } \
		else if ((DOM)->dims == 2 && (DOM)->dtype == PHB_F32) { using S = float; constexpr int D = 2; __VA_ARGS__; } \
		else if ((DOM)->dims == 3 && (DOM)->dtype == PHB_F32) { using S = float; constexpr int D = 3; __VA_ARGS__; } \
		else return setError(PHB_ERR_ARG, "unsupported dims/dtype");                                \
	} while (0)

#define PHB_TILES(DOM) dim3((DOM)->ntiles), dim3(PHB_TILE), 0, (cudaStream_t)stream

// The device view of a launch whose quad kernels may use vector loads: every field operand
// on a 16-byte boundary with a cell count that keeps the component rows aligned (vec4), and
// the metric rows aligned (metal).
template <typename S, int D>
static Dom<S, D> quadView(const phb_domain *dom, std::initializer_list<const void *> fields) {
	Dom<S, D> dm(*dom);
	int ok = dom->ncells % 4 == 0;
	for (const void *p : fields)
		if (p && ((uintptr_t)p & 15)) ok = 0;
	dm.vec4 = ok;
	dm.metal = ((uintptr_t)dom->metrics & 15) == 0 && dom->metric_stride % 4 == 0;
	return dm;
}

extern "C" int phb_advection_matrix(const phb_domain *dom, const void *u, void *C, void *Adiag, float *C_lo, phb_stream stream) {
	if (!dom || !u || !C || !Adiag) return setError(PHB_ERR_ARG, "phb_advection_matrix: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	if (dom->dims > 1 && (dom->nonortho & NO_MATRIX_BITS)) {
		PHB_DISPATCH(dom, (kAdvectionMatrix<S, D, false, true><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)u, (S *)C, (S *)Adiag, C_lo)));
		return checkLaunch("kAdvectionMatrix<non-orthogonal>");
	}
	PHB_DISPATCH(dom, kAdvectionMatrix<S, D><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)u, (S *)C, (S *)Adiag, C_lo));
	return checkLaunch("kAdvectionMatrix");
}
extern "C" int phb_scalar_matrix(const phb_domain *dom, const void *u, const phb_scalar *sc, int channel, void *C, void *Adiag,
		float *C_lo, phb_stream stream) {
	if (!dom || !u || !sc || !C || !Adiag) return setError(PHB_ERR_ARG, "phb_scalar_matrix: null argument");
	if (sc->channels < 1 || channel < 0 || channel >= sc->channels || (sc->nu_count != 0 && sc->nu_count != 1 && sc->nu_count != sc->channels) ||
			(sc->nu_count > 0 && !sc->nu) || (dom->nfixed > 0 && (!sc->types || !sc->values || !sc->offsets || !sc->statics)))
		return setError(PHB_ERR_ARG, "phb_scalar_matrix: bad scalar description");
	if (dom->ntiles == 0) return PHB_OK;
	const ScalarView sv = scalarView(sc);
	if (dom->dims > 1 && (dom->nonortho & NO_MATRIX_BITS)) {
		PHB_DISPATCH(dom, (kAdvectionMatrix<S, D, true, true><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)u, (S *)C, (S *)Adiag, C_lo, sv,
			channel)));
		return checkLaunch("kAdvectionMatrix<scalar, non-orthogonal>");
	}
	PHB_DISPATCH(dom, kAdvectionMatrix<S, D, true><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)u, (S *)C, (S *)Adiag, C_lo, sv, channel));
	return checkLaunch("kAdvectionMatrix<scalar>");
}
extern "C" int phb_scalar_rhs(const phb_domain *dom, const void *phi, const void *u, const phb_scalar *sc, void *rhs, phb_stream stream) {
	if (!dom || !phi || !sc || !rhs || (dom->scheme != 0 && !u)) return setError(PHB_ERR_ARG, "phb_scalar_rhs: null argument");
	if (sc->channels < 1 || (sc->nu_count != 0 && sc->nu_count != 1 && sc->nu_count != sc->channels) || (sc->nu_count > 0 && !sc->nu) ||
			(dom->nfixed > 0 && (!sc->types || !sc->values || !sc->offsets || !sc->statics)))
		return setError(PHB_ERR_ARG, "phb_scalar_rhs: bad scalar description");
	if (dom->ntiles == 0) return PHB_OK;
	const ScalarView sv = scalarView(sc);
	PHB_DISPATCH(dom, kScalarRhs<S, D><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)phi, (const S *)u, sv, (S *)rhs));
	return checkLaunch("kScalarRhs");
}
extern "C" int phb_advection_rhs(const phb_domain *dom, const void *u, const void *src, int src_mode, void *rhs, phb_stream stream) {
	if (!dom || !u || !rhs || (src_mode != 0 && !src) || src_mode < 0 || src_mode > 2) return setError(PHB_ERR_ARG, "phb_advection_rhs: bad argument");
	if (dom->ntiles == 0) return PHB_OK;
	if (dom->scheme != 0)
		PHB_DISPATCH(dom, (kAdvectionRhs<S, D, true><<<PHB_TILES(dom)>>>(quadView<S, D>(dom, {u, src, rhs}), (const S *)u, (const S *)src,
			src_mode, (S *)rhs)));
	else
		PHB_DISPATCH(dom, (kAdvectionRhs<S, D, false><<<PHB_TILES(dom)>>>(quadView<S, D>(dom, {u, src, rhs}), (const S *)u, (const S *)src,
			src_mode, (S *)rhs)));
	return checkLaunch("kAdvectionRhs");
}
extern "C" int phb_pressure_matrix(const phb_domain *dom, const void *Adiag, void *P, float *P_lo, phb_stream stream) {
	if (!dom || !Adiag || !P) return setError(PHB_ERR_ARG, "phb_pressure_matrix: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	if (dom->dims > 1 && (dom->nonortho & NO_MATRIX_BITS)) {
		PHB_DISPATCH(dom, (kLaplaceMatrix<S, D, false, true><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)Adiag, (S *)P, P_lo)));
		return checkLaunch("kLaplaceMatrix<non-orthogonal>");
	}
	PHB_DISPATCH(dom, (kLaplaceMatrix<S, D, false><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)Adiag, (S *)P, P_lo)));
	return checkLaunch("kLaplaceMatrix");
}
extern "C" int phb_epot_matrix(const phb_domain *dom, void *E, float *E_lo, phb_stream stream) {
	if (!dom || !E) return setError(PHB_ERR_ARG, "phb_epot_matrix: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	PHB_DISPATCH(dom, (kLaplaceMatrix<S, D, true><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)nullptr, (S *)E, E_lo)));
	return checkLaunch("kLaplaceMatrix(epot)");
}
extern "C" int phb_pressure_rhs(const phb_domain *dom, const void *C, const void *Adiag, const void *u, const void *ustar,
		const void *src, int src_mode, void *hbya, phb_stream stream) {
	if (!dom || !C || !Adiag || !u || !ustar || !hbya || (src_mode != 0 && !src) || src_mode < 0 || src_mode > 2)
		return setError(PHB_ERR_ARG, "phb_pressure_rhs: bad argument");
	if (dom->ntiles == 0) return PHB_OK;
	if (dom->scheme != 0)
		PHB_DISPATCH(dom, (kPressureRhs<S, D, true><<<PHB_TILES(dom)>>>(quadView<S, D>(dom, {C, Adiag, u, ustar, src, hbya}),
			(const S *)C, (const S *)Adiag, (const S *)u, (const S *)ustar, (const S *)src, src_mode, (S *)hbya)));
	else
		PHB_DISPATCH(dom, (kPressureRhs<S, D, false><<<PHB_TILES(dom)>>>(quadView<S, D>(dom, {C, Adiag, u, ustar, src, hbya}),
			(const S *)C, (const S *)Adiag, (const S *)u, (const S *)ustar, (const S *)src, src_mode, (S *)hbya)));
	return checkLaunch("kPressureRhs");
}
extern "C" int phb_divergence(const phb_domain *dom, const void *field, void *div, phb_stream stream) {
	if (!dom || !field || !div) return setError(PHB_ERR_ARG, "phb_divergence: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	PHB_DISPATCH(dom, kDivergence<S, D><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)field, (S *)div));
	return checkLaunch("kDivergence");
}
extern "C" int phb_correct_velocity(const phb_domain *dom, const void *p, const void *hbya, const void *Adiag, void *u, phb_stream stream) {
	if (!dom || !p || !hbya || !Adiag || !u) return setError(PHB_ERR_ARG, "phb_correct_velocity: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	PHB_DISPATCH(dom, kCorrectVelocity<S, D><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)p, (const S *)hbya, (const S *)Adiag, (S *)u));
	return checkLaunch("kCorrectVelocity");
}
extern "C" int phb_uxb_epot_rhs(const phb_domain *dom, const void *u, const double *e_b, void *uxb, void *rhs, phb_stream stream) {
	if (!dom || !u || !e_b || !uxb || !rhs) return setError(PHB_ERR_ARG, "phb_uxb_epot_rhs: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	PHB_DISPATCH(dom, kUxbEpotRhs<S, D><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)u, e_b, (S *)uxb, (S *)rhs));
	return checkLaunch("kUxbEpotRhs");
}
extern "C" int phb_current_lorentz(const phb_domain *dom, const void *phi, const void *uxb, const double *e_b,
		const double *stuart, void *J, void *src, int accumulate, phb_stream stream) {
	if (!dom || !phi || !uxb || !e_b || (src && !stuart)) return setError(PHB_ERR_ARG, "phb_current_lorentz: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	PHB_DISPATCH(dom, kCurrentLorentz<S, D><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)phi, (const S *)uxb, e_b, stuart,
		(S *)J, (S *)src, accumulate));
	return checkLaunch("kCurrentLorentz");
}
extern "C" int phb_epot_rhs(const phb_domain *dom, const void *field, void *rhs, phb_stream stream) {
	if (!dom || !field || !rhs) return setError(PHB_ERR_ARG, "phb_epot_rhs: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	PHB_DISPATCH(dom, kEpotRhs<S, D><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)field, (S *)rhs));
	return checkLaunch("kEpotRhs");
}
extern "C" int phb_nonortho_rhs(const phb_domain *dom, int kind, const void *field, const phb_scalar *sc, const void *Adiag,
		void *rhs, phb_stream stream) {
	if (!dom || !field || !rhs || kind < PHB_NONORTHO_VELOCITY || kind > PHB_NONORTHO_PRESSURE ||
			(kind == PHB_NONORTHO_PRESSURE && !Adiag))
		return setError(PHB_ERR_ARG, "phb_nonortho_rhs: bad argument");
	if (kind == PHB_NONORTHO_SCALAR && (!sc || sc->channels < 1 || (sc->nu_count != 0 && sc->nu_count != 1 && sc->nu_count != sc->channels) ||
			(sc->nu_count > 0 && !sc->nu) || (dom->nfixed > 0 && (!sc->types || !sc->values || !sc->offsets || !sc->statics))))
		return setError(PHB_ERR_ARG, "phb_nonortho_rhs: bad scalar description");
	if (dom->ntiles == 0 || dom->dims < 2 || !(dom->nonortho & NO_RHS_BITS)) return PHB_OK;
	const ScalarView sv = scalarView(kind == PHB_NONORTHO_SCALAR ? sc : nullptr);
	if (kind == PHB_NONORTHO_PRESSURE)
		PHB_DISPATCH(dom, (kNonOrthoRhs<S, D, PHB_NONORTHO_PRESSURE><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)field, sv,
			(const S *)Adiag, (S *)rhs)));
	else if (kind == PHB_NONORTHO_VELOCITY)
		PHB_DISPATCH(dom, (kNonOrthoRhs<S, D, PHB_NONORTHO_VELOCITY><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)field, sv,
			(const S *)Adiag, (S *)rhs)));
	else
		PHB_DISPATCH(dom, (kNonOrthoRhs<S, D, PHB_NONORTHO_SCALAR><<<PHB_TILES(dom)>>>(Dom<S, D>(*dom), (const S *)field, sv,
			(const S *)Adiag, (S *)rhs)));
	return checkLaunch("kNonOrthoRhs");
}
