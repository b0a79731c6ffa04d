// Adjoint (reverse-mode) kernels of the PISO/MHD step: the transposes of the assembly
// kernels (phiPICT's *Grad kernels, piso/advection.cu:310-544,958-1195, pressure.cu:196-345,
// 525-750, velocity_correction.cu:301-375, mhd/potential.cu:981-1329) and the pieces of the
// adjoint linear solves (phiPICT's LinearSolveFunction and SparseOuterProduct,
// core/piso_diff.py:1154-1421).
//
// Each kernel mirrors one forward kernel of assembly.cu line by line in reverse: a thread
// takes one cell, recomputes the forward intermediates it needs, and accumulates the
// vector-Jacobian product into the adjoints of its inputs. Inputs shared with neighbouring
// cells (face fluxes, neighbour values) are scattered with FP64 atomics, so every adjoint
// output is accumulated (+=) and must be zeroed by the caller before the first
// contribution. The kernels run in FP64.
#include "phb_device.cuh"
#include "phb_launch.cuh"
#include "phb_upwind.cuh"

namespace phb {

using S = double;

__device__ __forceinline__ void aadd(double *p, double v) {
	if (v != 0.0) atomicAdd(p, v);
}

// d/d(field) of contraAt(B, g, mi, c, field): field[vidx(B, g, j)] += det Minv[c][j] * vbar
template <int D>
__device__ __forceinline__ void adjContra(const Dom<S, D> &dom, const int32_t *B, int64_t g, int64_t mi, int c, S vbar, S *fbar) {
	if (vbar == 0.0) return;
	const S det = dom.m(Tr<D>::DET, mi);
#pragma unroll
	for (int j = 0; j < D; ++j) aadd(fbar + vidx<D>(B, g, j), det * dom.m(Tr<D>::MINV + c * D + j, mi) * vbar);
}
// the same for a 3-component field (u x e_b); only the first D components enter
template <int D>
__device__ __forceinline__ void adjContra3(const Dom<S, D> &dom, const int32_t *B, int64_t g, int64_t mi, int c, S vbar, S *xbar) {
	if (vbar == 0.0) return;
	const S det = dom.m(Tr<D>::DET, mi);
#pragma unroll
	for (int j = 0; j < D; ++j) aadd(xbar + vidx3(B, g, j), det * dom.m(Tr<D>::MINV + c * D + j, mi) * vbar);
}
// boundary velocity adjoint: the same layout as the fixed-face velocity buffer
template <int D>
__device__ __forceinline__ S *fixedVelBar(const int32_t *FR, int fc, int k, S *ubbar) {
	return FR[F_VELSTATIC] ? ubbar + FR[F_VELOFF] + k : ubbar + FR[F_VELOFF] + k * FR[F_FACECELLS] + fc;
}
// d/d(u_b) of contraFixed(FR, fc, c) (zero on Neumann faces)
template <int D>
__device__ __forceinline__ void adjContraFixed(const Dom<S, D> &dom, const int32_t *FR, int fc, int c, S vbar, S *ubbar) {
	if (FR[F_VELTYPE] != 0 || vbar == 0.0 || !ubbar) return;
	const int64_t fi = FR[F_TOFF] + fc;
	const S det = dom.fm(Tr<D>::DET, fi);
#pragma unroll
	for (int j = 0; j < D; ++j) aadd(fixedVelBar<D>(FR, fc, j, ubbar), det * dom.fm(Tr<D>::MINV + c * D + j, fi) * vbar);
}

// faceFluxes adjoint: flBar[f] (cotangent of the face flux fl[f] of cell c) -> the field
// (ubar) and, on fixed faces, the boundary velocity (ubbar)
template <int D>
__device__ __forceinline__ void adjFaceFluxes(const Dom<S, D> &dom, const Cell &c, const S (&flBar)[2 * D], S *ubar, S *ubbar) {
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		if (flBar[f] == 0.0) continue;
		const int dim = f >> 1;
		if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) {
			adjContraFixed<D>(dom, dom.fix(fRec(c.B, f)[5]), faceCell(c.B, f, c.p), dim, flBar[f], ubbar);
		} else {
			adjContra<D>(dom, c.B, c.g, c.mi, dim, S(0.5) * flBar[f], ubar);
			const Nbr n = neighbor<S, D>(dom, c, f);
			adjContra<D>(dom, n.B, n.g, n.mi, n.comp, n.flip ? -S(0.5) * flBar[f] : S(0.5) * flBar[f], ubar);
		}
	}
}

// upwindCorrection adjoint for one field value(g) at cell c with the fluxes fl: rb is the
// cotangent of r; the field's cotangent goes to vbar(g), the fluxes' to flBar. As phiPICT's
// adjoint of the deferred correction (piso/advection.cu:1049-1063), the correction is taken
// as its linear form -F/2 (phi_U - phi_UU) with the upwind branch and the skip of a vanishing
// phi_D - phi_U frozen.
template <int D, typename Val, typename VBar>
__device__ __forceinline__ void adjUpwindCorrection(const Cell &c, const S (&fl)[2 * D], Val value, VBar vbar, S rb,
		S (&flBar)[2 * D]) {
	if (rb == 0.0) return;
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		const int ax = f >> 1;
		const int sign = (f & 1) ? 1 : -1;
		const S fout = S(sign) * fl[f];
		const bool outflow = fout >= S(0);
		if (!farUpwind(c.B, c.p, f, outflow)) continue;
		int64_t step = 1;
		if (ax >= 1) step *= c.B[B_NX];
		if (ax >= 2) step *= c.B[B_NY];
		const int64_t gN = c.g + sign * step;
		const int64_t gUU = outflow ? c.g - sign * step : c.g + 2 * sign * step;
		const int64_t gU = outflow ? c.g : gN;
		const S phiP = value(c.g), phiN = value(gN), phiUU = value(gUU);
		const S phiU = outflow ? phiP : phiN;
		const S phiD = outflow ? phiN : phiP;
		const S dD = phiD - phiU;
		if ((dD < S(0) ? -dD : dD) < S(1e-20)) continue;
		// r -= fout/2 (phi_U - phi_UU)
		vbar(gU, -S(0.5) * fout * rb);
		vbar(gUU, S(0.5) * fout * rb);
		flBar[f] += S(sign) * (-S(0.5) * (phiU - phiUU) * rb);
	}
}

// --- linear-solve pieces -------------------------------------------------------------------
// C^T as a stencil: slot f of cell i holds C[j][f'] where j is the neighbour across f and f'
// the face of j that leads back to i (the opposite face, or the entry face of a connection).
template <int D, typename V = S>
__global__ void __launch_bounds__(PHB_TILE) kTransposeStencil(Dom<V, D> dom, const V *__restrict__ C, V *__restrict__ CT) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<V, D>(dom, sB, l0, nc);
	const int64_t N = dom.ncells;
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		CT[c.g] = C[c.g];
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) { CT[(f + 1) * N + c.g] = 0; continue; }
			const Nbr n = neighbor<V, D>(dom, c, f);
			int back = f ^ 1;
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_CONNECTED) {
				const int code = fRec(c.B, f)[2];
				back = 2 * (code >> 1) + (code & 1);
			}
			CT[(f + 1) * N + c.g] = C[(back + 1) * N + n.g];
		}
	}
}

// Mbar[s][i] += scale * sum_k lam[i,k] x[nb_s(i),k]: the adjoint of a solve M x = b with
// respect to the stencil values (nb_0 = i); K = components sharing the matrix
template <int D, int K>
__global__ void __launch_bounds__(PHB_TILE) kAdjOuter(Dom<S, D> dom, const S *__restrict__ lam, const S *__restrict__ x, S scale,
		S *__restrict__ Mbar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	const int64_t N = dom.ncells;
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		S lv[K];
		S d = 0;
#pragma unroll
		for (int k = 0; k < K; ++k) {
			const int64_t o = K == 1 ? (int64_t)c.g : vidx<D>(c.B, c.g, k);
			lv[k] = lam[o];
			d += lv[k] * x[o];
		}
		Mbar[c.g] += scale * d;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			const int64_t nb = neighborIndex<S, D>(dom, c, f);
			if (nb < 0) continue;
			S s = 0;
#pragma unroll
			for (int k = 0; k < K; ++k) s += lv[k] * x[K == 1 ? nb : vidx<D>(c.B, nb, k)];
			Mbar[(f + 1) * N + c.g] += scale * s;
		}
	}
}

// --- assembly adjoints ---------------------------------------------------------------------
// kAdvectionMatrix: Cbar (with the adjoint of Adiag already added to slot 0) -> ubar via the
// face fluxes F_f = (contra_P + contra_N)/2 (C depends on u only through them)
// With LINEAR_UPWIND an upwinded face puts all of s F on the diagonal (outflow) or on the
// face slot (inflow); the branch, taken from the fluxes of u, is frozen (advection.cu:380-400).
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjAdvectionMatrix(Dom<S, D> dom, const S *__restrict__ Cbar, const S *__restrict__ u,
		S *__restrict__ ubar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	const int64_t N = dom.ncells;
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const S det = detAt<S, D>(dom, c.mi);
		const S d0 = Cbar[c.g];
		S fl[2 * D];
		if (dom.scheme != 0) faceFluxes<S, D>(dom, c, u, fl);
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) continue;
			const S faceSign = (f & 1) ? S(1) : S(-1);
			// CENTRAL: diag += 0.5 s F / det, off_f += 0.5 s F / det
			S Fbar = S(0.5) * faceSign * (d0 + Cbar[(f + 1) * N + c.g]) / det;
			if (dom.scheme != 0) {
				const S fout = faceSign * fl[f];
				if (farUpwind(c.B, c.p, f, fout >= S(0))) Fbar = faceSign * (fout >= S(0) ? d0 : Cbar[(f + 1) * N + c.g]) / det;
			}
			// F = (velC + velN)/2
			adjContra<D>(dom, c.B, c.g, c.mi, f >> 1, S(0.5) * Fbar, ubar);
			const Nbr n = neighbor<S, D>(dom, c, f);
			adjContra<D>(dom, n.B, n.g, n.mi, n.comp, n.flip ? -S(0.5) * Fbar : S(0.5) * Fbar, ubar);
		}
	}
}

// boundarySource adjoint: Bbar[dim] (per component) -> the fixed-face velocities
template <int D>
__device__ __forceinline__ void adjBoundarySource(const Dom<S, D> &dom, const Cell &c, const S *Bbar, S nu, S *ubbar) {
	if (!ubbar) return;
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) {
		if (!atBound(c.B, f, c.p) || fType(c.B, f) != FT_FIXED) continue;
		const S faceNormal = (f & 1) ? S(1) : S(-1);
		const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
		const int fc = faceCell(c.B, f, c.p);
		const S alpha = alphaFixed<S, D>(dom, FR, fc, f >> 1);
		const S flux = contraFixed<S, D>(dom, FR, fc, f >> 1) * faceNormal;
		const S slip = FR[F_VELTYPE] == 0 ? S(0) : S(1);
		// B_d = sum_f -vel_d flux + vel_d (1 - slip) 2 nu alpha
		S fluxBar = 0;
#pragma unroll
		for (int d = 0; d < D; ++d) {
			const S vel = fixedVel<S, D>(dom, FR, fc, d);
			aadd(fixedVelBar<D>(FR, fc, d, ubbar), Bbar[d] * (-flux + (S(1) - slip) * nu * S(2) * alpha));
			fluxBar -= Bbar[d] * vel;
		}
		adjContraFixed<D>(dom, FR, fc, f >> 1, fluxBar * faceNormal, ubbar);
	}
}

// The deferred LINEAR_UPWIND correction of every velocity component at cell c (advection
// and HbyA right-hand sides): Bbar[d] is the cotangent of the component's correction sum
// (before the division by det) -> ubar through the values and the fluxes of u.
template <int D>
__device__ __forceinline__ void adjUpwindTerms(const Dom<S, D> &dom, const Cell &c, const S *u, const S (&Bbar)[D], S *ubar,
		S *ubbar) {
	S fl[2 * D], flBar[2 * D];
	faceFluxes<S, D>(dom, c, u, fl);
#pragma unroll
	for (int f = 0; f < 2 * D; ++f) flBar[f] = 0;
#pragma unroll
	for (int d = 0; d < D; ++d)
		adjUpwindCorrection<D>(c, fl, [&](int64_t g) { return u[vidx<D>(c.B, g, d)]; },
				[&](int64_t g, S v) { aadd(ubar + vidx<D>(c.B, g, d), v); }, Bbar[d], flBar);
	adjFaceFluxes<D>(dom, c, flBar, ubar, ubbar);
}

// kAdvectionRhs: rhs_d = u_d/dt + B_d/det + S_d
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjAdvectionRhs(Dom<S, D> dom, const S *__restrict__ rhsbar, const S *__restrict__ u,
		S *__restrict__ ubar, S *__restrict__ srcbar, S *__restrict__ ubbar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const int inst = c.B[B_INST];
		const S dt = dom.dt[inst], nu = dom.nu[inst];
		const S det = detAt<S, D>(dom, c.mi);
		S Bbar[D];
#pragma unroll
		for (int d = 0; d < D; ++d) {
			const int64_t o = vidx<D>(c.B, c.g, d);
			const S r = rhsbar[o];
			aadd(ubar + o, r / dt); // atomically: the upwind terms of other cells add here too
			if (srcbar) srcbar[o] += r;
			Bbar[d] = r / det;
		}
		adjBoundarySource<D>(dom, c, Bbar, nu, ubbar);
		if (dom.scheme != 0) adjUpwindTerms<D>(dom, c, u, Bbar, ubar, ubbar);
	}
}

// kScalarRhs (CENTRAL): rhs_c = (det phi_c/dt + sum over fixed faces of the face terms)/det;
// Dirichlet faces: -v flux + v nu 2 alpha; Neumann-type faces: -phi flux + v nu area
// (advection.cu:545-698). rhsbar -> phibar, the fixed-face scalar values (valuesbar, the
// layout of phb_scalar::values) and the fixed-face velocities through the flux (ubbar).
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjScalarRhs(Dom<S, D> dom, ScalarView sv, const S *__restrict__ phi,
		const S *__restrict__ u, const S *__restrict__ rhsbar, S *__restrict__ phibar, S *__restrict__ valuesbar,
		S *__restrict__ ubar, S *__restrict__ ubbar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const int inst = c.B[B_INST];
		const S dt = dom.dt[inst];
		const double nuVel = dom.nu[inst];
		const S det = detAt<S, D>(dom, c.mi);
		S fl[2 * D], flBar[2 * D];
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) flBar[f] = 0;
		if (dom.scheme != 0) faceFluxes<S, D>(dom, c, u, fl);
		for (int ch = 0; ch < sv.channels; ++ch) {
			const int64_t o = sidx(c.B, c.g, ch, sv.channels);
			const S rb = rhsbar[o] / det; // cotangent of r (rhs = r / det)
			if (rb == 0.0) continue;
			if (dom.scheme != 0) // the deferred LINEAR_UPWIND correction of the channel
				adjUpwindCorrection<D>(c, fl, [&](int64_t g) { return phi[sidx(c.B, g, ch, sv.channels)]; },
						[&](int64_t g, S v) { aadd(phibar + sidx(c.B, g, ch, sv.channels), v); }, rb, flBar);
			const S nu = S(scalarNu(sv, ch, nuVel));
			S pb = rb * det / dt;
#pragma unroll
			for (int f = 0; f < 2 * D; ++f) {
				if (!atBound(c.B, f, c.p) || fType(c.B, f) != FT_FIXED) continue;
				const S faceNormal = (f & 1) ? S(1) : S(-1);
				const int fid = fRec(c.B, f)[5];
				const int32_t *FR = dom.fix(fid);
				const int fc = faceCell(c.B, f, c.p);
				const int64_t vo = sv.offsets[fid] + (sv.statics[fid] ? ch : (int64_t)ch * FR[F_FACECELLS] + fc);
				const S value = ((const S *)sv.values)[vo];
				const S flux = contraFixed<S, D>(dom, FR, fc, f >> 1) * faceNormal;
				S fluxBar;
				if (sv.types[(int64_t)fid * sv.channels + ch] == 0) {
					if (valuesbar) aadd(valuesbar + vo, rb * (-flux + nu * S(2) * alphaFixed<S, D>(dom, FR, fc, f >> 1)));
					fluxBar = -rb * value;
				} else {
					const int64_t fi = FR[F_TOFF] + fc;
					S m2 = 0;
#pragma unroll
					for (int k = 0; k < D; ++k) { const S v = dom.fm(Tr<D>::MINV + (f >> 1) * D + k, fi); m2 += v * v; }
					const S area = dom.fm(Tr<D>::DET, fi) * sqrt(m2);
					if (valuesbar) aadd(valuesbar + vo, rb * nu * area);
					pb -= rb * flux;
					fluxBar = -rb * phi[o];
				}
				adjContraFixed<D>(dom, FR, fc, f >> 1, fluxBar * faceNormal, ubbar);
			}
			aadd(phibar + o, pb);
		}
		if (dom.scheme != 0) adjFaceFluxes<D>(dom, c, flBar, ubar, ubbar);
	}
}

// kPressureRhs: h_d = (u_d/dt - sum_f C_f ustar_{j,d} + B_d/det + S_d) / A
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjPressureRhs(Dom<S, D> dom, const S *__restrict__ C, const S *__restrict__ Adiag,
		const S *__restrict__ u, const S *__restrict__ ustar, const S *__restrict__ h, const S *__restrict__ hbar, S *__restrict__ ubar,
		S *__restrict__ ustarbar, S *__restrict__ Cbar, S *__restrict__ Abar, S *__restrict__ srcbar, S *__restrict__ ubbar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	const int64_t N = dom.ncells;
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const int inst = c.B[B_INST];
		const S dt = dom.dt[inst], nu = dom.nu[inst];
		const S rD = S(1) / Adiag[c.g];
		const S det = detAt<S, D>(dom, c.mi);
		S qbar[D], Bbar[D], aAcc = 0;
#pragma unroll
		for (int d = 0; d < D; ++d) {
			const int64_t o = vidx<D>(c.B, c.g, d);
			qbar[d] = hbar[o] * rD;
			aAcc -= hbar[o] * h[o] * rD;
			aadd(ubar + o, qbar[d] / dt); // atomically: the upwind terms of other cells add here too
			if (srcbar) srcbar[o] += qbar[d];
			Bbar[d] = qbar[d] / det;
		}
		Abar[c.g] += aAcc;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			const int64_t nb = neighborIndex<S, D>(dom, c, f);
			if (nb < 0 || nb == c.g) continue;
			const S cv = C[(f + 1) * N + c.g];
			S s = 0;
#pragma unroll
			for (int d = 0; d < D; ++d) {
				const int64_t on = vidx<D>(c.B, nb, d);
				s -= qbar[d] * ustar[on];
				aadd(ustarbar + on, -cv * qbar[d]);
			}
			Cbar[(f + 1) * N + c.g] += s;
		}
		adjBoundarySource<D>(dom, c, Bbar, nu, ubbar);
		// HbyA repeats the predictor's deferred correction of u (pressure.cu:474-515)
		if (dom.scheme != 0) adjUpwindTerms<D>(dom, c, u, Bbar, ubar, ubbar);
	}
}

// kDivergence of a [dims] field with fixed faces on the boundary velocity
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjDivergence(Dom<S, D> dom, const S *__restrict__ dbar, S *__restrict__ fbar,
		S *__restrict__ ubbar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const S db = dbar[c.g];
		if (db == 0.0) continue;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			const int dim = f >> 1;
			const S flb = ((f & 1) ? S(1) : S(-1)) * db;
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) {
				const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
				adjContraFixed<D>(dom, FR, faceCell(c.B, f, c.p), dim, flb, ubbar);
				continue;
			}
			adjContra<D>(dom, c.B, c.g, c.mi, dim, S(0.5) * flb, fbar);
			const Nbr n = neighbor<S, D>(dom, c, f);
			adjContra<D>(dom, n.B, n.g, n.mi, n.comp, n.flip ? -S(0.5) * flb : S(0.5) * flb, fbar);
		}
	}
}

template <int D>
__device__ __forceinline__ int64_t acrossIndex(const Dom<S, D> &dom, const Cell &c, int f) {
	if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) return c.g;
	return neighbor<S, D>(dom, c, f).g;
}

// kCorrectVelocity: u_d = -grad_d / A + h_d, grad = Minv^T gr, gr_r = fac (p_up - p_low)
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjCorrectVelocity(Dom<S, D> dom, const S *__restrict__ p, const S *__restrict__ Adiag,
		const S *__restrict__ ubar, S *__restrict__ hbar, S *__restrict__ pbar, S *__restrict__ Abar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const S rD = S(1) / Adiag[c.g];
		S fac[D], gr[D];
		int64_t up[D], low[D];
#pragma unroll
		for (int dim = 0; dim < D; ++dim) {
			const bool lowFixed = c.p[dim] == 0 && fType(c.B, dim * 2) == FT_FIXED;
			const bool upFixed = c.p[dim] == c.B[B_NX + dim] - 1 && fType(c.B, dim * 2 + 1) == FT_FIXED;
			fac[dim] = (lowFixed || upFixed) ? S(1) : S(0.5);
			low[dim] = lowFixed ? (int64_t)c.g : acrossIndex<D>(dom, c, dim * 2);
			up[dim] = upFixed ? (int64_t)c.g : acrossIndex<D>(dom, c, dim * 2 + 1);
			gr[dim] = (p[up[dim]] - p[low[dim]]) * fac[dim];
		}
		S gradbar[D], aAcc = 0;
#pragma unroll
		for (int d = 0; d < D; ++d) {
			const int64_t o = vidx<D>(c.B, c.g, d);
			const S ub = ubar[o];
			hbar[o] += ub;
			gradbar[d] = -rD * ub;
			S grad = 0;
#pragma unroll
			for (int r = 0; r < D; ++r) grad += dom.m(Tr<D>::MINV + r * D + d, c.mi) * gr[r];
			aAcc += ub * grad * rD * rD;
		}
		Abar[c.g] += aAcc;
#pragma unroll
		for (int r = 0; r < D; ++r) {
			S g = 0;
#pragma unroll
			for (int k = 0; k < D; ++k) g += dom.m(Tr<D>::MINV + r * D + k, c.mi) * gradbar[k];
			g *= fac[r];
			aadd(pbar + up[r], g);
			aadd(pbar + low[r], -g);
		}
	}
}

// kLaplaceMatrix (pressure): off_f = (alpha_P/A_P + alpha_N/A_N)/2, diag = -sum off_f
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjPressureMatrix(Dom<S, D> dom, const S *__restrict__ Adiag, const S *__restrict__ Pbar,
		S *__restrict__ Abar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	const int64_t N = dom.ncells;
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const S AP = Adiag[c.g];
		const S d0 = Pbar[c.g];
		S own = 0;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) continue;
			const S w = Pbar[(f + 1) * N + c.g] - d0;
			own += w * S(-0.5) * alphaAt<S, D>(dom, c.mi, f >> 1) / (AP * AP);
			const Nbr n = neighbor<S, D>(dom, c, f);
			const S AN = Adiag[n.g];
			aadd(Abar + n.g, w * S(-0.5) * alphaAt<S, D>(dom, n.mi, n.comp) / (AN * AN));
		}
		aadd(Abar + c.g, own);
	}
}

// kUxbEpotRhs, flux part: rhs = div of the face fluxes of x = u x e_b (potential BCs)
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjEpotDivergence(Dom<S, D> dom, const S *__restrict__ rbar, S *__restrict__ xbar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const S rb = rbar[c.g];
		if (rb == 0.0) continue;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			const int dim = f >> 1;
			const S flb = ((f & 1) ? S(1) : S(-1)) * rb;
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) {
				const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
				const int bc = potBC(dom.fmask, FR, faceCell(c.B, f, c.p));
				if (bc == PB_INSULATING || bc == PB_THIN_WALL) continue;
				adjContra3<D>(dom, c.B, c.g, c.mi, dim, flb, xbar);
				continue;
			}
			adjContra3<D>(dom, c.B, c.g, c.mi, dim, S(0.5) * flb, xbar);
			const Nbr n = neighbor<S, D>(dom, c, f);
			adjContra3<D>(dom, n.B, n.g, n.mi, n.comp, n.flip ? -S(0.5) * flb : S(0.5) * flb, xbar);
		}
	}
}

// x = u x e_b: xbar -> ubar (2D velocities lifted to 3D with u_z = 0)
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjCross(Dom<S, D> dom, const double *__restrict__ eb, const S *__restrict__ xbar,
		S *__restrict__ ubar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const double *e = eb + 3 * c.B[B_INST];
		const S w0 = xbar[vidx3(c.B, c.g, 0)], w1 = xbar[vidx3(c.B, c.g, 1)], w2 = xbar[vidx3(c.B, c.g, 2)];
		ubar[vidx<D>(c.B, c.g, 0)] += -w1 * e[2] + w2 * e[1];
		ubar[vidx<D>(c.B, c.g, 1)] += w0 * e[2] - w2 * e[0];
		if (D > 2) ubar[vidx<D>(c.B, c.g, D > 2 ? 2 : 0)] += -w0 * e[1] + w1 * e[0];
	}
}

// kCurrentLorentz with accumulate = 0: src_d = N (J x e_b)_d, J from phi and x = u x e_b.
// Sbar -> phibar, xbar (+=), Nbar[inst] (+=)
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kAdjLorentz(Dom<S, D> dom, const S *__restrict__ phi, const S *__restrict__ uxb,
		const double *__restrict__ eb, const double *__restrict__ stuart, const S *__restrict__ Sbar, S *__restrict__ phibar,
		S *__restrict__ xbar, double *__restrict__ Nbar) {
	__shared__ int32_t sB[PHB_BREC];
	int l0, nc;
	loadTile<S, D>(dom, sB, l0, nc);
	for (int j = 0; j < CPT; ++j) {
		Cell c;
		if (!cellAt<D>(sB, l0, nc, j, c)) break;
		const int inst = c.B[B_INST];
		const double *e = eb + 3 * inst;
		const S Nst = stuart[inst];
		// forward: the face currents and J (as kCurrentLorentz)
		const S phiP = phi[c.g];
		S alphaP[D], cvelP[D], xP[D];
#pragma unroll
		for (int k = 0; k < D; ++k) xP[k] = uxb[vidx3(c.B, c.g, k)];
#pragma unroll
		for (int d = 0; d < D; ++d) { alphaP[d] = alphaAt<S, D>(dom, c.mi, d); cvelP[d] = contraVec<S, D>(dom, c.mi, d, xP); }
		S jf[2 * D];
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			const int dim = f >> 1;
			const S faceSign = (f & 1) ? S(1) : S(-1);
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) {
				const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
				const int fc = faceCell(c.B, f, c.p);
				const int bc = potBC(dom.fmask, FR, fc);
				if (bc == PB_INSULATING || bc == PB_THIN_WALL) jf[f] = 0;
				else if (bc == PB_DIRICHLET) jf[f] = alphaP[dim] * faceSign * (phiP - potValue<S, D>(dom, FR, fc)) + cvelP[dim];
				else jf[f] = cvelP[dim];
				continue;
			}
			const Nbr n = neighbor<S, D>(dom, c, f);
			const S alphaN = alphaAt<S, D>(dom, n.mi, n.comp);
			S xN[D];
#pragma unroll
			for (int k = 0; k < D; ++k) xN[k] = uxb[vidx3(n.B, n.g, k)];
			S cvelN = contraVec<S, D>(dom, n.mi, n.comp, xN);
			if (n.flip) cvelN = -cvelN;
			jf[f] = -S(0.5) * (alphaP[dim] + alphaN) * faceSign * (phi[n.g] - phiP) + S(0.5) * (cvelP[dim] + cvelN);
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
		const S e0 = e[0], e1 = e[1], e2 = e[2];
		const S F[3] = {J[1] * e2 - J[2] * e1, J[2] * e0 - J[0] * e2, J[0] * e1 - J[1] * e0};
		// reverse
		S Fb[3] = {0, 0, 0};
		S nAcc = 0;
#pragma unroll
		for (int d = 0; d < D; ++d) {
			const S sb = Sbar[vidx<D>(c.B, c.g, d)];
			nAcc += sb * F[d];
			Fb[d] = Nst * sb;
		}
		aadd(Nbar + inst, nAcc);
		const S Jb[3] = {-Fb[1] * e2 + Fb[2] * e1, Fb[0] * e2 - Fb[2] * e0, -Fb[0] * e1 + Fb[1] * e0};
		if (D == 2) aadd(xbar + vidx3(c.B, c.g, 2), Jb[2]);
		S javgb[D];
#pragma unroll
		for (int k = 0; k < D; ++k) {
			S s = 0;
#pragma unroll
			for (int r = 0; r < D; ++r) s += dom.m(r * D + k, c.mi) * Jb[r];
			javgb[k] = s * invDet;
		}
		S phiPb = 0, cvelPb[D];
#pragma unroll
		for (int d = 0; d < D; ++d) cvelPb[d] = 0;
#pragma unroll
		for (int f = 0; f < 2 * D; ++f) {
			const int dim = f >> 1;
			const S faceSign = (f & 1) ? S(1) : S(-1);
			const S jb = S(0.5) * javgb[dim];
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) {
				const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
				const int bc = potBC(dom.fmask, FR, faceCell(c.B, f, c.p));
				if (bc == PB_INSULATING || bc == PB_THIN_WALL) continue;
				if (bc == PB_DIRICHLET) phiPb += alphaP[dim] * faceSign * jb;
				cvelPb[dim] += jb;
				continue;
			}
			const Nbr n = neighbor<S, D>(dom, c, f);
			const S coeff = S(0.5) * (alphaP[dim] + alphaAt<S, D>(dom, n.mi, n.comp));
			aadd(phibar + n.g, -coeff * faceSign * jb);
			phiPb += coeff * faceSign * jb;
			cvelPb[dim] += S(0.5) * jb;
			adjContra3<D>(dom, n.B, n.g, n.mi, n.comp, n.flip ? -S(0.5) * jb : S(0.5) * jb, xbar);
		}
		aadd(phibar + c.g, phiPb);
#pragma unroll
		for (int d = 0; d < D; ++d) adjContra3<D>(dom, c.B, c.g, c.mi, d, cvelPb[d], xbar);
	}
}

} // namespace phb

using namespace phb;

#define PHB_ADJ(DOM, ...)                                                                            \
	do {                                                                                             \
		if (!(DOM) || (DOM)->dtype != PHB_F64) return setError(PHB_ERR_ARG, "adjoint kernels take float64 domains"); \
		if ((DOM)->ntiles == 0) return PHB_OK;                                                       \
		cudaStream_t s_ = (cudaStream_t)stream;                                                      \
		if ((DOM)->dims == 2) { constexpr int D = 2; Dom<S, D> dm(*(DOM)); __VA_ARGS__; }                \
		else if ((DOM)->dims == 3) { constexpr int D = 3; Dom<S, D> dm(*(DOM)); __VA_ARGS__; }           \
		else return setError(PHB_ERR_ARG, "dims");                                                  \
	} while (0)
#define PHB_TL dim3(dom->ntiles), dim3(PHB_TILE), 0, s_

// the transpose reads the topology and the stencil only: any value type of the domain
extern "C" int phb_transpose_stencil(const phb_domain *dom, const void *C, void *CT, phb_stream stream) {
	if (!dom || !C || !CT) return setError(PHB_ERR_ARG, "phb_transpose_stencil: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	cudaStream_t s_ = (cudaStream_t)stream;
	auto run = [&](auto tag) {
		using T = decltype(tag);
		if (dom->dims == 2) kTransposeStencil<2, T><<<dim3(dom->ntiles), dim3(PHB_TILE), 0, s_>>>(Dom<T, 2>(*dom), (const T *)C, (T *)CT);
		else kTransposeStencil<3, T><<<dim3(dom->ntiles), dim3(PHB_TILE), 0, s_>>>(Dom<T, 3>(*dom), (const T *)C, (T *)CT);
	};
	if (dom->dims != 2 && dom->dims != 3) return setError(PHB_ERR_ARG, "dims");
	if (dom->dtype == PHB_F64) run(double{});
	else if (dom->dtype == PHB_F32) run(float{});
	else return setError(PHB_ERR_ARG, "phb_transpose_stencil: dtype");
	return checkLaunch("kTransposeStencil");
}

extern "C" int phb_adj_outer(const phb_domain *dom, int ncomp, const double *lam, const double *x, double scale, double *Mbar,
		phb_stream stream) {
	if (!lam || !x || !Mbar || (ncomp != 1 && ncomp != dom->dims)) return setError(PHB_ERR_ARG, "phb_adj_outer: bad argument");
	PHB_ADJ(dom, {
		if (ncomp == 1) kAdjOuter<D, 1><<<PHB_TL>>>(dm, lam, x, scale, Mbar);
		else kAdjOuter<D, D><<<PHB_TL>>>(dm, lam, x, scale, Mbar);
	});
	return checkLaunch("kAdjOuter");
}

extern "C" int phb_adj_advection_matrix(const phb_domain *dom, const double *Cbar, const double *u, double *ubar, phb_stream stream) {
	if (!Cbar || !ubar || (dom && dom->scheme != 0 && !u)) return setError(PHB_ERR_ARG, "phb_adj_advection_matrix: null argument");
	PHB_ADJ(dom, kAdjAdvectionMatrix<D><<<PHB_TL>>>(dm, Cbar, u, ubar));
	return checkLaunch("kAdjAdvectionMatrix");
}

extern "C" int phb_adj_advection_rhs(const phb_domain *dom, const double *rhsbar, const double *u, double *ubar, double *srcbar,
		double *ubbar, phb_stream stream) {
	if (!rhsbar || !ubar || (dom && dom->scheme != 0 && !u)) return setError(PHB_ERR_ARG, "phb_adj_advection_rhs: null argument");
	PHB_ADJ(dom, kAdjAdvectionRhs<D><<<PHB_TL>>>(dm, rhsbar, u, ubar, srcbar, ubbar));
	return checkLaunch("kAdjAdvectionRhs");
}

extern "C" int phb_adj_scalar_rhs(const phb_domain *dom, const phb_scalar *sc, const double *phi, const double *u,
		const double *rhsbar, double *phibar, double *valuesbar, double *ubar, double *ubbar, phb_stream stream) {
	if (!sc || !phi || !rhsbar || !phibar || (dom && dom->scheme != 0 && (!u || !ubar)))
		return setError(PHB_ERR_ARG, "phb_adj_scalar_rhs: null argument");
	if (sc->channels < 1 || (sc->nu_count != 0 && sc->nu_count != 1 && sc->nu_count != sc->channels) || (sc->nu_count > 0 && !sc->nu) ||
			(dom && dom->nfixed > 0 && (!sc->types || !sc->values || !sc->offsets || !sc->statics)))
		return setError(PHB_ERR_ARG, "phb_adj_scalar_rhs: bad scalar description");
	const ScalarView sv = scalarView(sc);
	PHB_ADJ(dom, kAdjScalarRhs<D><<<PHB_TL>>>(dm, sv, phi, u, rhsbar, phibar, valuesbar, ubar, ubbar));
	return checkLaunch("kAdjScalarRhs");
}

extern "C" int phb_adj_pressure_rhs(const phb_domain *dom, const double *C, const double *Adiag, const double *u, const double *ustar,
		const double *h,
		const double *hbar, double *ubar, double *ustarbar, double *Cbar, double *Abar, double *srcbar, double *ubbar,
		phb_stream stream) {
	if (!C || !Adiag || !ustar || !h || !hbar || !ubar || !ustarbar || !Cbar || !Abar || (dom && dom->scheme != 0 && !u))
		return setError(PHB_ERR_ARG, "phb_adj_pressure_rhs: null argument");
	PHB_ADJ(dom, kAdjPressureRhs<D><<<PHB_TL>>>(dm, C, Adiag, u, ustar, h, hbar, ubar, ustarbar, Cbar, Abar, srcbar, ubbar));
	return checkLaunch("kAdjPressureRhs");
}

extern "C" int phb_adj_divergence(const phb_domain *dom, const double *dbar, double *fbar, double *ubbar, phb_stream stream) {
	if (!dbar || !fbar) return setError(PHB_ERR_ARG, "phb_adj_divergence: null argument");
	PHB_ADJ(dom, kAdjDivergence<D><<<PHB_TL>>>(dm, dbar, fbar, ubbar));
	return checkLaunch("kAdjDivergence");
}

extern "C" int phb_adj_correct_velocity(const phb_domain *dom, const double *p, const double *Adiag, const double *ubar,
		double *hbar, double *pbar, double *Abar, phb_stream stream) {
	if (!p || !Adiag || !ubar || !hbar || !pbar || !Abar) return setError(PHB_ERR_ARG, "phb_adj_correct_velocity: null argument");
	PHB_ADJ(dom, kAdjCorrectVelocity<D><<<PHB_TL>>>(dm, p, Adiag, ubar, hbar, pbar, Abar));
	return checkLaunch("kAdjCorrectVelocity");
}

extern "C" int phb_adj_pressure_matrix(const phb_domain *dom, const double *Adiag, const double *Pbar, double *Abar, phb_stream stream) {
	if (!Adiag || !Pbar || !Abar) return setError(PHB_ERR_ARG, "phb_adj_pressure_matrix: null argument");
	PHB_ADJ(dom, kAdjPressureMatrix<D><<<PHB_TL>>>(dm, Adiag, Pbar, Abar));
	return checkLaunch("kAdjPressureMatrix");
}

extern "C" int phb_adj_uxb_epot_rhs(const phb_domain *dom, const double *e_b, const double *rbar, double *xbar, double *ubar,
		phb_stream stream) {
	if (!e_b || !xbar || !ubar) return setError(PHB_ERR_ARG, "phb_adj_uxb_epot_rhs: null argument");
	PHB_ADJ(dom, {
		if (rbar) kAdjEpotDivergence<D><<<PHB_TL>>>(dm, rbar, xbar);
		kAdjCross<D><<<PHB_TL>>>(dm, e_b, xbar, ubar);
	});
	return checkLaunch("kAdjUxbEpotRhs");
}

extern "C" int phb_adj_lorentz(const phb_domain *dom, const double *phi, const double *uxb, const double *e_b, const double *stuart,
		const double *srcbar, double *phibar, double *xbar, double *stuartbar, phb_stream stream) {
	if (!phi || !uxb || !e_b || !stuart || !srcbar || !phibar || !xbar || !stuartbar) return setError(PHB_ERR_ARG, "phb_adj_lorentz: null argument");
	PHB_ADJ(dom, kAdjLorentz<D><<<PHB_TL>>>(dm, phi, uxb, e_b, stuart, srcbar, phibar, xbar, stuartbar));
	return checkLaunch("kAdjLorentz");
}
