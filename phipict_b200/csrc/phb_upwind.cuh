// Face fluxes and the LINEAR_UPWIND pieces shared by the assembly kernels and their adjoints.
#pragma once
#include "phb_device.cuh"

namespace phb {

// computeFluxesNDLoop (piso/device/discretization.cuh:758-838): contravariant face fluxes
// of `field` (not multiplied by the face sign). Fixed faces take the boundary velocity.
template <typename S, int D>
__device__ __forceinline__ void faceFluxes(const Dom<S, D> &dom, const Cell &c, const S *__restrict__ field, S *fl) {
#pragma unroll
	for (int dim = 0; dim < D; ++dim) {
		const S velC = contraAt<S, D>(dom, c.B, c.g, c.mi, dim, field);
#pragma unroll
		for (int up = 0; up < 2; ++up) {
			const int f = dim * 2 + up;
			if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) {
				const int32_t *FR = dom.fix(fRec(c.B, f)[5]);
				fl[f] = contraFixed<S, D>(dom, FR, faceCell(c.B, f, c.p), dim);
			} else {
				const Nbr n = neighbor<S, D>(dom, c, f);
				S velN = contraAt<S, D>(dom, n.B, n.g, n.mi, n.comp, field);
				if (n.flip) velN = -velN;
				fl[f] = (velN + velC) * S(0.5);
			}
		}
	}
}

// hasFarUpwindCell (piso/device/shared_stencils.cuh:35-43): the downwind neighbour across face
// f and the far-upwind cell lie inside the block, so the face can be upwinded (LINEAR_UPWIND).
__device__ __forceinline__ bool farUpwind(const int32_t *B, const int *p, int f, bool outflow) {
	const int ax = f >> 1;
	const int sign = (f & 1) ? 1 : -1;
	const int last = B[B_NX + ax] - 1;
	const int iD = p[ax] + sign;
	if (iD < 0 || iD > last) return false;
	const int iUU = outflow ? p[ax] - sign : p[ax] + 2 * sign;
	return iUU >= 0 && iUU <= last;
}
// r -= the linear-upwind correction F 0.5 psi (phi_D - phi_U), psi = (phi_U - phi_UU) / (phi_D - phi_U),
// of every upwinded face of cell c for the field value(g), face by face
// (advection.cu:892-934, :652-688)
template <typename S, int D, typename Val>
__device__ __forceinline__ void upwindCorrection(const Cell &c, const S *fl, Val value, S &r) {
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
		const S phiP = value(c.g);
		const S phiN = value(c.g + sign * step);
		const S phiUU = value(outflow ? c.g - sign * step : c.g + 2 * sign * step);
		const S phiU = outflow ? phiP : phiN;
		const S phiD = outflow ? phiN : phiP;
		const S dD = phiD - phiU;
		const S absDD = dD < S(0) ? -dD : dD;
		if (absDD < S(1e-20)) continue;
		const S psi = (phiU - phiUU) / dD;
		r -= fout * S(0.5) * psi * dD;
	}
}

} // namespace phb
