"""Python side of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_build/liboracle.so`` (compiled from oracle.cpp by ``oracle/build.py``),
packs one environment of a ``phipict_b200.Domain`` description into the oracle's flat
format, and runs the reference PISO/MHD step on the CPU with the oracle's kernels and
solvers (step order of core/piso_simulation.py:3525-4169 and simulation/mhd.py:543-1002).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this module. The
domain description is read from the blocks and boundaries (sizes, face types, connection
axes, boundary data, vertex coordinates); every derived quantity (metrics, neighbours,
CSR pattern, matrices) is recomputed here by the oracle itself.
"""
from __future__ import annotations

import ctypes as ct
import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

HDR, BREC, FREC = 8, 40, 12

_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            from oracle import build as _b

            _b.build()
        _lib = ct.CDLL(str(LIB))
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


class OracleDomain:
    """One environment of a domain in the oracle's packed format, in dtype S."""

    def __init__(self, domain, env: int = 0, dtype=np.float64):
        import torch

        self.S = np.dtype(dtype)
        self.suf = "_d" if self.S == np.float64 else "_f"
        lib = load()
        d = domain.getSpatialDims()
        self.dims = d
        blocks = domain.getBlocks()
        self.blocks = blocks
        bidx = {id(b): i for i, b in enumerate(blocks)}
        offs = []
        off = 0
        for b in blocks:
            offs.append(off)
            off += math.prod(b.getSizes())
        self.n = off
        self.offsets = offs
        TS = 2 * d * d + 1
        self.TS = TS
        fixed = []
        for i, b in enumerate(blocks):
            for f, bd in enumerate(b.getBoundaries()):
                if type(bd).__name__ == "FixedBoundary":
                    fixed.append((i, f, bd))
        nf = len(fixed)
        desc = np.zeros(HDR + len(blocks) * BREC + max(1, nf) * FREC, dtype=np.int32)
        desc[0:4] = [d, len(blocks), self.n, nf]
        fid = {(i, f): k for k, (i, f, _) in enumerate(fixed)}
        for i, b in enumerate(blocks):
            r = HDR + i * BREC
            sz = b.getSizes()
            desc[r:r + 4] = [sz[0], sz[1], sz[2], offs[i]]
            for f, bd in enumerate(b.getBoundaries()):
                base = r + 4 + f * 6
                name = type(bd).__name__
                if name == "FixedBoundary":
                    desc[base] = 0
                    desc[base + 5] = fid[(i, f)]
                elif name == "PeriodicBoundary":
                    desc[base] = 1
                else:
                    desc[base] = 2
                    desc[base + 1] = bidx[id(bd.connectedBlock)]
                    ax = list(bd.axes) + [0] * (3 - len(bd.axes))
                    desc[base + 2:base + 5] = ax[:3]
        # cell transforms
        Tc = np.zeros((self.n, TS), dtype=self.S)
        for i, b in enumerate(blocks):
            n_b = math.prod(b.getSizes())
            if b.vertexCoordinates is not None:
                coords = np.ascontiguousarray(b.vertexCoordinates[0].detach().cpu().numpy().astype(self.S))
                out = np.zeros((n_b, TS), dtype=self.S)
                nx, ny, nz = b.getSizes()
                getattr(lib, "orc_cell_transforms" + self.suf)(d, nx, ny, nz, _p(coords), _p(out))
                Tc[offs[i]:offs[i] + n_b] = out
            else:
                Tc[offs[i]:offs[i] + n_b] = _identity(d, TS, self.S)
        # fixed faces
        fvel, fpot, fmask = [], [], []
        Tf = []
        vo = po = mo = to = 0
        fcw = np.zeros(max(1, nf), dtype=self.S)
        for k, (i, f, bd) in enumerate(fixed):
            b = blocks[i]
            fc = bd.face_cells()
            r = HDR + len(blocks) * BREC + k * FREC
            v = bd.velocity.detach().cpu()
            ve = v[env if v.shape[0] > 1 else 0]
            static = v.dim() == 2
            vals = ve.reshape(-1).numpy().astype(self.S)
            fvel.append(vals)
            pv = bd.getPotentialValues()
            pt = bd.getPotentialTypes()
            desc[r:r + FREC] = [i, f, 1 if static else 0, int(bd.velocityType), int(bd.getPotentialBC()),
                                mo if pt is not None else -1, po if pv is not None else -1, vo, fc, to, 0, 0]
            vo += vals.size
            if pv is not None:
                pvals = pv.detach().cpu()[env if pv.shape[0] > 1 else 0].reshape(-1).numpy().astype(self.S)
                fpot.append(pvals)
                po += fc
            if pt is not None:
                fmask.append(pt.detach().cpu().reshape(-1).numpy().astype(np.int8))
                mo += fc
            fcw[k] = bd.getPotentialCw()
            if b.vertexCoordinates is not None:
                coords = np.ascontiguousarray(b.vertexCoordinates[0].detach().cpu().numpy().astype(self.S))
                out = np.zeros((fc, TS), dtype=self.S)
                nx, ny, nz = b.getSizes()
                getattr(lib, "orc_face_transforms" + self.suf)(d, nx, ny, nz, _p(coords), f, _p(out))
                Tf.append(out)
            else:
                Tf.append(np.tile(_identity(d, TS, self.S), (fc, 1)))
            to += fc
        # passive scalar per fixed face and channel: type, values (static: one per channel)
        C = domain.getPassiveScalarChannels() if hasattr(domain, "getPassiveScalarChannels") else 0
        self.channels = C
        self.scalar_faces = []
        for k, (i, f, bd) in enumerate(fixed):
            if C == 0 or bd.passiveScalar is None:
                self.scalar_faces.append(None)
                continue
            ps = bd.passiveScalar.detach().cpu()
            pe = ps[env if ps.shape[0] > 1 else 0].numpy().astype(self.S)  # [C] or [C, *face]
            types = list(bd._scalar_types())
            self.scalar_faces.append((pe.ndim == 1, pe.reshape(C, -1), types, bd.isPassiveScalarBoundaryTypeStatic()))
        # advection scheme (0 CENTRAL, 1 LINEAR_UPWIND)
        self.scheme = int(domain.getAdvectionScheme()) if hasattr(domain, "getAdvectionScheme") else 0
        self.desc = desc
        self.Tc = np.ascontiguousarray(Tc)
        self.Tf = np.ascontiguousarray(np.concatenate(Tf) if Tf else np.zeros((1, TS), dtype=self.S))
        self.fvel = np.ascontiguousarray(np.concatenate(fvel) if fvel else np.zeros(1, dtype=self.S))
        self.fpot = np.ascontiguousarray(np.concatenate(fpot) if fpot else np.zeros(1, dtype=self.S))
        self.fmask = np.ascontiguousarray(np.concatenate(fmask) if fmask else np.zeros(1, dtype=np.int8))
        self.fcw = fcw
        self.row = np.zeros(self.n + 1, dtype=np.int32)
        self._f("orc_row_pointers")(*self._dargs(), _p(self.row))
        self.nnz = int(self.row[-1])
        self.col = np.zeros(self.nnz, dtype=np.int32)
        # the column pattern shared by all matrices of the domain
        _, self.col = self.laplace_matrix(epot=True)
        del torch

    # --- plumbing ---
    def _f(self, name):
        return getattr(load(), name + self.suf)

    def _dargs(self):
        return (_p(self.desc), _p(self.Tc), _p(self.Tf), _p(self.fvel), _p(self.fpot), _p(self.fcw), _p(self.fmask))

    def vec(self, comps: int = 1) -> np.ndarray:
        return np.zeros(comps * self.n, dtype=self.S)

    def _a(self, x):
        return np.ascontiguousarray(np.asarray(x, dtype=self.S))

    # --- kernels (each mirrors one reference kernel, see oracle.cpp) ---
    def advection_matrix(self, u, dt, nu, flags=0):
        """flags: the non-orthogonal bits (NON_ORTHO_CENTER_MATRIX, NON_ORTHO_DIRECT_MATRIX)."""
        val = np.zeros(self.nnz, dtype=self.S)
        A = self.vec()
        self._f("orc_adv_matrix")(*self._dargs(), _p(self._a(u)), ct.c_double(dt), ct.c_double(nu), _p(self.row),
                                  _p(self.col), _p(val), _p(A), self.scheme, int(flags))
        return val, A

    def _scalar_face_data(self, c):
        """Channel c's fixed-face types, values, offsets and static flags (one environment)."""
        nf = max(1, len(self.scalar_faces))
        types = np.zeros(nf, dtype=np.int8)
        offs = np.zeros(nf, dtype=np.int64)
        stat = np.zeros(nf, dtype=np.int8)
        vals, o = [], 0
        for k, fd in enumerate(self.scalar_faces):
            if fd is None:
                stat[k] = 1
                offs[k] = o
                vals.append(np.zeros(1, dtype=self.S))
                o += 1
                continue
            static, v, t, _ = fd
            types[k] = t[c]
            stat[k] = 1 if static else 0
            offs[k] = o
            vals.append(np.ascontiguousarray(v[c]).astype(self.S))
            o += v.shape[1]
        return types, np.ascontiguousarray(np.concatenate(vals) if vals else np.zeros(1, dtype=self.S)), offs, stat

    def scalar_matrix(self, u, dt, nu, channel, flags=0):
        """advection.cu:27-305 with forPassiveScalar for one channel (its diffusivity nu)."""
        types, _, _, _ = self._scalar_face_data(channel)
        val = np.zeros(self.nnz, dtype=self.S)
        A = self.vec()
        self._f("orc_scalar_matrix")(*self._dargs(), _p(self._a(u)), ct.c_double(dt), ct.c_double(nu), _p(types),
                                     _p(self.row), _p(self.col), _p(val), _p(A), self.scheme, int(flags))
        return val, A

    def scalar_rhs(self, phi_c, dt, nu, channel, u=None, flags=0, phires=None):
        """advection.cu:545-698 for one channel's field phi_c [n]; u (the block velocity) gives
        the LINEAR_UPWIND fluxes; phires (the channel's scalar result) the non-orthogonal terms."""
        types, vals, offs, stat = self._scalar_face_data(channel)
        rhs = self.vec()
        uu = self._a(u) if u is not None else self.vec(self.dims)
        self._f("orc_scalar_rhs")(*self._dargs(), _p(self._a(phi_c)), ct.c_double(dt), ct.c_double(nu), _p(types),
                                  _p(vals), _p(offs), _p(stat), _p(rhs), _p(uu), self.scheme, int(flags),
                                  _p(self._a(phires)) if phires is not None else None)
        return rhs

    def advection_rhs(self, u, src, dt, nu, flags=0, ures=None):
        """ures: the velocity result [d][n] whose non-orthogonal terms enter (flags)."""
        rhs = self.vec(self.dims)
        src_arr, static = self._src(src)
        self._f("orc_adv_rhs")(*self._dargs(), _p(self._a(u)), _p(src_arr), static, ct.c_double(dt), ct.c_double(nu), _p(rhs),
                               self.scheme, int(flags), _p(self._a(ures)) if ures is not None else None)
        return rhs

    def _src(self, src):
        if src is None:
            return None, 0
        s = self._a(src)
        return s, 1 if s.size == self.dims else 0

    def laplace_matrix(self, A=None, epot=False, flags=0):
        val = np.zeros(self.nnz, dtype=self.S)
        col = np.zeros(self.nnz, dtype=np.int32)
        self._f("orc_laplace_matrix")(*self._dargs(), _p(self._a(A) if A is not None else self.vec()), 1 if epot else 0,
                                      _p(self.row), _p(col), _p(val), int(flags))
        return val, col

    def pressure_nonortho(self, A, p, flags, div):
        """pressure.cu:839-860: div + the non-orthogonal terms of the pressure result p."""
        out = self._a(div).copy()
        self._f("orc_pressure_nonortho")(*self._dargs(), _p(self._a(A)), _p(self._a(p)), int(flags), _p(out))
        return out

    def pressure_rhs(self, Cval, A, u, ustar, src, dt, nu):
        h = self.vec(self.dims)
        src_arr, static = self._src(src)
        self._f("orc_pressure_rhs")(*self._dargs(), _p(self.row), _p(self.col), _p(self._a(Cval)), _p(self._a(A)),
                                    _p(self._a(u)), _p(self._a(ustar)), _p(src_arr), static, ct.c_double(dt),
                                    ct.c_double(nu), _p(h), self.scheme)
        return h

    def divergence(self, field):
        out = self.vec()
        self._f("orc_divergence")(*self._dargs(), _p(self._a(field)), _p(out))
        return out

    def correct_velocity(self, p, hbya, A):
        out = self.vec(self.dims)
        self._f("orc_correct_velocity")(*self._dargs(), _p(self._a(p)), _p(self._a(hbya)), _p(self._a(A)), _p(out))
        return out

    def epot_rhs(self, field):
        out = self.vec()
        self._f("orc_epot_rhs")(*self._dargs(), _p(self._a(field)), _p(out))
        return out

    def current_density(self, phi, uxb):
        J = self.vec(3)
        self._f("orc_current_density")(*self._dargs(), _p(self._a(phi)), _p(self._a(uxb)), _p(J))
        return J

    def spmv(self, val, x, col=None):
        y = np.zeros_like(self._a(x))
        self._f("orc_spmv")(self.n, _p(self.row), _p(self.col if col is None else col), _p(self._a(val)), _p(self._a(x)), _p(y))
        return y

    def solve(self, val, b, x, tol, maxit=5000, bicg=False, col=None):
        """Returns (status, iterations, criterion); x is updated in place."""
        it = ct.c_int(0)
        crit = ct.c_double(0)
        fn = self._f("orc_bicgstab" if bicg else "orc_cg")
        st = fn(self.n, _p(self.row), _p(self.col if col is None else col), _p(self._a(val)), _p(self._a(b)), _p(x),
                ct.c_double(tol), int(maxit), ct.byref(it), ct.byref(crit))
        return st, it.value, crit.value

    def csr_matrix(self, val, col=None):
        import scipy.sparse as sp

        return sp.csr_matrix((np.asarray(val, dtype=np.float64), self.col if col is None else col, self.row),
                             shape=(self.n, self.n))


def _identity(d, TS, S):
    t = np.zeros(TS, dtype=S)
    for i in range(d):
        t[i * d + i] = 1
        t[d * d + i * d + i] = 1
    t[2 * d * d] = 1
    return t


def resolve_tol(tol, rhs: np.ndarray, dtype) -> float:
    """SolverTolerance / float / None -> absolute tolerance (solvers/tolerance.py:180-257)."""
    eps = np.finfo(dtype).eps
    default = 1e-8 if np.dtype(dtype) == np.float64 else 1e-5
    if tol is None:
        return default
    if isinstance(tol, (int, float)):
        return float(tol)
    n = rhs.size
    scale = float(np.linalg.norm(rhs.astype(np.float64))) / math.sqrt(n) if n else 0.0
    t = 0.0
    if tol.rtol is not None:
        t = tol.rtol * scale
    if tol.atol is not None:
        t = max(t, tol.atol)
    t = max(t, 8.0 * eps * scale)
    if not t > 0:
        t = default
    return t


class OracleSim:
    """Reference PISO (+ inductionless MHD) step of one environment on the CPU."""

    def __init__(self, od: OracleDomain, u0: np.ndarray, dt: float, nu: float, *, corrector_steps=2,
                 advection_tol=None, pressure_tol=None, source=None, mhd=None, maxit=5000, scalar=None,
                 nonortho_flags=0, advect_non_ortho_steps=1, pressure_non_ortho_steps=1, pressure_bicg=False):
        self.od = od
        self.pressure_bicg = bool(pressure_bicg)
        # core/piso_simulation.py:3225-3345,3839-3891,3978-4117: with non-orthogonal flags the
        # right-hand sides carry the lagged cross terms of the current result, re-solved
        # advect/pressure_non_ortho_steps times
        self.flags = int(nonortho_flags)
        self.advect_no_steps = int(advect_non_ortho_steps)
        self.pressure_no_steps = int(pressure_non_ortho_steps)
        self.dt = dt
        self.nu = nu
        self.corrector_steps = corrector_steps
        self.advection_tol = advection_tol
        self.pressure_tol = pressure_tol
        self.maxit = maxit
        self.u = od._a(u0).copy()             # block velocity u^n, [d][n]
        self.u_res = od.vec(od.dims)          # velocityResult (zero until the first step)
        self.p = od.vec()
        self.src = None if source is None else od._a(source).copy()
        self.mhd = mhd                        # dict(stuart=, e_b=, potential_tol=, singular=)
        if mhd is not None:
            self.phi = od.vec()
            self.uxb = od.vec(3)
            self.Eval, self.Ecol = od.laplace_matrix(epot=True)
        # passive scalar: dict(phi=[C][n] initial field, nu=None | [1] | [C] diffusivities)
        self.scalar = scalar
        if scalar is not None:
            self.phi_s = od._a(scalar["phi"]).reshape(od.channels, od.n).copy()
        self.iterations = {}

    def _mean_sub(self, x):
        return x - x.mean()

    def scalar_step(self):
        """core/piso_simulation.py:3225-3345, 3589-3775: every channel advected and diffused
        implicitly with the step-start velocity, zero initial guess, re-solved with the cross
        terms of its result when non-orthogonal flags are set. Returns the channel-0
        matrix when the velocity step reuses it (same diffusivity as the velocity, one set of
        face types for all channels), else None."""
        od, C = self.od, self.od.channels
        nus = self.scalar.get("nu")
        static_nu = nus is None or len(nus) == 1
        types_static = all(fd is None or fd[3] for fd in od.scalar_faces)
        split = not (static_nu and types_static)
        nu_of = (lambda c: self.nu) if nus is None else (lambda c: float(nus[0] if len(nus) == 1 else nus[c]))
        fl = self.flags
        mat = None if split else od.scalar_matrix(self.u, self.dt, nu_of(0), 0, flags=fl)
        its = []
        res = self.phi_s.copy()  # CopyScalarResultFromBlocks
        for c in range(C):
            Cval, _ = od.scalar_matrix(self.u, self.dt, nu_of(c), c, flags=fl) if split else mat
            for no_step in range(self.advect_no_steps if fl else 1):
                rhs = od.scalar_rhs(self.phi_s[c], self.dt, nu_of(c), c, u=self.u, flags=fl,
                                    phires=res[c] if fl else None)
                tol = resolve_tol(self.advection_tol, rhs, od.S)
                x = od.vec() if no_step == 0 else res[c].copy()
                st, it, _ = od.solve(Cval, rhs, x, tol, self.maxit, bicg=True)
                if st != 1:
                    raise RuntimeError(f"oracle scalar solve failed ({st})")
                res[c] = x
                its.append(it)
        self.phi_s = res
        self.iterations["scalar"] = its
        reuse = nus is None and not split
        return mat if reuse else None

    def step(self):
        od, d, n = self.od, self.od.dims, self.od.n
        reused = self.scalar_step() if self.scalar is not None else None
        if self.mhd is not None:
            J = od.current_density(self.phi, self.uxb).reshape(3, n)
            e = np.asarray(self.mhd["e_b"], dtype=od.S)
            N = od.S.type(self.mhd["stuart"])
            F = N * np.cross(J.T, e).T  # [3][n]
            F = F[:d].reshape(-1).astype(od.S)
            if self.src is None:
                self.src = F
            else:
                base = self.src if self.src.size == d * n else np.repeat(self.src, n)
                self.src = (F + base).astype(od.S)
        fl = self.flags
        Cval, A = reused if reused is not None else od.advection_matrix(self.u, self.dt, self.nu, flags=fl)
        its = []
        if fl:
            self.u_res = self.u.copy()  # CopyVelocityResultFromBlocks
        for no_step in range(self.advect_no_steps if fl else 1):
            rhs = od.advection_rhs(self.u, self.src, self.dt, self.nu, flags=fl, ures=self.u_res if fl else None)
            tol = resolve_tol(self.advection_tol, rhs, od.S)
            for k in range(d):
                xk = od.vec() if (fl and no_step == 0) else self.u_res[k * n:(k + 1) * n].copy()
                st, it, _ = od.solve(Cval, rhs[k * n:(k + 1) * n].copy(), xk, tol, self.maxit, bicg=True)
                if st != 1:
                    raise RuntimeError(f"oracle momentum solve failed ({st})")
                self.u_res[k * n:(k + 1) * n] = xk
                its.append(it)
        self.iterations["velocity"] = its
        Pval, Pcol = od.laplace_matrix(A, flags=fl)
        for c in range(self.corrector_steps):
            h = od.pressure_rhs(Cval, A, self.u, self.u_res, self.src, self.dt, self.nu)
            for pstep in range(self.pressure_no_steps if fl else 1):
                div = od.divergence(h)
                if fl:
                    div = od.pressure_nonortho(A, self.p, fl, div)
                ptol = resolve_tol(self.pressure_tol, div, od.S)
                p = od.vec() if pstep == 0 else self.p.copy()
                st, it, _ = od.solve(Pval, div, p, ptol, self.maxit, bicg=self.pressure_bicg, col=Pcol)
                if st != 1:
                    raise RuntimeError(f"oracle pressure solve failed ({st})")
                self.iterations[f"pressure{c}"] = it
                self.p = self._mean_sub(p).astype(od.S)
            self.u_res = od.correct_velocity(self.p, h, A)
        self.u = self.u_res.copy()
        if self.mhd is not None:
            self.potential_step()

    def potential_step(self):
        od, d, n = self.od, self.od.dims, self.od.n
        e = np.asarray(self.mhd["e_b"], dtype=od.S)
        u3 = np.zeros((3, n), dtype=od.S)
        u3[:d] = self.u_res.reshape(d, n)
        self.uxb = np.cross(u3.T, e).T.astype(od.S).reshape(-1)
        rhs = od.epot_rhs(self.uxb[: d * n])
        singular = self.mhd.get("singular", True)
        if singular:
            rhs = self._mean_sub(rhs).astype(od.S)
            self.phi = self._mean_sub(self.phi).astype(od.S)
        tol = resolve_tol(self.mhd.get("potential_tol"), rhs, od.S)
        phi = self.phi.copy()
        st, it, _ = od.solve(self.Eval, rhs, phi, tol, self.maxit, col=self.Ecol)
        self.iterations["epot"] = it
        if singular:
            phi = self._mean_sub(phi).astype(od.S)
        self.phi = phi
