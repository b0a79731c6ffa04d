"""Generate the reference field fixtures ``tests/golden/ref_<case>_<dtype>.npz`` by running
phiPICT itself (its unmodified Python package and ``_C`` extension) on a CUDA GPU.

The reference has no CPU path (its domain setters require CUDA tensors), so this runs on a
GPU machine with the reference built by ``oracle/build_ref.py`` into ``oracle/_ref``:

    PYTHONPATH=oracle/_ref python tests/golden/make_ref_fields.py --out tests/golden

It writes one ``.npz`` per case and dtype holding the inputs (vertices, initial velocity,
inflow) and the fields u, p (per block) and phi after each recorded step, plus a JSON line per
run (iterations, timing) to stdout. ``--amg`` writes ``ref_amg_pcg.npz``: phiPICT's
``_C.AMGPCGSolve`` on the cases of ``amg_cases.py``. ``--time-duct`` also times the reference's plain
(non-AMG; pyamg is not installed) GPU step on the full 3-block 64x48x48 duct.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np
import torch

sys.path.insert(0, str(Path(__file__).resolve().parent))
import ref_cases as rc  # noqa: E402


def run_case(pp, case: str, dtype, tight: bool, out: Path) -> dict:
    inputs = rc.c1_inputs() if case == "c1" else rc.c2r_inputs()
    build = rc.build_c1 if case == "c1" else rc.build_c2r
    record = rc.C1_RECORD if case == "c1" else rc.C2R_RECORD
    p = rc.C1 if case == "c1" else rc.C2R
    dev = torch.device("cuda")
    dom = build(pp, inputs, dtype, dev)
    sim = rc.make_sim(pp, dom, case, tight)
    data = {k: np.asarray(v) for k, v in inputs.items()}
    t0 = time.time()
    ok = True
    for step in range(1, p["steps"] + 1):
        ok = bool(sim.single_step()) and ok
        if step in record:
            for k, v in rc.fields(dom).items():
                data[f"s{step}_{k}"] = v
    torch.cuda.synchronize()
    wall = time.time() - t0
    tag = f"{case}_{'fp64' if dtype == torch.float64 else 'fp32'}{'' if tight else '_tol1e-8'}"
    data["meta"] = np.array(json.dumps(dict(case=case, dtype=str(dtype), tight=tight, steps=p["steps"],
                                            record=list(record), params=p, all_steps_ok=ok,
                                            generator="phiPICT " + getattr(pp, "__version__", "?"),
                                            device=torch.cuda.get_device_name(0))))
    np.savez_compressed(out / f"ref_{tag}.npz", **data)
    return dict(tag=tag, ok=ok, wall_s=round(wall, 3))


def time_duct(pp, steps: int, warmup: int, dtype) -> dict:
    """The reference's own GPU step on the full duct (3 x 64x48x48), plain FP64 CG/BiCGStab."""
    p = dict(rc.C2R, nx=64, ny=48, nz=48)
    saved = dict(rc.C2R)
    rc.C2R.update(p)
    try:
        inputs = rc.c2r_inputs()
        dom = rc.build_c2r(pp, inputs, dtype, torch.device("cuda"))
        t = pp.SolverTolerance(rtol=1e-10)
        sim = rc.make_sim(pp, dom, "c2r", False, advection_tol=t, pressure_tol=t, potential_tol=t)
    finally:
        rc.C2R.clear()
        rc.C2R.update(saved)
    for _ in range(warmup):
        sim.single_step()
    torch.cuda.synchronize()
    t0 = time.time()
    for _ in range(steps):
        sim.single_step()
    torch.cuda.synchronize()
    dt = (time.time() - t0) / steps
    cells = 3 * 64 * 48 * 48
    return dict(workload="duct3d 3x64x48x48 reference GPU step", dtype=str(dtype), ms_per_step=round(dt * 1e3, 2),
                mcell_steps_per_s=round(cells / dt / 1e6, 3), steps=steps)


def amg_fixture(out: Path) -> None:
    """Run phiPICT's _C.AMGPCGSolve on every case of amg_cases.py: ref_amg_pcg.npz holds each
    case's solution and result infos (residual, iterations, converged, finite)."""
    import amg_cases as ac
    from phipict import _C

    data = {}
    for name in ac.CASES:
        case = ac.build(name)
        args, kw = ac.torch_args(case, torch.device("cuda"), torch)
        infos = _C.AMGPCGSolve(*args, **kw)
        torch.cuda.synchronize()
        data[f"{name}_x"] = args[6].double().cpu().numpy().reshape(case["nenv"], -1)
        data[f"{name}_info"] = np.array([[i.finalResidual, i.usedIterations, float(i.converged),
                                          float(i.isFiniteResidual)] for i in infos])
        print(json.dumps(dict(tag=f"amg_{name}", infos=data[f"{name}_info"].tolist())), flush=True)
    data["meta"] = np.array(json.dumps(dict(device=torch.cuda.get_device_name(0))))
    np.savez_compressed(out / "ref_amg_pcg.npz", **data)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="tests/golden")
    ap.add_argument("--time-duct", action="store_true")
    ap.add_argument("--skip-fixtures", action="store_true")
    ap.add_argument("--cases", default="c1_fp64,c1_fp32,c2r_fp64", help="comma list of <case>_<dtype>")
    ap.add_argument("--grads", action="store_true", help="also the gradient cases of the differentiable step")
    ap.add_argument("--viscosity-grad", action="store_true",
                    help="gradient cases: also the gradient with respect to the viscosity")
    ap.add_argument("--amg", action="store_true", help="also the CSR AMG-PCG cases of amg_cases.py (_C.AMGPCGSolve)")
    a = ap.parse_args()
    import phipict as pp

    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    if not a.skip_fixtures:
        runs = {"c1_fp64": ("c1", torch.float64, True), "c1_fp32": ("c1", torch.float32, False),
                "c2r_fp64": ("c2r", torch.float64, True)}
        for name in a.cases.split(","):
            case, dtype, tight = runs[name]
            print(json.dumps(run_case(pp, case, dtype, tight, out)), flush=True)
    if a.grads:
        for case, make in (("g1", rc.g1_inputs), ("g2", rc.g2_inputs)):
            inputs = make()
            t0 = time.time()
            g = rc.grad_run(pp, case, inputs, torch.device("cuda"), viscosity=a.viscosity_grad)
            data = {k: np.asarray(v) for k, v in inputs.items()}
            data.update({k: np.asarray(v) for k, v in g.items()})
            data["meta"] = np.array(json.dumps(dict(case=case, params=rc.G1 if case == "g1" else rc.G2,
                                                    device=torch.cuda.get_device_name(0))))
            np.savez_compressed(out / f"ref_{case}_grad.npz", **data)
            print(json.dumps(dict(tag=f"{case}_grad", loss=g["loss"], wall_s=round(time.time() - t0, 2))), flush=True)
        runs = [("g3", lambda: rc.g3_grad_run(pp, rc.g3_inputs(), torch.device("cuda")), rc.g3_inputs, rc.G3),
                ("g1u", lambda: rc.grad_run(pp, "g1", rc.g1_inputs(), torch.device("cuda"), viscosity=True, upwind=True),
                 rc.g1_inputs, rc.G1),
                ("g3u", lambda: rc.g3_grad_run(pp, rc.g3_inputs(), torch.device("cuda"), upwind=True), rc.g3_inputs,
                 rc.G3)]
        for tag, run, make, params in runs:
            g = run()
            data = {k: np.asarray(v) for k, v in make().items()}
            data.update({k: np.asarray(v) for k, v in g.items()})
            data["meta"] = np.array(json.dumps(dict(case=tag, params=params, upwind=tag.endswith("u"),
                                                    device=torch.cuda.get_device_name(0))))
            np.savez_compressed(out / f"ref_{tag}_grad.npz", **data)
            print(json.dumps(dict(tag=f"{tag}_grad", loss=g["loss"], grads=sorted(k for k in g if k.startswith("grad_")))),
                  flush=True)
    if a.amg:
        amg_fixture(out)
    if a.time_duct:
        print(json.dumps(time_duct(pp, 3, 1, torch.float64)), flush=True)
        print(json.dumps(time_duct(pp, 3, 1, torch.float32)), flush=True)


if __name__ == "__main__":
    main()
