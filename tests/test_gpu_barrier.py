"""The bounded wait of the persistent solvers' grid barrier (csrc/krylov.cu gridBarrier):
with one CTA of a cooperative launch absent, every other CTA's wait runs out after its spin
limit, the launch ends with the barrier error flag set instead of waiting for good, and the
context stays usable for the next solve."""
import ctypes as ct
import time

import pytest
import torch

import phipict_b200 as pb
from phipict_b200 import _lib
from cases import hartmann_2d, seeded_state

pytestmark = pytest.mark.gpu


def _selftest(lib, ctas, rounds, absent, limit, scratch):
    err, done = ct.c_int(-1), ct.c_int(-1)
    rc = lib.phb_barrier_selftest(ctas, rounds, absent, limit, scratch.data_ptr(), ct.byref(err), ct.byref(done),
                                  _lib.stream_ptr(scratch.device))
    assert rc == 0, lib.phb_last_error()
    return err.value, done.value


@pytest.mark.parametrize("per_sm", [1, 3])
def test_barrier_passes_with_every_cta_present(cuda, per_sm):
    """One CTA per SM, and three (432 or 444 CTAs: many arrival groups, the last one short)."""
    lib = _lib.load()
    scratch = torch.zeros(512, dtype=torch.uint8, device="cuda")
    ctas = per_sm * torch.cuda.get_device_properties(0).multi_processor_count - (12 if per_sm == 3 else 0)
    assert _selftest(lib, ctas, 300, -1, 1 << 20, scratch) == (0, 300)


@pytest.mark.parametrize("absent", [0, 5, 17])
def test_barrier_wait_runs_out_when_a_cta_is_absent(cuda, absent):
    lib = _lib.load()
    scratch = torch.zeros(512, dtype=torch.uint8, device="cuda")
    ctas = torch.cuda.get_device_properties(0).multi_processor_count
    t0 = time.time()
    err, done = _selftest(lib, ctas, 50, absent, 1 << 14, scratch)
    assert err == 1 and done == 0
    assert time.time() - t0 < 30
    # the context is still usable: a step runs and converges
    dom = hartmann_2d(8, 6)
    seeded_state(dom, 1)
    dom.PrepareSolve()
    sim = pb.Simulation(dom, 0.01, non_orthogonal=False, advection_tol=pb.SolverTolerance(rtol=1e-10),
                        pressure_tol=pb.SolverTolerance(rtol=1e-10))
    assert sim.single_step(), sim.last_error


def test_selftest_rejects_bad_arguments(cuda):
    lib = _lib.load()
    scratch = torch.zeros(512, dtype=torch.uint8, device="cuda")
    err, done = ct.c_int(), ct.c_int()
    assert lib.phb_barrier_selftest(0, 1, -1, 1 << 14, scratch.data_ptr(), ct.byref(err), ct.byref(done), None) == -1
    assert lib.phb_barrier_selftest(1 << 20, 1, -1, 1 << 14, scratch.data_ptr(), ct.byref(err), ct.byref(done), None) != 0
