"""The allocation-free time-step entry point, checked against the context's compute_dt.

streams_b200_compute_dt_noalloc serves callers that cannot let the library call cudaMalloc:
host codes that own all device memory through their own pool or mapping, or that run under a
fixed memory budget.  It works on the caller's device arrays and keeps its block partials in a
static device array of the library.  This file is collected last so that a failure here leaves
every other test already run.
"""
import numpy as np
import pytest

from conftest import channel_ini, requires_gpu


@pytest.mark.gpu
@requires_gpu
def test_compute_dt_noalloc_matches_context_dt(tmp_path):
    import torch
    from streams_b200 import Case, Solver, lib

    nx, ny, nz, ng = 32, 24, 16, 3
    case = Case(tmp_path, channel_ini(nx=nx, ny=ny, nz=nz))
    s = Solver.from_case(case)
    s.init_run()
    s.advance(2)
    dt_ref = s.compute_dt()  # the existing entry point on the context's own arrays
    aux = torch.from_numpy(s.debug_fetch(0)).cuda()
    w = torch.from_numpy(s.copy_to_field()).cuda()
    g = case.grid()
    metric = [torch.from_numpy(np.ctypeslib.as_array(getattr(g, name), shape=(n,)).copy()).cuda()
              for name, n in (("dcsidx", nx), ("detady", ny), ("dzitdz", nz),
                              ("dcsidxs", nx), ("detadys", ny), ("dzitdzs", nz))]
    p = case.params()
    gamma = p.cp0 / (p.cp0 - p.rgas0)
    dt = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # two calls in a row share the static scratch
        dt.fill_(0.0)
        torch.cuda.synchronize()
        rc = lib.streams_b200_compute_dt_noalloc(nx, ny, nz, ng, w.data_ptr(), aux.data_ptr(),
                                                 *[m.data_ptr() for m in metric],
                                                 p.rgas0, p.prandtl, gamma, p.cfl, dt.data_ptr(), stream)
        torch.cuda.synchronize()
        assert rc == 0, lib.streams_b200_global_error().decode()
        got = float(dt.item())
        assert abs(got - dt_ref) <= 1e-11 * dt_ref, (call, got, dt_ref)


def test_compute_dt_noalloc_rejects_oversized_input():
    from streams_b200 import EINVAL, lib
    n = 2048  # 2048^3 cells exceed the static scratch limit; rejected before any device work
    rc = lib.streams_b200_compute_dt_noalloc(n, n, n, 3, *([1] * 8), 1.0, 0.72, 1.4, 0.8, 1, None)
    assert rc == EINVAL
    assert "static scratch limit" in lib.streams_b200_global_error().decode()


@pytest.mark.parametrize("gamma,rgas0,prandtl", [(1.0, 1.0, 0.72), (0.5, 1.0, 0.72), (float("nan"), 1.0, 0.72),
                                                  (1.4, 0.0, 0.72), (1.4, 1.0, -1.0)])
def test_compute_dt_noalloc_rejects_bad_gas_constants(gamma, rgas0, prandtl):
    # one constant gamma serves only a calorically perfect gas; nonsense constants are refused
    # before any device work (a thermally perfect case must call the context's compute_dt)
    from streams_b200 import EINVAL, lib
    rc = lib.streams_b200_compute_dt_noalloc(8, 8, 8, 3, *([1] * 8), rgas0, prandtl, gamma, 0.8, 1, None)
    assert rc == EINVAL
    assert "compute_dt_noalloc" in lib.streams_b200_global_error().decode()
