"""Shared fixtures of the test suite.

CPU tests (``-m "not gpu"``) cover the oracle against the reference's golden row, the host
set-up and the C-ABI library surface.  GPU tests (``-m gpu``) are the parity tests proper: they
run the CUDA path through the C ABI and compare it with the oracle on the same inputs.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "streams-2_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def _ensure_built():
    """Build the oracle and the CUDA library when a fresh checkout lacks them (both build on a
    CPU-only machine: nvcc cross-compiles for sm_100a)."""
    import subprocess
    for target, d in ((ROOT / "oracle" / "_build" / "liboracle.so", ROOT / "oracle"),
                      (ROOT / "streams-2_b200" / "lib" / "libstreams_b200.so", ROOT / "streams-2_b200")):
        if not target.exists():
            subprocess.run(["make", "-s", "-C", str(d), "-j8"], check=True)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    _ensure_built()


def gpu_available() -> bool:
    try:
        import torch  # noqa: F401  (plumbing only: device presence)
        return torch.cuda.is_available()
    except Exception:
        return False


def channel_ini(nx=32, ny=24, nz=16, *, lx=6.283185307179586, ly=2.0, lz=3.141592653589793, mach=1.5,
                re_bulk=3000.0, theta_wall=0.0, visc_model=1, vt_exp=0.76, sensor=0.05, ep_order=6,
                weno_scheme=3, weno_version=0, nkeep=0, amp=0.1, seed=1, y_stretch=1.5, cfl=0.8,
                num_iter=100, print_control=1, correct_bound_ord=1, reynolds_tau=None) -> str:
    """Input file of a seeded synthetic channel case (the shape of the benchmark channel).

    A [synthetic] section selects the seeded Poiseuille + uniform-noise initial field and the
    tanh-stretched staggered y grid; the rest is the solver's own singleideal.ini syntax.
    """
    syn = [f"kind = channel_poiseuille", f"amp = {amp!r}", f"seed = {seed}", f"y_stretch = {y_stretch!r}"]
    if reynolds_tau is None:
        syn.append(f"reynolds_bulk = {re_bulk!r}")
    return f"""[grid]
grid_dim = 1
domain_size_x = {lx!r}
domain_size_y = {ly!r}
domain_size_z = {lz!r}
nxmax = {nx}
nymax = {ny}
nzmax = {nz}
ng = 3
metrics_order = {ep_order}
grid_type = 3
dyptarget = 0.7
jbgrid = 32
ysmoosteps = 50

[bc]
xmin = 0
xmax = 0
ymin = 6
ymax = 6
zmin = 0
zmax = 0
xmin_nr = 0
xmax_nr = 0
ymin_nr = 0
ymax_nr = 0
zmin_nr = 0
zmax_nr = 0
correct_bound_ord = {correct_bound_ord}

[mpi]
x_split = 1
y_split = 1
z_split = 1

[controls]
restart_type = 0
cfl = {cfl!r}
iter_dt_recompute = 1
num_iter = {num_iter}

[numerics]
ep_order = {ep_order}
nkeep = {nkeep}
visc_order = {ep_order}
conservative_viscous = 1
weno_scheme = {weno_scheme}
weno_version = {weno_version}
flux_splitting = 0
sensor_threshold = {sensor!r}
rk_type = 1
rand_type = 1

[flow]
flow_init = 0
Mach = {mach!r}
Reynolds = {reynolds_tau if reynolds_tau is not None else 150.0!r}
theta_wall = {theta_wall!r}
xshock_imp = 0.
shock_angle = 0.
T_ref = 220.
aoa = 0.

[fluid]
gam = 1.4
Prandtl = 0.72
visc_model = {visc_model}
vt_exp = {vt_exp!r}
s_suth = 110.4
calorically_perfect = 1

[output]
print_control = {print_control}
dtsave_restart = 50.
dtsave = 50.
dtstat = 50.
dtslice = 50.
igslice = 0
jgslice = 0
kgslice = 0
enable_plot3d = 0
enable_vtk = 0

[synthetic]
{chr(10).join(syn)}
"""


@pytest.fixture(scope="session")
def golden():
    import json
    d = ROOT / "tests" / "golden"
    return {"ini": (d / "subsonic_channel.ini").read_text(),
            "row": json.loads((d / "subsonic_channel.json").read_text())["expected"]}


requires_gpu = pytest.mark.skipif(not gpu_available(), reason="no CUDA device")
