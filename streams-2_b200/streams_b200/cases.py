"""Seeded synthetic channel cases in the solver's own input-file syntax.

The same builder serves the tests, the benchmark and the batched / served forms: a channel of
any size and flow parameters, with the seeded Poiseuille + uniform-noise initial field of the
benchmark channel, and the random case mixes of the batched and served workloads.
"""
from __future__ import annotations

import math
import random


# A thermally perfect gas for tests and examples: cp/R = sum of a_l T^l (T in kelvin),
# l = -2..2 (so that the inverse powers and the logarithm of the l = -1 term are exercised),
# about 3.49 at 220 K and 3.7 at 600 K, and the energy datum a_3 = 0.  Pass cp_poly=SYNTHETIC_CP_POLY
# (or any (indx_cp_l, indx_cp_r, coefficients) triple) to the case builders.
SYNTHETIC_CP_POLY = (-2, 2, (1000.0, 10.0, 3.3, 5.0e-4, 2.0e-7, 0.0))


def _gas_keys(cp_poly) -> str:
    """[fluid] keys of the gas model: calorically perfect, or a cp(T) polynomial."""
    if cp_poly is None:
        return "calorically_perfect = 1"
    lo, hi, coef = cp_poly
    if len(coef) != hi - lo + 2:
        raise ValueError("cp_poly needs indx_cp_r - indx_cp_l + 2 coefficients")
    return (f"calorically_perfect = 0\nindx_cp_l = {lo}\nindx_cp_r = {hi}\n"
            f"cp_coeff = {', '.join(repr(float(c)) for c in coef)}")


def channel_ini(nx=32, ny=24, nz=16, *, lx=6.283185307179586, ly=2.0, lz=3.141592653589793, mach=1.5,
                re_bulk=3000.0, theta_wall=0.0, visc_model=1, vt_exp=0.76, sensor=0.05, ep_order=6,
                weno_scheme=3, weno_version=0, nkeep=0, amp=0.1, seed=1, y_stretch=1.5, cfl=0.8,
                num_iter=100, print_control=1, correct_bound_ord=1, reynolds_tau=None,
                conservative_viscous=1, flux_splitting=0, cp_poly=None) -> str:
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
ng = {max(3, ep_order // 2, weno_scheme)}
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
conservative_viscous = {conservative_viscous}
weno_scheme = {weno_scheme}
weno_version = {weno_version}
flux_splitting = {flux_splitting}
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
{_gas_keys(cp_poly)}

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


def bl_ini(nx=64, ny=48, nz=16, *, lx=100.0, ly=12.0, lz=8.0, mach=2.0, reynolds_tau=400.0,
           reynolds_delta=None, theta_wall=1.0, visc_model=1, vt_exp=0.76, sensor=0.05, ep_order=6,
           weno_scheme=3, weno_version=0, amp=0.05, x_recyc=None, nr_outflow=1, nr_top=1, cfl=0.8,
           jbgrid=None, dyptarget=0.7, nywr=None, lywr=None, ysmoosteps=10, conservative_viscous=1,
           num_iter=100, print_control=1, correct_bound_ord=1, rand_type=1, shock_angle=None,
           xshock_imp=None, flux_splitting=0, cp_poly=None) -> str:
    """Input file of a spatially developing supersonic boundary layer (the benchmark's boundary
    layer workload): box lx x ly x lz inflow thicknesses, BL grid (grid_type 4, wall-resolved part
    of nywr points up to lywr), recycling-rescaling inflow at xmin, extrapolation with a
    characteristic non-reflecting treatment at the outflow and top (types nr_outflow / nr_top),
    isothermal wall at theta_wall (1 = recovery temperature), periodic z, and the synthetic
    power-law initial field ([synthetic] kind = bl_powerlaw)."""
    if reynolds_delta is None:
        reynolds_delta = 25.0 * reynolds_tau ** 1.1  # free-stream Re_delta of a Mach-2 layer of that Re_tau
    if x_recyc is None:
        x_recyc = 0.8 * lx
    if nywr is None:
        nywr = max(8, (3 * ny) // 4)
    if lywr is None:
        lywr = 2.5
    if jbgrid is None:
        jbgrid = max(4.0, nywr / 4.0)
    # an impinging oblique shock at the top (SBLI) replaces the top's extrapolation (tag 7)
    ymax_tag, shock = (2, 0.0) if shock_angle is None else (7, shock_angle)
    if shock_angle is not None:
        nr_top = 0
        if xshock_imp is None:
            xshock_imp = 0.6 * lx
    return f"""[grid]
grid_dim = 1
domain_size_x = {lx!r}
domain_size_y = {ly!r}
domain_size_z = {lz!r}
nxmax = {nx}
nymax = {ny}
nzmax = {nz}
ng = {max(3, ep_order // 2, weno_scheme)}
metrics_order = {ep_order}
grid_type = 4
jbgrid = {jbgrid!r}
dyptarget = {dyptarget!r}
nywr = {nywr}
lywr = {lywr!r}
ysmoosteps = {ysmoosteps}

[bc]
xmin = 10
xmax = 2
ymin = 6
ymax = {ymax_tag}
zmin = 0
zmax = 0
xmin_nr = 0
xmax_nr = {nr_outflow}
ymin_nr = 0
ymax_nr = {nr_top}
zmin_nr = 0
zmax_nr = 0
x_recyc = {x_recyc!r}
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
nkeep = 0
visc_order = {ep_order}
conservative_viscous = {conservative_viscous}
weno_scheme = {weno_scheme}
weno_version = {weno_version}
flux_splitting = {flux_splitting}
sensor_threshold = {sensor!r}
rk_type = 1
rand_type = {rand_type}

[flow]
flow_init = 1
Mach = {mach!r}
Reynolds = {reynolds_tau!r}
theta_wall = {theta_wall!r}
xshock_imp = {xshock_imp if xshock_imp is not None else 0.0!r}
shock_angle = {shock!r}
T_ref = 220.
aoa = 0.

[fluid]
gam = 1.4
Prandtl = 0.72
visc_model = {visc_model}
vt_exp = {vt_exp!r}
s_suth = 110.4
{_gas_keys(cp_poly)}

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
kind = bl_powerlaw
amp = {amp!r}
reynolds_delta = {reynolds_delta!r}
reynolds_tau = {reynolds_tau!r}
"""


# grid choices of the batched workload (48 boxes)
BATCH_NX = (64, 96, 128)
BATCH_NY = (64, 96)
BATCH_NZ = (32, 64, 96)


def batch_mix(nboxes: int = 48, seed: int = 2024) -> list[dict]:
    """The batched workload: per box a grid drawn from {64,96,128} x {64,96} x {32,64,96},
    bulk Mach uniform in [0.3, 2.0], bulk Reynolds uniform in [2000, 6000], and the benchmark
    channel's initial field (its own noise seed)."""
    rng = random.Random(seed)
    out = []
    for b in range(nboxes):
        out.append(dict(nx=rng.choice(BATCH_NX), ny=rng.choice(BATCH_NY), nz=rng.choice(BATCH_NZ),
                        mach=round(rng.uniform(0.3, 2.0), 6), re_bulk=round(rng.uniform(2000.0, 6000.0), 3),
                        seed=b + 1))
    return out


def shock_angle_for(mach: float, deflection_deg: float = 8.0, gam: float = 1.4) -> float:
    """Weak-shock angle [deg] of the theta-beta-Mach relation for a given flow deflection."""
    th = math.radians(deflection_deg)

    def f(b):
        return 2.0 / math.tan(b) * (mach ** 2 * math.sin(b) ** 2 - 1.0) / (mach ** 2 * (gam + math.cos(2 * b)) + 2.0) - math.tan(th)
    lo, hi = math.asin(1.0 / mach) + 1e-9, math.radians(64.0)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0.0:
            hi = mid
        else:
            lo = mid
    return math.degrees(0.5 * (lo + hi))


def serve_mix(nreq: int, rate_per_s: float, seed: int = 7, cells_min: int = 48 ** 3,
              cells_max: int = 384 * 192 * 128, steps=(200, 2000), mixed_fraction: float = 0.5,
              sbli_fraction: float = 0.3) -> list[dict]:
    """A Poisson stream of solve requests: arrival offsets with exponential gaps at rate_per_s;
    70 % channels and 30 % shock / boundary-layer interactions (an 8-degree impinging shock);
    grids log-uniform in cell count between cells_min and cells_max (aspect 2:1:1 rounded to
    multiples of 16); Mach uniform in [0.5, 2.5] (channels, bulk Mach) or [1.8, 2.5] (SBLI, where
    the 8-degree shock stays attached); step counts uniform in `steps`; FP64 or mixed precision."""
    rng = random.Random(seed)
    t = 0.0
    out = []
    for r in range(nreq):
        t += rng.expovariate(rate_per_s)
        cells = math.exp(rng.uniform(math.log(cells_min), math.log(cells_max)))
        base = (cells / 4.0) ** (1.0 / 3.0)
        nx = max(32, int(round(2 * base / 16)) * 16)
        ny = max(32, int(round(base / 16)) * 16)
        nz = max(32, int(round(base / 16)) * 16)
        sbli = rng.random() < sbli_fraction
        mach = round(rng.uniform(1.8, 2.5) if sbli else rng.uniform(0.5, 2.5), 6)
        req = dict(rid=r, arrival=t, nx=nx, ny=ny, nz=nz, mach=mach, nsteps=rng.randint(*steps),
                   precision=1 if rng.random() < mixed_fraction else 0)
        if sbli:
            req.update(kind="sbli", shock_angle=round(shock_angle_for(mach), 6))
        else:
            req.update(kind="channel", seed=r + 1)
        out.append(req)
    return out
