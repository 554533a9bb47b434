"""Exact FP64 operation counts of the hybrid face flux, through the oracle's own code.

The oracle's face flux (euler_*_hybrid_kernel of kernels_cpu.F90 with compute_roe_average,
eigenvectors_* and wenorec_1d) is instantiated with the counting scalar of oracle/flops.hpp and
evaluated at interior faces of a small developed channel: once with every face a WENO face
(sensor threshold < 0) and once with every face central (threshold > 1).  The counts do not
depend on the data or the direction (no data-dependent branches at interior faces; checked over
all three directions).  Writes profiles/fp64_flops.json, which bench.py reads for the FP64
roofline of the flux passes, and which tests/test_flop_count.py checks against the oracle.

    python oracle/count_flops.py            (from the repository root)

Measurement infrastructure: it runs the oracle, never the product.
"""
from __future__ import annotations

import json
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "oracle", ROOT / "streams-2_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

# the flux schemes the benchmark and the tests run: (weno_scheme, ep_order, weno_version)
SCHEMES = {"weno5_central6": (3, 6, 0), "weno5z_central6": (3, 6, 1), "weno3_central4": (2, 4, 0),
           "weno7_central8": (4, 8, 0)}


def face_counts(weno_scheme: int, ep_order: int, weno_version: int) -> dict:
    from oracle_py import Oracle
    from streams_b200.cases import channel_ini
    out = {}
    for kind, sensor in (("weno_face", -1.0), ("central_face", 1.01)):
        with tempfile.TemporaryDirectory() as d:
            o = Oracle(d, channel_ini(nx=20, ny=16, nz=12, sensor=sensor, weno_scheme=weno_scheme,
                                      ep_order=ep_order, weno_version=weno_version))
            o.init_run()
            o.run(1)
            counts = [o.face_flops(direction, 10, 8, 6) for direction in range(3)]
        if any(c != counts[0] for c in counts):
            raise RuntimeError(f"face counts differ between directions: {counts}")
        out[kind] = counts[0]
    return out


def main() -> int:
    res = {"source": "oracle/count_flops.py: face_flux_t<Counted> of the oracle (oracle/flops.hpp) at an interior "
                     "face of a developed 20x16x12 channel, all faces WENO or all central",
           "conventions": "+, -, *, / and sqrt one operation each; an FMA counts two; fabs, sign changes and "
                          "constants of the case count nothing; max and comparisons are 'cmp', not flops",
           "divergence_per_cell_per_direction": 10,
           "schemes": {name: face_counts(*args) for name, args in SCHEMES.items()}}
    path = ROOT / "profiles" / "fp64_flops.json"
    path.write_text(json.dumps(res, indent=1) + "\n")
    print("wrote", path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
