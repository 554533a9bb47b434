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


def channel_ini(*args, **kwargs) -> str:
    """The package's synthetic channel input file (streams_b200.cases.channel_ini)."""
    from streams_b200.cases import channel_ini as build
    return build(*args, **kwargs)


@pytest.fixture(scope="session")
def golden():
    import json
    d = ROOT / "tests" / "golden"
    return {"ini": (d / "subsonic_channel.ini").read_text(),
            "row": json.loads((d / "subsonic_channel.json").read_text())["expected"]}


requires_gpu = pytest.mark.skipif(not gpu_available(), reason="no CUDA device")
