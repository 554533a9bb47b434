"""The C-ABI library: loads, exports every symbol the headers declare, validates inputs, and
fails loudly (no silent CPU path) when no device is present.  No compute without a GPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

from conftest import ROOT, channel_ini, gpu_available


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(streams_b200_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import streams_b200
    lib = C.CDLL(str(streams_b200.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(streams_b200.EXPORTED) <= set(names)


def test_library_build_targets_sm100a():
    """The build recipe compiles every CUDA source for sm_100a only (no other architecture, no
    PTX for JIT); the device-side check of the loaded image is test_loaded_kernels_are_sm100."""
    text = (ROOT / "streams-2_b200" / "Makefile").read_text()
    flags = re.findall(r"-gencode\s+arch=(\S+),code=(\S+)", text)
    assert flags and all(f == ("compute_100a", "sm_100a") for f in flags), flags


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="no CUDA device")
def test_loaded_kernels_are_sm100():
    """The kernels the driver loaded from the library are sm_100 binaries (binaryVersion 100,
    from cudaFuncGetAttributes on one kernel of every source file)."""
    import streams_b200
    streams_b200.Solver  # noqa: B018  (the library is mapped on first use)
    versions = (C.c_int * 8)()
    n = streams_b200.lib.streams_b200_kernel_binary_versions(versions, 8)
    assert n == 3, n
    assert all(versions[q] == 100 for q in range(n)), list(versions)[:n]


def test_abi_version():
    import streams_b200
    assert streams_b200.lib.streams_b200_abi_version() == 3


def test_case_load_and_params(tmp_path):
    import streams_b200
    case = streams_b200.Case(tmp_path, channel_ini(16, 12, 8))
    p = case.params()
    assert (p.nx, p.ny, p.nz, p.ng) == (16, 12, 8, 3)
    assert p.bctags[2] == 6 and p.bctags[3] == 6 and p.is_y_staggered == 1
    assert p.force_zero_flux[2] == 1 and p.force_zero_flux[3] == 1
    info = case.info()
    assert info["volchan"] == pytest.approx(2.0 * 16 * 8)
    w = case.field()
    assert w.shape == (5, 14, 18, 22)
    assert streams_b200.lib.streams_b200_footprint_bytes(C.byref(p)) > w.nbytes


def test_case_rejects_unsupported_input(tmp_path):
    import streams_b200
    bad = channel_ini(16, 12, 8).replace("flux_splitting = 0", "flux_splitting = 3")
    with pytest.raises(streams_b200.BackendError, match="flux_splitting"):
        streams_b200.Case(tmp_path, bad)
    bad = channel_ini(16, 12, 8).replace("rk_type = 1", "rk_type = 2")
    with pytest.raises(streams_b200.BackendError, match="rk_type"):
        streams_b200.Case(tmp_path, bad)
    with pytest.raises(streams_b200.BackendError, match="missing input key"):
        streams_b200.Case(tmp_path, "[grid]\nnxmax = 4\n")


def test_create_validates_parameters(tmp_path):
    import streams_b200
    case = streams_b200.Case(tmp_path, channel_ini(16, 12, 8))
    p = case.params()
    p.precision = 7
    with pytest.raises(streams_b200.BackendError) as e:
        streams_b200.Solver(p, case.grid())
    assert e.value.code == streams_b200.EINVAL


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_create_without_device_fails_loudly(tmp_path):
    import streams_b200
    case = streams_b200.Case(tmp_path, channel_ini(16, 12, 8))
    with pytest.raises(streams_b200.BackendError) as e:
        streams_b200.Solver(case.params(), case.grid())
    assert e.value.code == streams_b200.ENODEV


def test_grid_limits_fail_loudly(tmp_path):
    """The x pass's launch grid bounds ny (4 rows per block row) and nz (one grid plane each);
    create rejects larger blocks before touching the device."""
    from streams_b200 import BackendError, Case, Solver
    from streams_b200.cases import channel_ini
    case = Case(tmp_path, channel_ini(16, 12, 8))
    for field, value in (("nz", 65536), ("ny", 4 * 65535 + 1)):
        p = case.params()
        setattr(p, field, value)
        with pytest.raises(BackendError, match="at most"):
            Solver(p, case.grid())
