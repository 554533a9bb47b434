"""The committed FP64 operation counts (profiles/fp64_flops.json, read by bench.py for the FP64
roofline of the flux passes) are what the oracle's face-flux code counts today."""
import json

from conftest import ROOT


def test_committed_flop_counts_match_the_oracle():
    import sys
    sys.path.insert(0, str(ROOT / "oracle"))
    import count_flops
    committed = json.loads((ROOT / "profiles" / "fp64_flops.json").read_text())
    for name, args in count_flops.SCHEMES.items():
        assert committed["schemes"][name] == count_flops.face_counts(*args), name
    # a WENO face costs several central faces (the characteristic projection of 2 WS points and
    # five reconstructions against 3 l-levels of split-form pairs)
    c = committed["schemes"]["weno5_central6"]
    assert 3 * c["central_face"]["flops"] < c["weno_face"]["flops"] < 10 * c["central_face"]["flops"]
