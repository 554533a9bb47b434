"""Generate the golden fixtures of the reference's own regression suite.

The STREAmS-2 regression runner (tests/run_all_tests.py of the reference) copies an example
input, patches it with Python's configparser and compares the last row of progress.out with the
row stored in tests/tests.ini.  This script reproduces that patching for the Cartesian case
``subsonic_channel`` and writes:

  subsonic_channel.ini   the patched input (values only, comments dropped)
  subsonic_channel.json  the expected 14-column progress row and its tolerance
  supersonic_bl.ini,     the reference's boundary-layer and shock-interaction example inputs
  supersonic_sbli.ini    (init_bl with hasan_meanprofile and add_synthetic_perturbations), with the
                         grid reduced to 256 x 64 x 32 (nywr 40) and 10 steps so a test runs them

The runner splits each patch on the first ',' of every ';'-separated item, so the item
``controls,num_iter=10,controls,rand_type=0`` sets num_iter to "10,controls,rand_type=0"
(read back as 10 by Fortran list-directed input) and leaves rand_type at its example value.

Usage:  python tests/golden/make_golden.py <reference root>   (the STREAmS-2 source tree)
"""
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def parse_ini(text):
    sections, order, cur = {}, [], None
    for raw in text.splitlines():
        s = raw.strip()
        if not s or s[0] in "#;":
            continue
        if s.startswith("["):
            cur = s[1:s.index("]")].strip()
            if cur not in sections:
                sections[cur] = {}
                order.append(cur)
            continue
        if "=" in s and cur is not None:
            k, v = s.split("=", 1)
            v = v.split(";")[0].strip()
            sections[cur][k.strip()] = v
    return sections, order


def patch_items(line):
    items = []
    for pair in line.split(";"):
        section, rest = pair.split(",", 1)
        key, value = rest.split("=", 1)
        items.append((section.strip(), key.strip(), value.strip()))
    return items


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the STREAmS-2 source tree>")
    ref = Path(sys.argv[1])
    tests = (ref / "tests" / "tests.ini").read_text().splitlines()
    tests = [t.strip() for t in tests if t.strip()]
    i = tests.index("[subsonic_channel]")
    patches, expected = tests[i + 1], [float(x) for x in tests[i + 2].split()]
    sections, order = parse_ini((ref / "examples" / "subsonic_channel" / "singleideal.ini").read_text())
    for sec, key, val in patch_items(patches):
        sections.setdefault(sec, {})[key] = val
    out = []
    for sec in order:
        out.append(f"[{sec}]")
        out += [f"{k} = {v}" for k, v in sections[sec].items()]
        out.append("")
    (HERE / "subsonic_channel.ini").write_text("\n".join(out))
    (HERE / "subsonic_channel.json").write_text(json.dumps({
        "case": "subsonic_channel",
        "source": "reference tests/tests.ini [subsonic_channel]; reference runner tolerance 1e-12 absolute",
        "columns": ["icyc", "dt", "time", "residual_rhou", "-dpdx/dt", "rhobulk", "ubulk", "tbulk",
                    "rhomin", "rhomax", "tmin", "tmax", "pmin", "pmax"],
        "expected": expected,
    }, indent=1))
    print("wrote", HERE / "subsonic_channel.ini", HERE / "subsonic_channel.json")
    for ex in ("supersonic_bl", "supersonic_sbli"):
        sections, order = parse_ini((ref / "examples" / ex / "singleideal.ini").read_text())
        reduced = {("grid", "nxmax"): "256", ("grid", "nymax"): "64", ("grid", "nzmax"): "32",
                   ("grid", "nywr"): "40", ("controls", "num_iter"): "10", ("output", "print_control"): "1"}
        for (sec, key), val in reduced.items():
            sections[sec][key] = val
        out = []
        for sec in order:
            out.append(f"[{sec}]")
            out += [f"{k} = {v}" for k, v in sections[sec].items()]
            out.append("")
        (HERE / f"{ex}.ini").write_text("\n".join(out))
        print("wrote", HERE / f"{ex}.ini")


if __name__ == "__main__":
    main()
