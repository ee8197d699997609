"""The `jst` command-line front end keeps the reference CLI's flags, stdout
lines and output files (jst-rs/src/bin/jst.rs:58-125, solver.rs:229-255)."""

from __future__ import annotations

import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, load_config

import jst_oracle as jo

pytestmark = pytest.mark.gpu

JST = ROOT / "purinecfd_b200" / "bin" / "jst"


def rust_exp(v: float, prec: int) -> str:
    """Rust `{:.Pe}` formatting."""
    m, e = f"{v:.{prec}e}".split("e")
    return f"{m}e{int(e)}"


@pytest.mark.parametrize("path", ["fused", "passes"])
def test_cli_outputs_match_reference_formats_and_oracle(tmp_path, path):
    steps = 12
    cmd = [str(JST), "--mesh", str(GOLDEN / "fangdata.txt"), "--config", str(GOLDEN / "config.json"), "--steps",
           str(steps), "--out", str(tmp_path / "result.csv"), "--reslog", str(tmp_path / "res.log"), "--path", path]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    out = p.stdout
    assert "mesh " in out and "10 rings x 12 points -> 108 cells" in out
    assert len(re.findall(r"^step:\s+\d+ \| residual:", out, re.M)) == steps
    wall = re.search(r"wall clock:\s+([0-9.]+) s", out)       # jst-py/tools/benchmark.py's regexes
    fres = re.search(r"final residual:\s+([0-9.eE+-]+)", out)
    assert wall and fres
    assert f"all data is written in {tmp_path / 'result.csv'}" in out

    o = jo.OracleSolver(load_config(), *(lambda r: (r[2], r[0], r[1]))(jo.parse_mesh((GOLDEN / "fangdata.txt").read_text())))
    _, _, _, _, hist = o.run(steps, history=True)
    lines = (tmp_path / "res.log").read_text().splitlines()
    assert lines[0] == "step,residual" and len(lines) == steps + 1
    for k, ln in enumerate(lines[1:], start=1):
        a, b = ln.split(",")
        assert int(a) == k
        assert re.fullmatch(r"-?\d\.\d{6}e-?\d+", b), b
        assert abs(float(b) - hist[k - 1]) <= 5e-7 * hist[k - 1]
    assert fres.group(1) == rust_exp(float(lines[-1].split(",")[1]), 6)

    rows = (tmp_path / "result.csv").read_text().splitlines()
    assert rows[0] == "i,j,x,y,rho,p,T,u,v,miubl"
    assert len(rows) == 1 + 108
    want = {n: o.get(n) for n in ("cx", "cy", "rho", "p", "T", "u", "v", "nut")}
    for r in rows[1:]:
        f = r.split(",")
        i, j = int(f[0]) - 1, int(f[1]) - 1
        for col, name in zip(f[2:], ("cx", "cy", "rho", "p", "T", "u", "v", "nut")):
            assert re.fullmatch(r"-?\d\.\d{8}e-?\d+", col), col
            w = want[name][i, j]
            scale = np.max(np.abs(want[name]))
            assert abs(float(col) - w) <= 1e-8 * scale + 6e-9 * abs(w), (name, col, w)
        # geometry columns are exact: the same FP64 numbers, formatted like Rust
        assert f[2] == rust_exp(want["cx"][i, j], 8) and f[3] == rust_exp(want["cy"][i, j], 8)


def test_cli_reports_mesh_errors(tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("not a header\n1.0 2.0\n")
    p = subprocess.run([str(JST), "--mesh", str(bad), "--config", str(GOLDEN / "config.json")], capture_output=True,
                       text=True, timeout=120)
    assert p.returncode == 1 and "bad header" in p.stderr
