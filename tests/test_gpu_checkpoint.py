"""Checkpoint dump and restart (no counterpart in the reference): a run
split by a save and a load into a fresh solver continues where it stopped."""

from __future__ import annotations

import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, load_config
from gpu_common import STATE_FIELDS, cylinder_case, rel_field_err

pytestmark = pytest.mark.gpu


def _solver(cfg, xy, nr, nt, **kw):
    from purinecfd_b200 import Solver
    return Solver(cfg, xy, nr, nt, **kw)


@pytest.mark.parametrize("kind", ["fused_fp64", "passes", "fused_split"])
def test_restart_continues_the_run(tmp_path, kind):
    from purinecfd_b200 import PATH_FUSED, PATH_PASSES, PREC_FP32_SPLIT, PREC_FP64
    kw = {"fused_fp64": dict(kernel_path=PATH_FUSED, precision=PREC_FP64),
          "passes": dict(kernel_path=PATH_PASSES, precision=PREC_FP64),
          "fused_split": dict(kernel_path=PATH_FUSED, precision=PREC_FP32_SPLIT)}[kind]
    # FP32 split: the uninterrupted run carries the last stage's FP32 V/dt into
    # the next step, the restarted one re-derives it from U in FP64, so the
    # two agree to FP32 rounding (the split path's own tolerance is 1e-5)
    tol = 1e-5 if kind == "fused_split" else 1e-12
    cfg, xy, nr, nt = cylinder_case()
    a = _solver(cfg, xy, nr, nt, **kw)
    a.run(20)
    b = _solver(cfg, xy, nr, nt, **kw)
    b.run(10)
    ck = tmp_path / "state.ckpt"
    b.save_checkpoint(ck)
    c = _solver(cfg, xy, nr, nt, **kw)
    c.load_checkpoint(ck)
    assert c.step == 10 and abs(c.totaltime - b.totaltime) <= 1e-15 * b.totaltime
    c.run(10)
    assert c.step == 20
    assert abs(c.totaltime - a.totaltime) <= tol * a.totaltime
    for name in STATE_FIELDS:
        assert rel_field_err(c.get(name), a.get(name)) < tol, name


def test_checkpoint_rejects_other_mesh_and_damaged_files(tmp_path):
    from purinecfd_b200 import JstError
    cfg, xy, nr, nt = cylinder_case()
    a = _solver(cfg, xy, nr, nt)
    a.run(2)
    ck = tmp_path / "a.ckpt"
    a.save_checkpoint(ck)
    cfg2, xy2, nr2, nt2 = cylinder_case(33, 64)
    other = _solver(cfg2, xy2, nr2, nt2)
    with pytest.raises(JstError):
        other.load_checkpoint(ck)
    cut = tmp_path / "cut.ckpt"
    cut.write_bytes(ck.read_bytes()[:100])
    with pytest.raises(JstError):
        a.load_checkpoint(cut)
    with pytest.raises(JstError):
        a.load_checkpoint(tmp_path / "missing.ckpt")


def test_cli_restart_continues_step_numbering(tmp_path):
    jst = ROOT / "purinecfd_b200" / "bin" / "jst"
    base = [str(jst), "--mesh", str(GOLDEN / "fangdata.txt"), "--config", str(GOLDEN / "config.json")]
    ck = tmp_path / "run.ckpt"
    p1 = subprocess.run(base + ["--steps", "6", "--checkpoint", str(ck), "--out", str(tmp_path / "a.csv"),
                                "--reslog", str(tmp_path / "a.log")], capture_output=True, text=True, timeout=300)
    assert p1.returncode == 0, p1.stderr
    p2 = subprocess.run(base + ["--steps", "6", "--restart", str(ck), "--out", str(tmp_path / "b.csv"),
                                "--reslog", str(tmp_path / "b.log")], capture_output=True, text=True, timeout=300)
    assert p2.returncode == 0, p2.stderr
    steps = [int(m) for m in re.findall(r"^step:\s+(\d+) \|", p2.stdout, re.M)]
    assert steps == list(range(7, 13))
    p3 = subprocess.run(base + ["--steps", "12", "--out", str(tmp_path / "c.csv"), "--reslog", str(tmp_path / "c.log")],
                        capture_output=True, text=True, timeout=300)
    assert p3.returncode == 0, p3.stderr
    b = np.loadtxt(tmp_path / "b.csv", delimiter=",", skiprows=1)
    c = np.loadtxt(tmp_path / "c.csv", delimiter=",", skiprows=1)
    assert np.allclose(b, c, rtol=1e-8, atol=0.0)
    assert (tmp_path / "b.log").read_text().splitlines()[1].startswith("7,")
