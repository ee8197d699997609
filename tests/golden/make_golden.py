#!/usr/bin/env python3
"""Regenerate the golden fixtures in this directory from the reference.

Run where a checkout of the reference is available and pass its root
directory with --reference; nothing at test time reads the reference, only
the files written here.

What it writes:

* ``config.json`` — the reference's sample configuration (the values every
  golden case was produced with).
* ``fangdata.txt``, ``cyl_17x40.txt`` — the reference's two bundled O-meshes,
  produced by this package's own generator (purinecfd_b200.meshgen) and checked
  byte-for-byte against the reference's files.
* ``cyl_10x12.json``, ``cyl_17x40.json`` — the reference's own golden data
  (exported by its jst-py/tools/dump_golden.py; read by its jst-rs/tests/golden.rs
  and tests/test_regression.py).  Before writing, each file is re-derived by
  running the reference's exporter live and the two are compared field by
  field (agreement to ~1e-14 of the field scale; the residue is numpy
  summation order).
* ``ell_13x40_a5.json`` — an extra case made by running the reference's
  exporter live on a stretched ellipse mesh (13 rings x 40, stretch 1.15) at
  AOA = 5 deg, Ma = 0.5 (a copy of jst-py with that config.json, in a temp dir),
  so that v_inf != 0 and a different Mach number are pinned too.  Its mesh is
  written as ``ell_13x40.txt``.

Usage: python tests/golden/make_golden.py --reference <root of the reference checkout>
"""

from __future__ import annotations

import argparse
import json
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from purinecfd_b200 import meshgen  # noqa: E402

EXPORT_SNIPPET = r"""
import json, sys
sys.path.insert(0, '.')
from tools import dump_golden as dg
doc = dg.build(sys.argv[1], int(sys.argv[2]), int(sys.argv[3]))
json.dump(doc, open(sys.argv[4], 'w'))
"""


def run_exporter(jstpy: Path, mesh: Path, steps: int, warmup: int) -> dict:
    with tempfile.TemporaryDirectory() as td:
        out = Path(td) / "g.json"
        subprocess.run([sys.executable, "-c", EXPORT_SNIPPET, str(mesh), str(steps), str(warmup), str(out)],
                       cwd=jstpy, check=True, capture_output=True)
        return json.loads(out.read_text())


def max_dev(a: dict, b: dict) -> float:
    worst = 0.0
    for sec in ("geometry", "init", "terms", "final"):
        for k, v in b[sec].items():
            if isinstance(v, list):
                x, y = np.asarray(a[sec][k], float), np.asarray(v, float)
                sc = np.max(np.abs(y)) or 1.0
                worst = max(worst, float(np.max(np.abs(x - y)) / sc))
            elif isinstance(v, float):
                worst = max(worst, abs(a[sec][k] - v) / (abs(v) or 1.0))
    return worst


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root directory of the reference checkout")
    args = ap.parse_args()
    ref = Path(args.reference)
    jstpy = ref / "jst-py"

    cfg = json.loads((ref / "config.json").read_text())
    (HERE / "config.json").write_text(json.dumps(cfg, indent=4) + "\n")

    meshes = {
        "fangdata.txt": (meshgen.ellipse_o_mesh(10, 12), 10, 12, ref / "fangdata.txt"),
        "cyl_17x40.txt": (meshgen.ellipse_o_mesh(17, 40, stretch=1.12), 17, 40, ref / "meshes" / "cyl_17x40.txt"),
    }
    for name, (pts, nr, nt, ref_path) in meshes.items():
        text = meshgen.format_mesh(pts, nr, nt)
        assert text == ref_path.read_text(), f"{name}: generator does not reproduce the reference mesh"
        (HERE / name).write_text(text)
        print(f"{name}: identical to the reference's file")

    for gname, mesh in (("cyl_10x12.json", ref / "fangdata.txt"), ("cyl_17x40.json", ref / "meshes" / "cyl_17x40.txt")):
        want = json.loads((ref / "tests" / "golden" / gname).read_text())
        live = run_exporter(jstpy, mesh, want["meta"]["steps"], want["meta"]["warmup"])
        dev = max_dev(live, want)
        assert dev < 1e-12, f"{gname}: live exporter deviates by {dev:e}"
        (HERE / gname).write_text(json.dumps(want, indent=0) + "\n")
        print(f"{gname}: reference golden, live re-export agrees to {dev:.2e} of field scale")

    # Extra live case: stretched ellipse, AOA 5 deg, Ma 0.5.
    pts = meshgen.ellipse_o_mesh(13, 40, stretch=1.15)
    mesh_text = meshgen.format_mesh(pts, 13, 40)
    (HERE / "ell_13x40.txt").write_text(mesh_text)
    cfg2 = json.loads(json.dumps(cfg))
    cfg2["simulation"]["AOA"] = 5.0
    cfg2["simulation"]["Ma"] = 0.5
    with tempfile.TemporaryDirectory() as td:
        tp = Path(td) / "jst-py"
        shutil.copytree(jstpy, tp, ignore=shutil.ignore_patterns("tests", "*.ipynb", "__pycache__"))
        (tp / "config.json").write_text(json.dumps(cfg2, indent=4))
        (tp / "ell_13x40.txt").write_text(mesh_text)
        doc = run_exporter(tp, tp / "ell_13x40.txt", 12, 2)
    doc["meta"]["mesh"] = "ell_13x40.txt"
    doc["meta"]["config_overrides"] = {"simulation": {"AOA": 5.0, "Ma": 0.5}}
    (HERE / "ell_13x40_a5.json").write_text(json.dumps(doc, indent=0) + "\n")
    print("ell_13x40_a5.json: live export from the reference's jst-py")


if __name__ == "__main__":
    main()
