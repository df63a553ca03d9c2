"""The row spans of the binning hit test (tomo_shell2026_b200/csrc/tomo_span.cuh)
on the host: tests/span_check.cpp compiles the same header with g++ (IEEE
single precision, no contraction) and, for random small, large, sliver,
axis-aligned and almost collinear triangles, checks that every box pixel the
kernels' float pre-reject passes lies inside its column's span.  A hit outside
the spans would be missed by the hit test, so this is the spans' exactness
condition; the GPU parity tests then cover the kernel that uses them."""
from __future__ import annotations

import re
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
@pytest.mark.parametrize("seed", [11, 12])
def test_spans_cover_every_prereject_pass(tmp_path, seed):
    exe = tmp_path / "span_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", str(HERE / "span_check.cpp"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), "150000", str(seed)], capture_output=True, text=True)
    line = out.stdout.strip().splitlines()[-1]
    m = dict(zip(*[iter(line.split())] * 2))
    assert out.returncode == 0 and int(m["violations"]) == 0, out.stdout[-2000:]
    n_pass, span, box = int(m["passed"]), int(m["span_items"]), int(m["box_items"])
    assert n_pass > 0
    # the spans hold every passing pixel and little else: far fewer items than the boxes
    assert n_pass <= span < 0.5 * box
