"""The link-time drop-in of the reference's solver entry points.

oracle/Makefile.ref (target ``gpu``) relinks the reference's own ``fem``
executable with ufem_b200/dropin/fem_eqs_gpu.c, which defines femEqsCGwJ,
femEqsCGwSSOR and femEqsBiCCSwJ (fem/fem_math.h:150-152) on top of
libufem_gpu.so; fem_eqs.o's CPU versions are weakened, so femSolve
(fem/fem_sol.c:1722-1730) calls the GPU solvers unchanged.  Each case runs
``fem -p -i in.fem -o out.res`` with the CPU build and with the relinked one,
for the default Jacobi PCG, ``-ssor`` and ``-nes``, and compares the two
result files token by token: the same tokens, integers equal, real numbers
within the file's printed precision (6 digits after the point: 2e-6
relative) or, for values near zero, 1e-9 of the file's largest magnitude.
"""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
CPU_FEM = os.path.join(ROOT, "oracle", "_ref", "serial", "fem")
GPU_FEM = os.path.join(ROOT, "oracle", "_ref", "gpu", "fem")
NUM = re.compile(r"^[-+]?(\d+\.\d*|\.\d+|\d+)([eE][-+]?\d+)?$")


def _tokens(path):
    return open(path).read().split()


def _compare(a_path, b_path):
    a, b = _tokens(a_path), _tokens(b_path)
    assert len(a) == len(b), (len(a), len(b))
    fa = [float(x) for x in a if NUM.match(x) and ("." in x or "e" in x.lower())]
    scale = max([abs(v) for v in fa] + [1e-300])
    worst = 0.0
    for x, y in zip(a, b):
        if x == y:
            continue
        assert NUM.match(x) and NUM.match(y), (x, y)
        assert ("." in x or "e" in x.lower()), ("integer token differs", x, y)
        u, v = float(x), float(y)
        d = abs(u - v)
        assert d <= 2e-6 * max(abs(u), abs(v)) or d <= 1e-9 * scale, (x, y)
        worst = max(worst, d / max(abs(u), abs(v), 1e-9 * scale))
    return worst


def _cases(tmp_path):
    from ufem_b200 import meshgen as mg
    out = []
    for name, m in (("plate_64x16", mg.plate_quad()),
                    ("beam_10x3x3", mg.beam_brick(10, 3, 3, 4.0, 1.0, 1.0, distort=0.1, seed=3))):
        p = str(tmp_path / f"{name}.fem")
        mg.write_fem(m, p)
        out.append((name, p))
    return out


@pytest.mark.parametrize("flags", [[], ["-ssor"], ["-nes"]], ids=["cgwj", "ssor", "bicgs"])
def test_relinked_fem_matches_the_cpu_fem(tmp_path, flags):
    if not (os.path.exists(CPU_FEM) and os.path.exists(GPU_FEM)):
        pytest.fail("reference builds missing: run __graft_entry__.build() (oracle/Makefile.ref all gpu)")
    for name, inp in _cases(tmp_path):
        res = {}
        for kind, exe in (("cpu", CPU_FEM), ("gpu", GPU_FEM)):
            out = str(tmp_path / f"{name}_{kind}.res")
            r = subprocess.run([exe, "-p", *flags, "-i", inp, "-o", out], capture_output=True, text=True, timeout=600)
            assert r.returncode == 0, (kind, name, r.stdout[-500:], r.stderr[-500:])
            res[kind] = out
        _compare(res["cpu"], res["gpu"])
