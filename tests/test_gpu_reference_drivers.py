"""Drop-in check with the reference's own callers: the reference's test drivers
(test/test_sgsknn.c, test/test_dgsknn.c, test/test_sgsknn_stl.cpp, test/test_dgsknn_stl.cpp),
unchanged, compiled against this repository's include/ and linked to rnn_b200/libgsknn.so by
``make -C oracle drivers`` into oracle/_ref/ (the build step does this where the reference
sources are present).

Each driver builds a heap with heapCreate_{s,d}, runs {s,d}gsknn through heap_t, runs the
reference algorithm ({s,d}gsknn_ref or the STL form) into plain arrays, and prints one line per
set difference that is not an exact tie with the row's k-th distance (test/test_sgsknn.c:13-60),
then a GFLOPS line. Here every call is this library's. Passing means no mismatch line beyond
floating-point rounding of the k-th distance, no "bug" line, and the GFLOPS line printed.
"""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_OUT = os.path.join(ROOT, "oracle", "_ref")
MISMATCH = re.compile(r"^\(([^,]+),([^,]+),(\d+),(\d+),([^,]+),([12]),(-?\d+)\)$")

CASES = [  # (driver, m, n, d, r, relative tolerance at the k-th distance)
    ("test_dgsknn.x", 4096, 4096, 32, 16, 1e-12),
    ("test_dgsknn.x", 3000, 1000, 100, 64, 1e-12),
    ("test_dgsknn_stl.x", 2048, 2048, 16, 10, 1e-12),
    ("test_sgsknn.x", 4096, 4096, 64, 32, 1e-5),
    ("test_sgsknn.x", 5000, 777, 300, 100, 1e-5),
    ("test_sgsknn_stl.x", 2048, 2048, 16, 10, 1e-5),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}x{c[2]}-d{c[3]}-k{c[4]}")
def test_reference_driver(case):
    exe, m, n, d, r, tol = case
    path = os.path.join(REF_OUT, exe)
    if not os.path.exists(path):
        pytest.skip(f"{exe} not built (make -C oracle drivers needs the reference sources)")
    out = subprocess.run([path, str(m), str(n), str(d), str(r)], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln.strip() for ln in out.stdout.strip().splitlines()]
    assert lines and re.search(r"GFLOPS;$", lines[-1]), out.stdout[-2000:]
    assert re.match(rf"{m},\s+{n},\s+{d},\s+{r},", lines[-1]), lines[-1]
    assert not any(ln.strip() == "bug" for ln in lines)
    worst = 0.0
    for ln in lines[:-1]:
        mt = MISMATCH.match(ln.strip())
        assert mt, f"unexpected output line: {ln!r}"
        root = float(mt.group(1)) if mt.group(6) == "1" else float(mt.group(2))
        member = float(mt.group(5))
        worst = max(worst, abs(member - root) / max(abs(root), 1e-30))
    assert worst <= tol, f"set difference beyond rounding: relative gap {worst:.3e}"
    print(f"{exe} {m}x{n} d={d} k={r}: {len(lines) - 1} near-tie lines, {lines[-1].strip()}")
