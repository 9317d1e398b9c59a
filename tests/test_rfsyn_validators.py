"""rfsyn's own validators and unit tests, compiled unmodified from its
sources and linked against librfsyn_fdtd_b200.so (oracle/Makefile target
`validators`), run on the GPU: every one must pass and print exactly what
it prints when linked against rfsyn's CPU engine (tests/golden/validators/,
made by tests/golden/make_golden.py).  The printed figures are rfsyn's
accuracy gates: CPML point and plane-wave reflection, Fresnel, energy
balance, probe DFT, oblique CPML, high contrast, long-term stability, the
tilted-slab measurement and the periodic energy audit."""
from __future__ import annotations

import subprocess
import tempfile
from pathlib import Path

import pytest

from tests.golden.make_golden import VALIDATOR_ARGS

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "oracle" / "_ref" / "validators"
GOLDEN = ROOT / "tests" / "golden" / "validators"


@pytest.mark.parametrize("name", sorted(VALIDATOR_ARGS))
def test_rfsyn_validator_on_gpu_matches_cpu_output(name):
    exe = BIN / name
    if not exe.exists():
        pytest.skip("rfsyn's validators were not built here (rfsyn sources absent at build time)")
    with tempfile.TemporaryDirectory() as wd:
        r = subprocess.run([str(exe), *VALIDATOR_ARGS[name]], cwd=wd, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout + r.stderr
    want = (GOLDEN / f"{name}.txt").read_text()
    assert r.stdout == want
