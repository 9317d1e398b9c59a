"""Generates the golden fixtures of tests/golden/ from rfsyn itself.

rfsyn's engine sources are compiled in place (oracle/Makefile, target
`ref`) into oracle/_ref/librfsyn_ref.so together with oracle/scene_driver.c,
which replays a scene through rfsyn's own public API (fdtd_grid_create,
cpml_create, materials_*, source_apply, fdtd_update_*, probe_*).  Each case
below is run there and its outputs saved as .npz.  Run in the container that
has rfsyn's sources:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from tests.cases import CASES, c1_scene, simulate_unit_cfg  # noqa: E402

OUT = Path(__file__).resolve().parent


def main() -> None:
    oracle.build(ref=True)
    if not oracle.ref_available():
        raise SystemExit("rfsyn sources not found: cannot regenerate golden fixtures")
    # rfsyn's own fdtd_simulate_echo on tests/simulate_unit.c's configuration
    cfg = simulate_unit_cfg()
    rc, td, fs = oracle.ref_simulate_echo(cfg)
    assert rc == 0
    np.savez_compressed(OUT / "simulate_unit.npz", td=td, fs=fs)
    for name, scene in CASES.items():
        r = oracle.run_ref(scene)
        np.savez_compressed(OUT / f"{name}.npz", td=r["td"], dft=r["dft"])
        print(name, r["td"].shape, float(np.abs(r["td"]).max()))
    r = oracle.run_ref(c1_scene())
    np.savez_compressed(OUT / "c1.npz", td=r["td"], dft=r["dft"])
    print("c1", r["td"].shape, float(np.abs(r["td"]).max()))
    validators()


# rfsyn's validators and unit tests with the arguments its CTest passes
# (CMakeLists.txt:266-305; stability at the minimum RFSYN_STABILITY_STEPS)
VALIDATOR_ARGS = {
    "simulate_unit": [], "materials_unit": [], "materials_tensor_unit": [], "periodic_materials_unit": [],
    "periodic_wrapping_unit": [], "validate_cpml": [], "validate_cpml_margin": [], "validate_cpml_planewave": [],
    "validate_materials_fresnel": [], "validate_probe_dft": [], "validate_materials_energy": [],
    "validate_cpml_oblique": [], "validate_materials_high_contrast": ["--full"],
    "validate_long_term_stability": ["--steps", "10000"], "validate_materials_tilted": [],
    "audit_periodic_energy": [], "subpixel_te_unit": [],
}


def validators() -> None:
    """stdout of rfsyn's validators linked against rfsyn itself."""
    import subprocess
    import tempfile

    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "validators_ref"], check=True)
    dst = OUT / "validators"
    dst.mkdir(exist_ok=True)
    for name, args in VALIDATOR_ARGS.items():
        with tempfile.TemporaryDirectory() as wd:
            r = subprocess.run([str(ROOT / "oracle" / "_ref" / "validators_ref" / name), *args], cwd=wd,
                               capture_output=True, text=True, timeout=1800)
        assert r.returncode == 0, (name, r.stdout, r.stderr)
        (dst / f"{name}.txt").write_text(r.stdout)
        print(name, "ok", len(r.stdout.splitlines()), "lines")


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "validators":
        validators()
    else:
        main()
