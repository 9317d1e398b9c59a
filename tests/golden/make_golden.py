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


if __name__ == "__main__":
    main()
