"""Generates the golden fixtures in this directory from the unmodified
reference (oracle/_ref, built by `make -C oracle` from the reference sources).

    python tests/golden/make_golden.py

Each fixture holds the configuration (JSON), and after the stated number of
steps the reference's zeta (Ooura layout, NX*NY*NZ_ doubles per component),
uk_dc, and the particle records (x, v, omega, f_hydro_previous,
torque_hydro_previous, fr_previous, x_nopbc, q).  fft_16.npz holds A2a_k of a
seeded random 16x32x8 field.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref, udf  # noqa: E402

CASES = {
    "ns32_dense_kbt": (dict(np_xyz=(5, 5, 5), n=6, seed=11, kbt=1e-3, min_gap=0.2), 5),
    "ns32_rot_off": (dict(np_xyz=(5, 5, 5), n=4, seed=7, kbt=1e-3, rotation="OFF"), 4),
    "ns_16x32x64_gravity_fixcell": (dict(np_xyz=(4, 5, 6), n=3, seed=5, kbt=0.0, gravity_g=0.5, mass_ratio=1.5,
                                         fix_cell=(True, False, True)), 4),
}


EL_CASES = {
    "el32_efield_x": (dict(np_xyz=(5, 5, 5), n=2, seed=3, surface_charge=-100.0, efield=(0.05, 0.0, 0.0)), 3),
    "el_16x32x64_pos": (dict(np_xyz=(4, 5, 6), n=3, seed=5, surface_charge=50.0, min_gap=0.5), 3),
}


def make_cfg(spec):
    spec = dict(spec)
    fc = spec.pop("fix_cell", None)
    cfg = udf.ns_config(spec.pop("np_xyz"), spec.pop("n"), **spec)
    if fc is not None:
        cfg["fix_cell"] = fc
    return cfg


def main():
    for name, (spec, steps) in CASES.items():
        cfg = make_cfg(spec)
        r = ref.RefSim(cfg)
        r.step(steps)
        p = r.particles()
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), cfg=json.dumps(cfg), steps=steps, zeta=r.zeta(),
                            uk_dc=r.uk_dc(), **{f"p_{k}": v for k, v in p.items()})
        print(name, "written")
    for name, (spec, steps) in EL_CASES.items():
        spec = dict(spec)
        cfg = udf.electrolyte_config(spec.pop("np_xyz"), spec.pop("n"), **spec)
        r = ref.RefSim(cfg)
        r.step(steps)
        p = r.particles()
        conc = np.stack([r.field(20), r.field(21)])
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), cfg=json.dumps(cfg), steps=steps, zeta=r.zeta(),
                            uk_dc=r.uk_dc(), conc=conc, **{f"p_{k}": v for k, v in p.items()})
        print(name, "written")
    cfg = udf.ns_config((4, 5, 3), 1, seed=1)
    r = ref.RefSim(cfg)
    a = np.random.default_rng(0).standard_normal((r.NX, r.NY, r.NZ))
    np.savez_compressed(os.path.join(HERE, "fft_16x32x8.npz"), cfg=json.dumps(cfg), a=a, a_k=r.A2a_k(a),
                        sekibun=r.sekibun())


if __name__ == "__main__":
    main()
