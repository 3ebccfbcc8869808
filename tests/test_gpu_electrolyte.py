"""GPU parity of the Electrolyte branch (two ion species, Nernst-Planck,
Poisson, Coulomb force) against the oracle.

Tolerances: FP64 path relative error <= 1e-10 (zeta, concentrations,
particle velocities); mixed path zeta / concentration <= 1e-4 relative after
the stated steps."""
import numpy as np
import pytest

from oracle import spm, udf

pytestmark = pytest.mark.gpu


def rel(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (n if n > 0 else 1.0)


def _run(cfg, nsteps, precision, efield_switch=None):
    import kapsel_old_b200 as kg

    g = kg.Simulation(cfg, precision=precision)
    o = spm.ElectrolyteOracle(cfg)
    worst = {}
    for s in range(nsteps):
        if efield_switch is not None and s == efield_switch[0]:
            g.set_efield(efield_switch[1])
            o.set_efield(efield_switch[1])
        g.step(1)
        o.step()
        zt = np.stack([o.S.truncate(o.zeta[d]) for d in range(2)])
        ct = np.stack([o.S.truncate(o.conc_k[n]) for n in range(2)])
        e = {"zeta": rel(g.zeta(), spm.SpmOracle.to_ooura(zt)),
             "conc": rel(g.concentration(), spm.SpmOracle.to_ooura(ct))}
        p = g.particles()
        e["v"] = rel(p["v"], o.p.v)
        e["x"] = np.abs(p["x"] - o.p.x).max()
        for k, v in e.items():
            worst[k] = max(worst.get(k, 0.0), v)
    return worst


def test_electrolyte_fp64_matches_oracle():
    cfg = udf.electrolyte_config((5, 5, 5), 2, seed=3, surface_charge=-100.0, efield=(0.05, 0.0, 0.0))
    w = _run(cfg, 4, 0)
    for k, v in w.items():
        assert v < 1e-10, (k, v, w)


def test_electrolyte_fp64_noncubic_positive_charge_field_switch():
    cfg = udf.electrolyte_config((4, 5, 6), 3, seed=5, surface_charge=50.0, min_gap=0.5)
    w = _run(cfg, 4, 0, efield_switch=(2, (0.0, 0.0, 0.05)))
    for k, v in w.items():
        assert v < 1e-10, (k, v, w)


def test_electrolyte_mixed_precision_bound():
    cfg = udf.electrolyte_config((5, 5, 5), 4, seed=7, surface_charge=-100.0, efield=(0.05, 0.0, 0.0))
    w = _run(cfg, 4, 1)
    assert w["zeta"] < 1e-4 and w["conc"] < 1e-4 and w["v"] < 1e-3, w
