"""Restart records on the GPU against the compiled reference (oracle/_ref).

(a) a record the reference saved is loaded by the GPU library, which then
    continues exactly as the reference's own resumed run (thermostat on:
    both seed the stream afresh and skip the one step the resumed loop
    takes before restoring);
(b) a record the GPU saved is restored by the reference, and both continue
    in step;
(c) FP64 electrolyte and mixed-precision Navier-Stokes contexts reload
    their own records and continue as the uninterrupted run.
Tolerances: FP64 <= 1e-10 relative (the records carry 17 digits)."""
import os

import numpy as np
import pytest

from oracle import ref, spm, udf

pytestmark = pytest.mark.gpu


def rel(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (n if n > 0 else 1.0)


def _need_ref():
    if not ref.available():
        pytest.skip("oracle/_ref not built")


def _trunc(zeta_ooura, cfg):
    S = spm.Spectral(spm.Params(cfg))
    z = spm.SpmOracle.from_ooura(zeta_ooura)
    return spm.SpmOracle.to_ooura(np.stack([S.truncate(z[d]) for d in range(2)]))


def _cfg():
    return udf.ns_config((5, 5, 5), 4, seed=9, kbt=1e-3, min_gap=1.0, gravity_g=0.3, mass_ratio=1.5)


def test_gpu_loads_reference_record(tmp_path):
    _need_ref()
    import kapsel_old_b200 as kg

    cfg = _cfg()
    a = ref.RefSim(cfg)
    a.step(5)
    path = os.path.join(tmp_path, "ref.res")
    a.save_restart(path)
    b = ref.RefSim(cfg)
    b.resume(path)
    b.step(4)
    g = kg.Simulation(cfg, precision=kg.FP64)
    g.load_restart(path)
    assert g.time()[0] == 5
    g.step(4)
    assert g.time()[0] == 9 and abs(g.time()[1] - b.scalars()["time"]) < 1e-12
    assert rel(g.zeta(), _trunc(b.zeta(), cfg)) < 1e-10
    pg, pb = g.particles(), b.particles()
    for k in ("x", "v", "omega"):
        assert rel(pg[k], pb[k]) < 1e-10, k


def test_reference_loads_gpu_record(tmp_path):
    _need_ref()
    import kapsel_old_b200 as kg

    cfg = _cfg()
    g = kg.Simulation(cfg, precision=kg.FP64)
    g.step(6)
    path = os.path.join(tmp_path, "gpu.res")
    g.save_restart(path)
    b = ref.RefSim(cfg)
    b.resume(path)
    assert b.ts() == 6
    assert rel(_trunc(b.zeta(), cfg), g.zeta()) < 1e-14
    assert np.array_equal(b.particles()["x"], g.particles()["x"])
    # continue both under the resumed-run stream
    g2 = kg.Simulation(cfg, precision=kg.FP64)
    g2.load_restart(path)
    b.step(3)
    g2.step(3)
    assert rel(g2.zeta(), _trunc(b.zeta(), cfg)) < 1e-10
    assert rel(g2.particles()["v"], b.particles()["v"]) < 1e-10


def test_electrolyte_and_mixed_reload_continue(tmp_path):
    import kapsel_old_b200 as kg

    el = udf.electrolyte_config((5, 5, 5), 2, seed=3, surface_charge=-100.0, efield=(0.05, 0.0, 0.0))
    a = kg.Simulation(el, precision=kg.FP64)
    a.step(3)
    path = os.path.join(tmp_path, "el.res")
    a.save_restart(path)
    b = kg.Simulation(el, precision=kg.FP64)
    b.load_restart(path)
    assert rel(b.concentration(), a.concentration()) < 1e-15
    a.step(3)
    b.step(3)
    assert rel(b.zeta(), a.zeta()) < 1e-12
    assert rel(b.concentration(), a.concentration()) < 1e-12
    assert rel(b.particles()["x"], a.particles()["x"]) < 1e-12

    ns = udf.ns_config((6, 6, 6), 8, seed=2, kbt=0.0, min_gap=1.0, gravity_g=0.2, mass_ratio=1.5)
    m = kg.Simulation(ns, precision=kg.MIXED)
    m.step(4, graph=True)
    path = os.path.join(tmp_path, "mixed.res")
    m.save_restart(path)
    n = kg.Simulation(ns, precision=kg.MIXED)
    n.load_restart(path)
    assert np.array_equal(n.zeta(), m.zeta())
    m.step(3, graph=True)
    n.step(3, graph=True)
    assert rel(n.zeta(), m.zeta()) < 1e-5
    assert rel(n.particles()["x"], m.particles()["x"]) < 1e-9
