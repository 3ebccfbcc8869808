"""Parity on the benchmark configurations themselves, against the compiled
reference (oracle/_ref, the serial FP64 build of the unmodified sources).

* 64^3 with 16 spheres (a=5, xi=2), the body force along -z applied as
  gravity, kBT=0, dt=0.01: the FP64 GPU step against the reference for 200
  steps, checked at growing intervals.
* 128^3 with 256 spheres (a=5, xi=2), kBT=1e-3 thermal kicks from the
  reference's own MT19937 stream: the FP64 GPU step against the reference
  for 10 steps, every step; the mixed-precision step against the same
  reference states.
* The same 128^3 suspension over its full 2000 steps: the mixed-precision
  step against the FP64 GPU step (pinned to the reference above), as an
  error curve.

Both sides initialise themselves from the same configuration (positions
through the user_specify route), so the initial projection is covered too.
Tolerances: FP64 relative error <= 1e-10 per quantity (zeta, the velocity
field, the k=0 mode, particle positions (absolute), velocities, angular
velocities and hydrodynamic forces); mixed precision velocity-field
relative L2 <= 1e-5 and particle velocities <= 1e-4 relative against the
FP64 reference over 10 steps; over 2000 steps against the FP64 GPU path
velocity-field relative L2 <= 1e-4, particle velocities <= 1e-3 relative
and positions <= 1e-5 absolute (grid units).
"""
import numpy as np
import pytest

from kapsel_old_b200 import workload
from oracle import ref, spm

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def rel(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (n if n > 0 else 1.0)


def _need_ref():
    if not ref.available():
        pytest.skip("oracle/_ref not built")


class _RefView:
    """The reference state in the GPU library's terms: zeta truncated to the
    2/3 box and the velocity field Zeta_k2u of it (operate_omega.h:124-128)."""

    def __init__(self, cfg):
        self.S = spm.Spectral(spm.Params(cfg))

    def state(self, R):
        z = spm.SpmOracle.from_ooura(R.zeta())
        zt = np.stack([self.S.truncate(z[d]) for d in range(2)])
        ukdc = R.uk_dc()
        return {"zeta": spm.SpmOracle.to_ooura(zt), "u": self.S.zeta_k2u(zt, ukdc), "uk_dc": ukdc,
                "p": R.particles()}


def _errors(g, rs):
    uo = rs["u"]
    e = {
        "zeta": rel(g.zeta(), rs["zeta"]),
        "u": rel(g.velocity(), uo),
        # uk_dc is N times the mean velocity: scale by N max|u|
        "uk_dc": np.abs(g.uk_dc() - rs["uk_dc"]).max() / (uo.size / 3 * max(np.abs(uo).max(), 1e-300)),
    }
    p, po = g.particles(), rs["p"]
    e["x"] = np.abs(p["x"] - po["x"]).max()
    e["v"] = rel(p["v"], po["v"])
    e["omega"] = rel(p["omega"], po["omega"])
    e["f_hydro"] = rel(p["f_hydro"], po["f_hydro"])
    return e


def test_plain_64cubed_16_fp64_200_steps_against_reference():
    _need_ref()
    import kapsel_old_b200 as kg

    cfg = workload.plain_64_16()
    R = ref.RefSim(cfg)
    g = kg.Simulation(cfg, precision=kg.FP64)
    view = _RefView(cfg)
    done = 0
    worst = {}
    for at in (1, 2, 5, 10, 20, 50, 100, 150, 200):
        R.step(at - done)
        g.step(at - done, graph=True)
        done = at
        e = _errors(g, view.state(R))
        for k, v in e.items():
            worst[k] = max(worst.get(k, 0.0), v)
            assert v < FP64_TOL, (at, k, v, e)
    assert g.time()[0] == 200
    # the spheres moved: the comparison is not of a resting state
    assert np.abs(g.particles()["v"]).max() > 1e-6, worst
    print("plain 64^3/16 FP64, 200 steps, worst:", {k: f"{v:.1e}" for k, v in worst.items()})


def test_mixed_128cubed_256_fp64_and_mixed_10_steps_against_reference():
    _need_ref()
    import kapsel_old_b200 as kg

    cfg = workload.mixed_128_256()
    R = ref.RefSim(cfg)
    g = kg.Simulation(cfg, precision=kg.FP64)
    m = kg.Simulation(cfg, precision=kg.MIXED)
    view = _RefView(cfg)
    worst, worst_m = {}, {}
    for s in range(1, 11):
        R.step(1)
        g.step(1, graph=True)
        m.step(1, graph=True)
        rs = view.state(R)
        e = _errors(g, rs)
        for k, v in e.items():
            worst[k] = max(worst.get(k, 0.0), v)
            assert v < FP64_TOL, (s, k, v, e)
        em = {"u": rel(m.velocity(), rs["u"]), "v": rel(m.particles()["v"], rs["p"]["v"])}
        for k, v in em.items():
            worst_m[k] = max(worst_m.get(k, 0.0), v)
        assert em["u"] < 1e-5 and em["v"] < 1e-4, (s, em)
    print("128^3/256, 10 steps, FP64 worst:", {k: f"{v:.1e}" for k, v in worst.items()},
          "mixed worst:", {k: f"{v:.1e}" for k, v in worst_m.items()})


def test_mixed_128cubed_256_2000_steps_against_fp64():
    import kapsel_old_b200 as kg

    cfg = workload.mixed_128_256()
    a = kg.Simulation(cfg, precision=kg.FP64)
    b = kg.Simulation(cfg, precision=kg.MIXED)
    curve = []
    done = 0
    for at in (1, 10, 100, 250, 500, 1000, 1500, 2000):
        a.step(at - done, graph=True)
        b.step(at - done, graph=True)
        done = at
        pa, pb = a.particles(), b.particles()
        e = {"step": at, "u": rel(b.velocity(), a.velocity()), "v": rel(pb["v"], pa["v"]),
             "x": float(np.abs(pb["x_nopbc"] - pa["x_nopbc"]).max())}
        curve.append(e)
        assert e["u"] < 1e-4 and e["v"] < 1e-3 and e["x"] < 1e-5, curve
    print("mixed vs FP64, 128^3/256:", "; ".join(f"{c['step']}: u {c['u']:.1e} v {c['v']:.1e} x {c['x']:.1e}"
                                                  for c in curve))


def test_electrolyte_128cubed_64_fp64_3_steps_against_reference():
    """The charged-colloid configuration (128^3, 64 spheres, Z = -100, salt
    with Debye length 4, Bjerrum length 0.7, E_x = 0.05) in FP64 against the
    compiled reference for 3 steps: zeta and the ion concentrations on the
    retained modes, particle positions and velocities, <= 1e-10."""
    _need_ref()
    import kapsel_old_b200 as kg

    cfg = workload.electrolyte_128_64()
    R = ref.RefSim(cfg)
    g = kg.Simulation(cfg, precision=kg.FP64)
    S = spm.Spectral(spm.Params(dict(cfg, eq="Navier_Stokes")))

    def trunc(a):
        z = spm.SpmOracle.from_ooura(a)
        return spm.SpmOracle.to_ooura(np.stack([S.truncate(z[c]) for c in range(len(z))]))

    for s in range(1, 4):
        R.step(1)
        g.step(1, graph=True)
        conc_ref = trunc(np.stack([R.field(20), R.field(21)]))
        e = {"zeta": rel(g.zeta(), trunc(R.zeta())), "conc": rel(g.concentration(), conc_ref)}
        pg, pr = g.particles(), R.particles()
        e["x"] = np.abs(pg["x"] - pr["x"]).max()
        e["v"] = rel(pg["v"], pr["v"])
        e["f_hydro"] = rel(pg["f_hydro"], pr["f_hydro"])
        for k, v in e.items():
            assert v < FP64_TOL, (s, k, v, e)
