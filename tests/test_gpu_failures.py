"""Failure detection without a GPU fault.

Faults are made on the host: parameters and particle records with a NaN or
a position outside the box, which the library refuses before anything
reaches the device, and a non-finite fluid state, which the step detects on
the device and returns as a status (no trap).  A bounded device wait is made
to run out on a barrier that nothing arrives at.  After each failure the
device keeps working, and a context whose state is replaced steps again.
The reference has no counterpart: it asserts or calls exit_job."""
import numpy as np
import pytest

from oracle import udf

pytestmark = pytest.mark.gpu

ENONFINITE, ERANGE, EINVAL, ETIMEOUT = -5, -6, -1, -7


def _cfg():
    return udf.ns_config((5, 5, 5), 3, seed=3, kbt=0.0, min_gap=1.0, gravity_g=0.3, mass_ratio=1.5)


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_nonfinite_fluid_state_reported_then_recovered(precision):
    import kapsel_old_b200 as kg

    prec = getattr(kg, precision)
    g = kg.Simulation(_cfg(), precision=prec)
    g.step(3)
    z, u, parts = g.zeta(), g.uk_dc(), g.particles()
    bad = z.copy()
    bad[0, 1, 2, 4] = np.nan  # one retained mode of zeta
    g.set_zeta(bad, u)
    with pytest.raises(kg.KapselError) as e:
        g.step(1)
    assert e.value.code == ENONFINITE
    # the status stays until the state is replaced (read without stepping:
    # no launch works on the NaN state)
    with pytest.raises(kg.KapselError) as e:
        g.step(0)
    assert e.value.code == ENONFINITE
    # a good state replaces it and the run continues as an undisturbed copy
    # (to roundoff: the restored context forms u_k of zeta in a launch of its
    # own, the undisturbed one in the fused last launch of its step)
    g.set_zeta(z, u)
    g.set_particle_state(parts)
    ref = kg.Simulation(_cfg(), precision=prec)
    ref.step(3)
    g.step(2)
    ref.step(2)
    tol = 1e-12 if prec == kg.FP64 else 1e-5
    zr = ref.zeta()
    assert np.linalg.norm(g.zeta() - zr) <= tol * np.linalg.norm(zr)
    assert np.abs(g.particles()["x"] - ref.particles()["x"]).max() <= tol * 32
    g.close()
    ref.close()


def test_invalid_particle_records_refused_on_the_host():
    import kapsel_old_b200 as kg

    g = kg.Simulation(_cfg(), precision=kg.FP64)
    g.step(1)
    good = g.particles()
    for key, value, code in (("v", np.nan, EINVAL), ("omega", np.inf, EINVAL), ("q", np.nan, EINVAL),
                             ("x", -1.0, ERANGE), ("x", 32.0, ERANGE), ("x", np.nan, EINVAL)):
        st = {k: v.copy() for k, v in good.items()}
        st[key][1, 0] = value
        with pytest.raises(kg.KapselError) as e:
            g.set_particle_state(st)
        assert e.value.code == code, (key, value, e.value.code)
    # nothing reached the device: the context steps on from its good state
    g.step(1)
    assert np.isfinite(g.particles()["v"]).all()
    g.close()


def test_bounded_device_wait_times_out_and_device_stays_usable():
    import kapsel_old_b200 as kg

    L = kg.load_library()
    assert L.kapsel_gpu_check_bounded_wait() == ETIMEOUT
    g = kg.Simulation(_cfg(), precision=kg.FP64)
    g.step(2)
    assert np.isfinite(g.zeta()).all()
    g.close()
