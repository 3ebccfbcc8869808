"""The oracle restatement against golden fixtures generated from the
unmodified reference (tests/golden/make_golden.py).  CPU only."""
import glob
import json
import os

import numpy as np
import pytest

from oracle import spm

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
STEP_CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLD, "ns*.npz")))
EL_CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLD, "el*.npz")))


def rel(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (n if n > 0 else 1.0)


def test_fixtures_present():
    assert len(STEP_CASES) >= 3
    assert len(EL_CASES) >= 2


@pytest.mark.parametrize("name", STEP_CASES + EL_CASES)
def test_oracle_matches_reference_steps(name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    cfg = json.loads(str(g["cfg"]))
    o = spm.ElectrolyteOracle(cfg) if cfg.get("eq") == "Electrolyte" else spm.SpmOracle(cfg)
    o.run(int(g["steps"]))
    if "conc" in g.files:
        for n in range(2):
            co = spm.SpmOracle.to_ooura(o.conc_k[n])
            assert np.abs(co - g["conc"][n]).max() < 1e-11 * np.abs(g["conc"][n]).max(), n
    zt = spm.SpmOracle.to_ooura(np.stack([o.S.truncate(o.zeta[d]) for d in range(2)]))
    zr = g["zeta"].copy()
    keep = np.broadcast_to(np.repeat(o.S.keep, 2, axis=2), zr.shape[1:])
    zr[:, ~keep] = 0.0  # the reference carries roundoff outside the 2/3 box
    assert rel(zt, zr) < 1e-12
    scale = o.P.NX * o.P.NY * o.P.NZ * max(np.abs(o.p.v).max(), 1e-300)
    assert np.abs(o.uk_dc - g["uk_dc"]).max() <= 1e-12 * scale + 1e-300
    for k, mine in (("x", o.p.x), ("x_nopbc", o.p.x_nopbc), ("q", o.p.q)):
        assert np.abs(mine - g["p_" + k]).max() < 1e-12, k
    for k, mine in (("v", o.p.v), ("omega", o.p.omega), ("f_hydro", o.p.f_hydro_previous),
                    ("torque_hydro", o.p.torque_hydro_previous), ("fr", o.p.fr_previous)):
        ref = g["p_" + k]
        if np.abs(ref).max() == 0:
            assert np.abs(mine).max() == 0, k
        else:
            assert rel(mine, ref) < 1e-12, k


def test_fft_convention_and_sekibun():
    g = np.load(os.path.join(GOLD, "fft_16x32x8.npz"))
    cfg = json.loads(str(g["cfg"]))
    S = spm.Spectral(spm.Params(cfg))
    ak = spm.SpmOracle.to_ooura(S.fwd(g["a"]))
    assert rel(ak, g["a_k"]) < 1e-14
    assert rel(S.inv(spm.SpmOracle.from_ooura(g["a_k"])), g["a"]) < 1e-14
    cells = spm.sekibun_cells(spm.Params(cfg))
    assert cells.shape == g["sekibun"].shape == (1935, 3)
    assert np.array_equal(cells, g["sekibun"])


def test_oracle_known_answer_viscous_decay():
    # a single transverse shear mode with no particles decays as exp(-nu k^2 t):
    # the nonlinear term of one Fourier mode vanishes and slaved Euler is exact
    cfg = {"np_xyz": (4, 4, 4), "particles": [], "dt": 0.05}
    o = spm.SpmOracle(cfg)
    N = o.P.N
    x = np.arange(N[0])[:, None, None]
    u = np.zeros((3,) + tuple(N))
    u[1] = 0.01 * np.sin(2 * np.pi * 2 * x / N[0]) * np.ones(N)
    o.zeta, o.uk_dc = o.S.u2zeta_k(u)
    e0 = np.abs(o.zeta).max()
    o.run(10)
    k2 = (2 * np.pi * 2 / N[0]) ** 2
    assert abs(np.abs(o.zeta).max() / e0 - np.exp(-o.P.NU * k2 * 0.5)) < 1e-12


def test_oracle_solenoidal_idempotent():
    cfg = {"np_xyz": (4, 4, 4), "particles": []}
    S = spm.Spectral(spm.Params(cfg))
    u = np.random.default_rng(1).standard_normal((3, 16, 16, 16))
    a = S.solenoidal_u(u)
    b = S.solenoidal_u(a)
    assert rel(b, a) < 1e-13
    div = sum(k * S.fwd(a[d]) for d, k in enumerate((S.kx, S.ky, S.kz)))
    assert np.abs(div).max() < 1e-10 * np.abs(S.fwd(a[0])).max()


def test_oracle_phi_volume():
    """The integral of the smoothed profile over the grid against the sphere
    volume 4/3 pi a^3 (the mass factor the reference uses,
    md_force.cxx:334-336): the smooth interface of width xi adds a
    second-order term, measured 1 + 0.066 (xi/a)^2 for a = 4, 5, 6."""
    from oracle import udf

    rng = np.random.default_rng(0)
    excess = []
    for a in (4.0, 5.0, 6.0):
        o = spm.SpmOracle(udf.ns_config((5, 5, 5), 1, seed=3, a=a, a_xi=2.0))
        V = 4.0 / 3.0 * np.pi * a ** 3
        for _ in range(3):
            x = np.array([[16.0, 16.0, 16.0]]) + rng.random((1, 3))
            phi, _ = o.phi_up(x, np.zeros((1, 3)), np.zeros((1, 3)))
            e = phi.sum() / V - 1.0
            assert 0.0 < e < 0.1 * (2.0 / a) ** 2, (a, e)
        excess.append(e)
    assert excess[0] > excess[1] > excess[2]
