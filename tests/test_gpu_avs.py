"""AVS snapshots written from device state against Output_avs (and
Output_avs_charge in the Electrolyte branch, Output_avs_p for the particles)
of the compiled reference (oracle/_ref) on the same state: identical
.fld/.cod text, and the velocity and phi columns of the binary .dat (and the
particle positions and body axes) equal to float32 rounding.  The reference's pressure column is never assigned in the
Navier_Stokes branch (uninitialised memory) and its tau columns read its
vorticity buffer in place of the velocity, so those columns are checked
against the viscous strain rate of the velocity computed here with numpy."""
import os

import numpy as np
import pytest

from oracle import ref, udf

pytestmark = pytest.mark.gpu


def _cfg(d):
    cfg = udf.ns_config((5, 5, 5), 3, seed=5, kbt=0.0, min_gap=1.0, gravity_g=0.5, mass_ratio=1.5)
    cfg["avs"] = {"dir": d, "name": "snap"}
    cfg["eta"] = 1.3
    return cfg


def _check_particle_files(dr, dg, ts, np_):
    """Output_avs_p: the particle .fld text and the float32 positions, radius
    and body-axis columns (rotation matrix of each quaternion)."""
    assert open(os.path.join(dr, "snapp.fld")).read() == open(os.path.join(dg, "snapp.fld")).read()
    for ext, rows in ((".cod", 3), (".dat", 10)):
        A = np.fromfile(os.path.join(dr, "avs", f"snapp_{ts}{ext}"), dtype=np.float32)
        B = np.fromfile(os.path.join(dg, "avs", f"snapp_{ts}{ext}"), dtype=np.float32)
        assert A.shape == B.shape == (rows * np_,), ext
        assert np.abs(A - B).max() <= 4e-7 * max(np.abs(A).max(), 1.0), ext


def _read(path, n=32):
    a = np.fromfile(path, dtype=np.float32).reshape(10, n, n, n)  # [col][k][j][i]
    return a.transpose(0, 3, 2, 1)  # -> [col][i][j][k]


def test_avs_snapshot_matches_reference(tmp_path):
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    import kapsel_old_b200 as kg

    dr, dg = os.path.join(tmp_path, "ref"), os.path.join(tmp_path, "gpu")
    os.makedirs(os.path.join(dr, "avs"))
    os.makedirs(dg)
    r = ref.RefSim(_cfg(dr))
    r.step(4)
    r.output_avs(init=True)
    g = kg.Simulation(_cfg(dg), precision=kg.FP64)
    g.step(4)
    g.write_avs(dg, "snap", nstep=2, init=True)
    for f in ("snap.fld", "snap.cod"):
        assert open(os.path.join(dr, f)).read() == open(os.path.join(dg, f)).read(), f
    _check_particle_files(dr, dg, 4, 3)
    A = _read(os.path.join(dr, "avs", "snap_4.dat"))
    B = _read(os.path.join(dg, "avs", "snap_4.dat"))
    for c in range(4):
        assert np.abs(A[c] - B[c]).max() <= 2e-7 * max(np.abs(A[c]).max(), 1e-30), c
    assert np.abs(A[0]).max() > 0 and np.abs(A[3]).max() > 0.5
    assert np.all(B[4] == 0)
    # tau = ETA (d_i u_j + d_j u_i) / 2 from the velocity columns
    u = B[:3].astype(np.float64)
    k = [np.fft.fftfreq(32) * 2 * np.pi for _ in range(3)]
    K = np.meshgrid(*k, indexing="ij")

    def d(f, ax):
        return np.real(np.fft.ifftn(1j * K[ax] * np.fft.fftn(f)))

    eta = 1.3
    tau = {"xy": 0.5 * eta * (d(u[1], 0) + d(u[0], 1)), "yz": 0.5 * eta * (d(u[2], 1) + d(u[1], 2)),
           "zx": 0.5 * eta * (d(u[2], 0) + d(u[0], 2)), "xx": eta * d(u[0], 0), "yy": eta * d(u[1], 1)}
    for c, key in zip(range(5, 10), ("xy", "yz", "zx", "xx", "yy")):
        scale = max(np.abs(tau[key]).max(), 1e-30)
        assert np.abs(B[c] - tau[key]).max() <= 1e-4 * scale, key


def test_avs_electrolyte_snapshot_matches_reference(tmp_path):
    """Output_avs_charge: the same .fld/.cod text and all seven columns (u,
    phi, surface charge, ionic charge density, Coulomb potential) equal to
    float32 rounding of the reference's snapshot of the same state."""
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    import kapsel_old_b200 as kg

    def cfg(d):
        c = udf.electrolyte_config((5, 5, 5), 2, seed=6, efield=(0.05, 0.0, 0.0))
        c["avs"] = {"dir": d, "name": "snap"}
        return c

    dr, dg = os.path.join(tmp_path, "ref"), os.path.join(tmp_path, "gpu")
    os.makedirs(os.path.join(dr, "avs"))
    os.makedirs(dg)
    r = ref.RefSim(cfg(dr))
    r.step(3)
    r.output_avs(init=True)
    g = kg.Simulation(cfg(dg), precision=kg.FP64)
    g.step(3)
    z_before = g.zeta()
    g.write_avs(dg, "snap", nstep=2, init=True)
    assert np.array_equal(g.zeta(), z_before)  # the snapshot leaves the state alone
    for f in ("snap.fld", "snap.cod"):
        assert open(os.path.join(dr, f)).read() == open(os.path.join(dg, f)).read(), f
    _check_particle_files(dr, dg, 3, 2)
    A = np.fromfile(os.path.join(dr, "avs", "snap_3.dat"), dtype=np.float32).reshape(7, 32, 32, 32)
    B = np.fromfile(os.path.join(dg, "avs", "snap_3.dat"), dtype=np.float32).reshape(7, 32, 32, 32)
    for c in range(7):
        scale = max(np.abs(A[c]).max(), 1e-30)
        assert np.abs(A[c] - B[c]).max() <= 4e-7 * scale, (c, np.abs(A[c] - B[c]).max() / scale)
    # every column carries signal: velocity, phi, surface charge, charge, potential
    assert all(np.abs(A[c]).max() > 0 for c in range(7))
