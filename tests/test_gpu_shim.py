"""The reference's own main loop (sp_3d_ns.cxx:442-657) with the GPU library
behind KAPSEL's function names (kapsel_old_b200/shim/kapsel_ref_shim.cxx).

Three programs built by oracle/Makefile (`make shim`) from the same serial
reference objects read the same input file and run the same steps:
  kapsel_ref_main           the reference alone;
  kapsel_ref_main_step      Time_evolution_hydro / _OBL replaced by the
                            whole-step shim (state on the GPU between steps);
  kapsel_ref_main_routines  NS_solver_slavedEuler, Make_phi_u_particle,
                            Calc_f_hydro_correct_precision, the LJ cell-list
                            force, MD_solver_position/velocity_* and the
                            Electrolyte routines (NSsolute_solver_Euler,
                            Rescale_solute, Make_Coulomb_force_x_on_fluid)
                            replaced by the routine shims (host arrays in
                            and out).
Their restart records (Save_Restart_udf at MSTEP; with the ion
concentrations in the Electrolyte branch) and output records (Output_udf
every GTS steps) are compared.  Tolerances: FP64 relative error
<= 1e-10 per quantity (zeta compared on the 2/3-truncated modes that every
step reads; the whole-step shim's host zeta holds only those); with
KAPSEL_SHIM_PRECISION=mixed the velocity-field bound of the mixed path,
zeta relative L2 <= 1e-5 and particle velocities <= 1e-4.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import ref, spm, udf

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
EXE = {k: os.path.join(ref.REF_DIR, f"kapsel_ref_main{s}") for k, s in
       (("ref", ""), ("step", "_step"), ("routines", "_routines"))}


def rel(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (n if n > 0 else 1.0)


def _need(*which):
    for w in which:
        if not os.path.exists(EXE[w]):
            pytest.skip(f"{EXE[w]} not built (make -C oracle shim)")


def _records(path):
    """{record number: {path: float}} of a stand-in record file."""
    out = {}
    with open(path) as f:
        for line in f:
            head, _, val = line.rstrip("\n").partition(" = ")
            _, n, key = head.split(" ", 2)
            try:
                out.setdefault(int(n), {})[key] = float(val)
            except ValueError:
                pass
    return out


def _run(which, cfg, tmp, env=None, extra=()):
    d = os.path.join(tmp, which)
    os.makedirs(d, exist_ok=True)
    lines = [("output.UDF = ON" if s.startswith("output.UDF") else s) for s in udf.spm_udf_lines(cfg)]
    lines += list(extra)  # later lines win (the stand-in UDF reader)
    kv = os.path.join(d, "in.kv")
    with open(kv, "w") as f:
        f.write("\n".join(lines) + "\n")
    e = dict(os.environ, **(env or {}))
    r = subprocess.run([EXE[which], f"-I{kv}", f"-O{d}/out.kv", f"-D{kv}", f"-R{d}/res.kv"], cwd=d,
                       capture_output=True, text=True, env=e, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return _records(os.path.join(d, "res.kv"))[0], _records(os.path.join(d, "out.kv")), r.stderr


_ZK = re.compile(r"resume\.CONTINUE\.Saved_Data\.Zeta\[(\d+)\]\[(\d+)\]\[(\d+)\]\.zeta([01])")


def _restart_state(rec, cfg):
    N = [1 << p for p in cfg["np_xyz"]]
    z = np.zeros((2, N[0], N[1], N[2] + 2))
    for k, v in rec.items():
        m = _ZK.fullmatch(k)
        if m:
            i, j, kk, c = (int(g) for g in m.groups())
            z[c, i, j, kk] = v
    S = spm.Spectral(spm.Params(dict(cfg, eq="Navier_Stokes")))
    zt = spm.SpmOracle.from_ooura(z)
    z = spm.SpmOracle.to_ooura(np.stack([S.truncate(zt[c]) for c in range(2)]))
    base = "resume.CONTINUE.Saved_Data."
    ukdc = np.array([rec[base + f"uk_dc.{a}"] for a in "xyz"])
    n = len(cfg["particles"])
    parts = {q: np.array([[rec[f"{base}Particles[{i}].{q}.{a}"] for a in "xyz"] for i in range(n)])
             for q in ("R", "v", "v_old", "omega", "f_hydro_previous", "torque_hydro_previous", "fr_previous")}
    return {"zeta": z, "uk_dc": ukdc, "ts": rec[base + "jikan.ts"], **parts}


_CK = re.compile(r"resume\.CONTINUE\.Saved_Data\.Concentration\[(\d+)\]\[(\d+)\]\[(\d+)\]\[(\d+)\]\.ck")


def _restart_conc(rec, cfg):
    """Concentration[n] of an Electrolyte restart record, Ooura layout."""
    N = [1 << p for p in cfg["np_xyz"]]
    c = np.zeros((2, N[0], N[1], N[2] + 2))
    seen = 0
    for k, v in rec.items():
        m = _CK.fullmatch(k)
        if m:
            n, i, j, kk = (int(g) for g in m.groups())
            c[n, i, j, kk] = v
            seen += 1
    assert seen == c.size, seen
    return c


def _out_particles(recs, n):
    """Per output record: R, v, omega of every particle (Output_udf)."""
    out = []
    for r in sorted(recs):
        if r == 0:
            continue
        d = recs[r]
        out.append({q: np.array([[d[f"Particles[{i}].{q}.{a}"] for a in "xyz"] for i in range(n)])
                    for q in ("R", "v", "omega")})
    return out


def _compare(a, b, cfg, tol, what):
    sa, sb = _restart_state(a[0], cfg), _restart_state(b[0], cfg)
    assert sa["ts"] == sb["ts"]
    # uk_dc is N times the mean velocity: its error is scaled by N max|u|,
    # u = Zeta_k2u of the reference state
    S = spm.Spectral(spm.Params(dict(cfg, eq="Navier_Stokes")))
    u = S.zeta_k2u(spm.SpmOracle.from_ooura(sa["zeta"]), sa["uk_dc"])
    errs = {"zeta": rel(sb["zeta"], sa["zeta"]),
            "uk_dc": np.abs(sb["uk_dc"] - sa["uk_dc"]).max() / (u[0].size * max(np.abs(u).max(), 1e-300))}
    if cfg["particles"]:
        errs["R"] = np.abs(sb["R"] - sa["R"]).max()
        for q in ("v", "v_old", "omega", "f_hydro_previous", "fr_previous"):
            errs[q] = rel(sb[q], sa[q])
        oa, ob = _out_particles(a[1], len(cfg["particles"])), _out_particles(b[1], len(cfg["particles"]))
        assert len(oa) == len(ob) > 0
        errs["records_R"] = max(np.abs(y["R"] - x["R"]).max() for x, y in zip(oa, ob))
        errs["records_v"] = max(rel(y["v"], x["v"]) for x, y in zip(oa, ob))
    if cfg.get("eq") == "Electrolyte":
        errs["conc"] = rel(_restart_conc(b[0], cfg), _restart_conc(a[0], cfg))
    for k, v in errs.items():
        assert v < tol.get(k, tol["default"]), (what, k, v, errs)
    return errs


def _ns_cfg():
    cfg = udf.ns_config((5, 5, 5), 6, seed=11, kbt=1e-3, min_gap=0.2)
    cfg["gts"], cfg["num_snap"] = 5, 4  # MSTEP = 20, records every 5 steps
    return cfg


def test_main_loop_whole_step_shim_fp64(tmp_path):
    _need("ref", "step")
    cfg = _ns_cfg()
    a = _run("ref", cfg, str(tmp_path))
    b = _run("step", cfg, str(tmp_path))
    assert "kapsel shim: Time_evolution on the GPU" in b[2]
    _compare(a, b, cfg, {"default": FP64_TOL}, "step")


def test_main_loop_routine_shims_fp64(tmp_path):
    _need("ref", "routines")
    cfg = _ns_cfg()
    cfg["gravity_g"], cfg["mass_ratio"] = 0.3, 1.2
    a = _run("ref", cfg, str(tmp_path))
    b = _run("routines", cfg, str(tmp_path))
    assert "kapsel shim: solver routines on the GPU" in b[2]
    _compare(a, b, cfg, {"default": FP64_TOL}, "routines")


def test_main_loop_whole_step_shim_lees_edwards(tmp_path):
    _need("ref", "step")
    cfg = udf.shear_le_config((5, 5, 5), 3, seed=4, shear_rate=0.05, kbt=1e-3, min_gap=1.0)
    cfg["gts"], cfg["num_snap"] = 4, 3
    a = _run("ref", cfg, str(tmp_path))
    b = _run("step", cfg, str(tmp_path))
    assert "kapsel shim: Time_evolution on the GPU" in b[2]
    _compare(a, b, cfg, {"default": FP64_TOL}, "step LE")


def test_main_loop_whole_step_shim_electrolyte(tmp_path):
    _need("ref", "step")
    cfg = udf.electrolyte_config((5, 5, 5), 2, seed=6, efield=(0.05, 0.0, 0.0))
    cfg["gts"], cfg["num_snap"] = 3, 2
    a = _run("ref", cfg, str(tmp_path))
    b = _run("step", cfg, str(tmp_path))
    assert "kapsel shim: Time_evolution on the GPU" in b[2]
    _compare(a, b, cfg, {"default": FP64_TOL}, "step electrolyte")


def test_main_loop_whole_step_shim_electrolyte_resumed(tmp_path):
    """A resumed Electrolyte run (resume.Calculation = CONTINUE with the
    reference's own restart record of step 6): the whole-step shim uploads
    the restored zeta, particles, ion concentrations and Rescale_solute
    targets and continues to step 12 as the reference does."""
    _need("ref", "step")
    cfg = udf.electrolyte_config((5, 5, 5), 2, seed=6, efield=(0.05, 0.0, 0.0))
    cfg["gts"], cfg["num_snap"] = 3, 2
    _run("ref", cfg, str(tmp_path / "first"))
    with open(os.path.join(str(tmp_path / "first"), "ref", "res.kv")) as f:
        saved = [ln for ln in f.read().splitlines() if "resume.CONTINUE.Saved_Data." in ln]
    extra = ["resume.Calculation = CONTINUE"] + saved
    cont = dict(cfg, num_snap=4)
    a = _run("ref", cont, str(tmp_path / "cont"), extra=extra)
    b = _run("step", cont, str(tmp_path / "cont"), extra=extra)
    assert "kapsel shim: Time_evolution on the GPU" in b[2]
    assert _restart_state(a[0], cont)["ts"] == 12
    _compare(a, b, cont, {"default": FP64_TOL}, "step electrolyte resumed")


def test_main_loop_routine_shims_electrolyte(tmp_path):
    """NSsolute_solver_Euler (with the solute_rhs routines it calls),
    Rescale_solute and Make_Coulomb_force_x_on_fluid behind their reference
    names, with the particle routines, in the reference's main loop; the
    concentrations are compared as well."""
    _need("ref", "routines")
    cfg = udf.electrolyte_config((5, 5, 5), 2, seed=6, efield=(0.05, 0.0, 0.0))
    cfg["gts"], cfg["num_snap"] = 3, 2
    a = _run("ref", cfg, str(tmp_path))
    b = _run("routines", cfg, str(tmp_path))
    assert "kapsel shim: Electrolyte routines on the GPU" in b[2]
    _compare(a, b, cfg, {"default": FP64_TOL}, "routines electrolyte")


def test_main_loop_whole_step_shim_mixed(tmp_path):
    _need("ref", "step")
    cfg = _ns_cfg()
    a = _run("ref", cfg, str(tmp_path))
    b = _run("step", cfg, str(tmp_path), env={"KAPSEL_SHIM_PRECISION": "mixed"})
    assert "mixed" in b[2]
    _compare(a, b, cfg, {"default": 1e-4, "zeta": 1e-5, "R": 1e-6, "records_R": 1e-6, "uk_dc": 1e-5}, "mixed")
