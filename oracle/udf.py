"""Writes the flat `path = value` UDF stand-in files the reference oracle reads.

TEST INFRASTRUCTURE ONLY (used by tests/golden/make_golden.py, tests and the
bench's CPU reference arm).  The keys are the dotted UDF paths that
Gourmet_file_io (input.cxx:438-1818) and the user_specify particle reader
(init_particle.cxx:226-288) ask for; values mirror the schema in
Udf/define.udf.  Only the spherical-particle Navier_Stokes,
Shear_Navier_Stokes_Lees_Edwards (DC shear) and Electrolyte branches are
produced.
"""
from __future__ import annotations


def _fmt(v):
    if isinstance(v, float):
        return repr(v)
    return str(v)


def spm_udf_lines(cfg: dict) -> list[str]:
    """Return the stand-in UDF lines for one SPM configuration.

    cfg keys (all optional except np_xyz and particles):
      eq: "Navier_Stokes" | "Shear_Navier_Stokes_Lees_Edwards" | "Electrolyte"
      shear_rate: Shear_rate of the DC external field (Lees-Edwards)
      np_xyz: (NPX, NPY, NPZ)  -> N = 1<<NP per axis (input.cxx:1392-1397)
      dx, rho, eta, kbt, alpha_v, alpha_o, dt, a, a_xi, mass_ratio,
      gravity_g, gravity_dir ("-X"/"-Y"/"-Z"), epsilon, lj_powers ("12:6"),
      lj_truncate ("ON"/"OFF"/"NONE"), rotation ("ON"/"OFF"),
      fix_cell (tuple of 3 bools), gts, num_snap,
      particles: list of dicts with x (3), v (3), omega (3), q (4)
      electrolyte: dict(dielectric, surface_charge, debye, val_p, val_n,
                        onsager_p, onsager_n, efield (3), init_profile)
    """
    eq = cfg.get("eq", "Navier_Stokes")
    L = []
    put = lambda k, v: L.append(f"{k} = {_fmt(v)}")
    put("resume.Calculation", "NEW")
    put("resume.CONTINUE.Saved_Data.jikan.ts", 0)
    put("constitutive_eq.type", eq)
    base = f"constitutive_eq.{eq}"
    put(f"{base}.DX", float(cfg.get("dx", 1.0)))
    put(f"{base}.RHO", float(cfg.get("rho", 1.0)))
    put(f"{base}.ETA", float(cfg.get("eta", 1.0)))
    put(f"{base}.kBT", float(cfg.get("kbt", 0.0)))
    if eq in ("Navier_Stokes", "Shear_Navier_Stokes_Lees_Edwards"):
        put(f"{base}.alpha_v", float(cfg.get("alpha_v", 1.0)))
        put(f"{base}.alpha_o", float(cfg.get("alpha_o", 1.0)))
        if eq != "Navier_Stokes":
            # input.cxx:634-645
            put(f"{base}.External_field.type", "DC")
            put(f"{base}.External_field.DC.Shear_rate", float(cfg.get("shear_rate", 0.0)))
    else:
        el = cfg["electrolyte"]
        put(f"{base}.Dielectric_cst", float(el["dielectric"]))
        put(f"{base}.INIT_profile", el.get("init_profile", "Uniform"))
        put(f"{base}.Add_salt.type", "salt")
        s = f"{base}.Add_salt.salt"
        put(f"{s}.Valency_positive_ion", float(el.get("val_p", 1.0)))
        put(f"{s}.Valency_negative_ion", float(el.get("val_n", -1.0)))
        put(f"{s}.Onsager_coeff_positive_ion", float(el.get("onsager_p", 1.0)))
        put(f"{s}.Onsager_coeff_negative_ion", float(el.get("onsager_n", 1.0)))
        put(f"{s}.Debye_length", float(el["debye"]))
        ef = el.get("efield", (0.0, 0.0, 0.0))
        if any(e != 0.0 for e in ef):
            put(f"{base}.Electric_field.type", "ON")
            put(f"{base}.Electric_field.ON.type", "DC")
            for n, e in zip("xyz", ef):
                put(f"{base}.Electric_field.ON.DC.E{n}", float(e))
        else:
            put(f"{base}.Electric_field.type", "OFF")

    parts = cfg["particles"]
    put("object_type.type", "spherical_particle")
    ps = "object_type.spherical_particle.Particle_spec[0]"
    put(f"{ps}.Particle_number", len(parts))
    put(f"{ps}.MASS_RATIO", float(cfg.get("mass_ratio", 1.0)))
    put(f"{ps}.Surface_charge", float(cfg.get("electrolyte", {}).get("surface_charge", 0.0)))
    put(f"{ps}.janus_axis", "NONE")
    put(f"{ps}.janus_propulsion", "OFF")
    put("A_XI", float(cfg.get("a_xi", 2.0)))
    put("A", float(cfg.get("a", 5.0)))
    put("gravity.G", float(cfg.get("gravity_g", 0.0)))
    put("gravity.G_direction", cfg.get("gravity_dir", "-Z"))
    put("EPSILON", float(cfg.get("epsilon", 1.0)))
    put("LJ_powers", cfg.get("lj_powers", "12:6"))
    npx, npy, npz = cfg["np_xyz"]
    put("mesh.NPX", npx)
    put("mesh.NPY", npy)
    put("mesh.NPZ", npz)
    put("time_increment.type", "manual")
    put("time_increment.manual.delta_t", float(cfg.get("dt", 0.01)))
    put("switch.ROTATION", cfg.get("rotation", "ON"))
    put("switch.LJ_truncate", cfg.get("lj_truncate", "ON"))
    put("switch.INIT_distribution.type", "user_specify")
    put("switch.INIT_orientation", "user_specify")
    put("switch.SLIP_tol", 1e-5)
    put("switch.SLIP_iter", 100)
    fc = cfg.get("fix_cell", (False, False, False))
    for n, f in zip("xyz", fc):
        put(f"switch.FIX_CELL.{n}", "ON" if f else "OFF")
    put("switch.pin.type", "NO")
    for i, p in enumerate(parts):
        t = f"switch.INIT_distribution.user_specify.Particles[{i}]"
        x = p["x"]
        v = p.get("v", (0.0, 0.0, 0.0))
        w = p.get("omega", (0.0, 0.0, 0.0))
        q = p.get("q", (1.0, 0.0, 0.0, 0.0))
        for n, val in zip("xyz", x):
            put(f"{t}.R.{n}", float(val))
        for n, val in zip("xyz", v):
            put(f"{t}.v.{n}", float(val))
        for n, val in zip("xyz", w):
            put(f"{t}.omega.{n}", float(val))
        for n, val in zip(("q0", "q1", "q2", "q3"), q):
            put(f"{t}.q.{n}", float(val))
    put("output.GTS", int(cfg.get("gts", 1000)))
    put("output.Num_snap", int(cfg.get("num_snap", 1)))
    avs = cfg.get("avs")  # {"dir": ..., "name": ...}: Output_avs files, BINARY
    if avs:
        put("output.AVS", "ON")
        put("output.ON.Out_dir", avs["dir"])
        put("output.ON.Out_name", avs["name"])
        put("output.ON.FileType", "BINARY")
    else:
        put("output.AVS", "OFF")
    put("output.UDF", "OFF")
    return L


def write_udf(path: str, cfg: dict) -> str:
    with open(path, "w") as f:
        f.write("\n".join(spm_udf_lines(cfg)) + "\n")
    return path


def place_spheres(n: int, box: tuple, a: float, min_gap: float, seed: int, max_tries: int = 200000):
    """Seeded uniform-random non-overlapping centres (PCG64), centre distance >= 2a+min_gap
    under the minimum image.  Used by both the oracle and the GPU runs."""
    import numpy as np

    rng = np.random.Generator(np.random.PCG64(seed))
    box = np.asarray(box, dtype=np.float64)
    dmin2 = (2 * a + min_gap) ** 2
    pts = []
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"cannot place {n} spheres of radius {a} in {tuple(box)}")
        c = rng.random(3) * box
        ok = True
        for p in pts:
            d = c - p
            d -= np.rint(d / box) * box
            if float(d @ d) < dmin2:
                ok = False
                break
        if ok:
            pts.append(c)
    return np.array(pts)


def ns_config(np_xyz, n_particles, seed, a=5.0, a_xi=2.0, kbt=0.0, dt=0.01, min_gap=1.0,
              gravity_g=0.0, mass_ratio=1.0, rotation="ON", velocities=None):
    """A Navier_Stokes configuration with seeded sphere positions."""
    N = [1 << int(p) for p in np_xyz]
    xs = place_spheres(n_particles, N, a, min_gap, seed) if n_particles else []
    parts = []
    for i, x in enumerate(xs):
        p = {"x": tuple(float(c) for c in x)}
        if velocities is not None:
            p["v"], p["omega"] = velocities[i]
        parts.append(p)
    return {"eq": "Navier_Stokes", "np_xyz": tuple(np_xyz), "particles": parts, "a": a, "a_xi": a_xi,
            "kbt": kbt, "dt": dt, "gravity_g": gravity_g, "mass_ratio": mass_ratio, "rotation": rotation}


def shear_le_config(np_xyz, n_particles, seed, shear_rate, a=5.0, a_xi=2.0, kbt=0.0, dt=0.01, min_gap=1.0,
                    rotation="ON"):
    """A Shear_Navier_Stokes_Lees_Edwards configuration (DC shear) with seeded
    sphere positions."""
    cfg = ns_config(np_xyz, n_particles, seed=seed, a=a, a_xi=a_xi, kbt=kbt, dt=dt, min_gap=min_gap,
                    rotation=rotation)
    cfg["eq"] = "Shear_Navier_Stokes_Lees_Edwards"
    cfg["shear_rate"] = float(shear_rate)
    return cfg


def electrolyte_config(np_xyz, n_particles, seed, surface_charge=-100.0, debye=4.0, bjerrum=0.7, kbt=1.0,
                       efield=(0.0, 0.0, 0.0), a=5.0, a_xi=2.0, dt=0.01, min_gap=1.0):
    """An Electrolyte configuration: two monovalent ion species (salt),
    Onsager coefficients 1, uniform initial profile, Dielectric_cst chosen so
    that e^2/(4 pi kBT eps) equals the Bjerrum length."""
    import math

    cfg = ns_config(np_xyz, n_particles, seed=seed, a=a, a_xi=a_xi, kbt=kbt, dt=dt, min_gap=min_gap)
    cfg["eq"] = "Electrolyte"
    cfg["alpha_v"] = 0.0
    cfg["alpha_o"] = 0.0
    cfg["electrolyte"] = dict(dielectric=1.0 / (4.0 * math.pi * kbt * bjerrum), surface_charge=float(surface_charge),
                              debye=float(debye), val_p=1.0, val_n=-1.0, onsager_p=1.0, onsager_n=1.0,
                              efield=tuple(float(e) for e in efield))
    return cfg
