"""kapsel_old_b200 -- B200-native Smoothed Profile Method step for KAPSEL.

Python mirror of the C ABI in include/kapsel_gpu.h (libkapsel_gpu.so, built
in-tree by kapsel_old_b200/build.py).  The reference is a C++ program whose
SPM step is Time_evolution_hydro (sp_3d_ns.cxx:61-212); this module exposes
the same state (zeta, uk_dc, particles) and the routine-level entry points
(A2a_k, A_k2a, Solenoidal_u, Make_phi_u_particle, Calc_f_hydro_correct_precision,
Force) on numpy arrays in the reference's own layouts.

There is no CPU fallback: importing the library fails loudly when the CUDA
extension is missing, and every call raises KapselError on a non-zero status.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkapsel_gpu.so")

FP64 = 0
MIXED = 1
EQ_NAVIER_STOKES = 0
EQ_SHEAR_LE = 2
EQ_ELECTROLYTE = 3
_EQ = {"Navier_Stokes": EQ_NAVIER_STOKES, "Shear_Navier_Stokes_Lees_Edwards": EQ_SHEAR_LE,
       "Electrolyte": EQ_ELECTROLYTE}
P_STRIDE = 35


class KapselError(RuntimeError):
    """A non-zero KAPSEL_E* status; `code` holds it."""

    code = 0


class _Params(ctypes.Structure):
    _fields_ = [
        ("np_xyz", ctypes.c_int * 3),
        ("eq", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("n_particles", ctypes.c_int),
        ("dx", ctypes.c_double),
        ("rho", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("kbt", ctypes.c_double),
        ("alpha_v", ctypes.c_double),
        ("alpha_o", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("a", ctypes.c_double),
        ("a_xi", ctypes.c_double),
        ("mass_ratio", ctypes.c_double),
        ("gravity_g", ctypes.c_double),
        ("gravity_dir", ctypes.c_int),
        ("epsilon", ctypes.c_double),
        ("lj_powers", ctypes.c_int),
        ("lj_truncate", ctypes.c_int),
        ("rotation", ctypes.c_int),
        ("fix_cell", ctypes.c_int * 3),
        ("mt_seed", ctypes.c_uint),
        ("dielectric", ctypes.c_double),
        ("surface_charge", ctypes.c_double),
        ("debye_length", ctypes.c_double),
        ("valency_p", ctypes.c_double),
        ("valency_n", ctypes.c_double),
        ("onsager_p", ctypes.c_double),
        ("onsager_n", ctypes.c_double),
        ("e_ext", ctypes.c_double * 3),
        ("frozen", ctypes.c_int),
        ("shear_rate", ctypes.c_double),
        ("neighbor_lists", ctypes.c_int),
    ]


_lib = None

_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load libkapsel_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise KapselError(f"{path} is missing: run kapsel_old_b200.build.build() (nvcc, sm_100a)")
    L = ctypes.CDLL(path)
    sig = {
        "kapsel_params_default": (None, [ctypes.POINTER(_Params)]),
        "kapsel_gpu_create": (ctypes.c_int, [ctypes.POINTER(_Params), ctypes.POINTER(_VP)]),
        "kapsel_gpu_destroy": (ctypes.c_int, [_VP]),
        "kapsel_gpu_set_particles": (ctypes.c_int, [_VP, _DP, _DP]),
        "kapsel_gpu_init_state": (ctypes.c_int, [_VP]),
        "kapsel_gpu_step": (ctypes.c_int, [_VP, ctypes.c_int]),
        "kapsel_gpu_step_graph": (ctypes.c_int, [_VP, ctypes.c_int]),
        "kapsel_gpu_get_zeta": (ctypes.c_int, [_VP, _DP, _DP]),
        "kapsel_gpu_set_zeta": (ctypes.c_int, [_VP, _DP, _DP]),
        "kapsel_gpu_get_velocity": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_get_particles": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_set_particle_state": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_get_time": (ctypes.c_int, [_VP, _IP, _DP]),
        "kapsel_gpu_get_dims": (ctypes.c_int, [_VP, _IP]),
        "kapsel_gpu_set_efield": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_get_oblique": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_set_oblique": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_double]),
        "kapsel_gpu_get_concentration": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_set_concentration": (ctypes.c_int, [_VP, _DP, _DP]),
        "kapsel_gpu_check_bounded_wait": (ctypes.c_int, []),
        "kapsel_gpu_set_x_split": (ctypes.c_int, [_VP, ctypes.c_int]),
        "kapsel_gpu_A2a_k": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_A_k2a": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_solenoidal_u": (ctypes.c_int, [_VP, _DP, _DP, _DP]),
        "kapsel_gpu_make_phi_u": (ctypes.c_int, [_VP, _DP, _DP, _DP, _DP]),
        "kapsel_gpu_calc_f_hydro": (ctypes.c_int, [_VP, _DP, _DP, _DP, _DP, _DP]),
        "kapsel_gpu_calc_fr": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_calc_lj": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_make_phi": (ctypes.c_int, [_VP, _DP]),
        "kapsel_gpu_ns_slaved_euler": (ctypes.c_int, [_VP, _DP, _DP]),
        "kapsel_gpu_ns_solute_euler": (ctypes.c_int, [_VP, _DP, _DP, _DP]),
        "kapsel_gpu_rescale_solute": (ctypes.c_int, [_VP, _DP, _DP, _DP]),
        "kapsel_gpu_coulomb_force": (ctypes.c_int, [_VP, _DP, _DP, _DP, _DP]),
        "kapsel_gpu_md_position": (ctypes.c_int, [_VP, ctypes.c_int]),
        "kapsel_gpu_md_velocity": (ctypes.c_int, [_VP, _DP, _DP, ctypes.c_int]),
        "kapsel_gpu_set_time": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_double]),
        "kapsel_gpu_strerror": (ctypes.c_char_p, [ctypes.c_int]),
        "kapsel_gpu_step_kernel_name": (ctypes.c_char_p, [_VP, ctypes.c_int]),
        "kapsel_gpu_step_graph_particles": (ctypes.c_int, [_VP, ctypes.c_int, _DP]),
        "kapsel_gpu_save_restart": (ctypes.c_int, [_VP, ctypes.c_char_p]),
        "kapsel_gpu_write_avs": (ctypes.c_int, [_VP, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
        "kapsel_gpu_load_restart": (ctypes.c_int, [_VP, ctypes.c_char_p]),
        "kapsel_batch_create": (ctypes.c_int, [ctypes.POINTER(_VP), ctypes.c_int, ctypes.c_int,
                                               ctypes.POINTER(_VP)]),
        "kapsel_batch_step": (ctypes.c_int, [_VP, ctypes.c_int]),
        "kapsel_batch_msd": (ctypes.c_int, [_VP, _DP]),
        "kapsel_batch_get_stream": (ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
        "kapsel_batch_destroy": (ctypes.c_int, [_VP]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def read_udf_native(path: str) -> list:
    """The records of a UDF file as the library's C++ reader flattens them
    (kapsel_udf_read): a list of {path: value} dicts, one per data block;
    numbers as float, strings (and select values) as str."""
    L = load_library()
    L.kapsel_udf_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(_VP)]
    L.kapsel_udf_records.argtypes = [_VP]
    L.kapsel_udf_size.argtypes = [_VP, ctypes.c_int]
    L.kapsel_udf_entry.argtypes = [_VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                   ctypes.POINTER(ctypes.c_char_p), _IP]
    L.kapsel_udf_destroy.argtypes = [_VP]
    h = _VP()
    rc = L.kapsel_udf_read(str(path).encode(), ctypes.byref(h))
    if rc != 0:
        raise KapselError(f"kapsel_udf_read({path}) status {rc}")
    out = []
    try:
        for r in range(L.kapsel_udf_records(h)):
            rec = {}
            for i in range(L.kapsel_udf_size(h, r)):
                pth, txt, iss = ctypes.c_char_p(), ctypes.c_char_p(), ctypes.c_int()
                L.kapsel_udf_entry(h, r, i, ctypes.byref(pth), ctypes.byref(txt), ctypes.byref(iss))
                t = txt.value.decode()
                rec[pth.value.decode()] = t if iss.value else float(t)
            out.append(rec)
    finally:
        L.kapsel_udf_destroy(h)
    return out


def params_from_udf_native(path: str, precision: int = FP64):
    """(kapsel_params, x, q) from an input UDF through the C++ reader
    (kapsel_udf_to_params); x, q are None unless the file places the
    particles itself (user_specify)."""
    L = load_library()
    L.kapsel_udf_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(_VP)]
    L.kapsel_udf_to_params.argtypes = [_VP, ctypes.c_int, ctypes.POINTER(_Params), _DP, _DP, _IP]
    L.kapsel_udf_get_double.argtypes = [_VP, ctypes.c_int, ctypes.c_char_p, _DP]
    L.kapsel_udf_destroy.argtypes = [_VP]
    h = _VP()
    if L.kapsel_udf_read(str(path).encode(), ctypes.byref(h)) != 0:
        raise KapselError(f"kapsel_udf_read({path}) failed")
    try:
        p = _Params()
        nu = ctypes.c_int()
        rc = L.kapsel_udf_to_params(h, precision, ctypes.byref(p), None, None, ctypes.byref(nu))
        if rc != 0:
            raise KapselError(f"kapsel_udf_to_params status {rc}")
        x = q = None
        if nu.value > 0:
            x = np.zeros((nu.value, 3))
            q = np.zeros((nu.value, 4))
            L.kapsel_udf_to_params(h, precision, ctypes.byref(p), _ptr(x), _ptr(q), ctypes.byref(nu))
        return p, x, q
    finally:
        L.kapsel_udf_destroy(h)


def params_from_config(cfg: dict, precision: int = FP64) -> _Params:
    """Build kapsel_params from a configuration dict (the UDF values of one
    spherical-particle species; keys as in oracle/udf.py)."""
    L = load_library()
    p = _Params()
    L.kapsel_params_default(ctypes.byref(p))
    for d in range(3):
        p.np_xyz[d] = int(cfg["np_xyz"][d])
    eq = cfg.get("eq", "Navier_Stokes")
    if eq not in _EQ:
        raise KapselError(f"constitutive_eq {eq!r} is not supported")
    p.eq = _EQ[eq]
    p.shear_rate = float(cfg.get("shear_rate", 0.0))
    p.precision = precision
    p.n_particles = len(cfg.get("particles", []))
    p.dx = float(cfg.get("dx", 1.0))
    p.rho = float(cfg.get("rho", 1.0))
    p.eta = float(cfg.get("eta", 1.0))
    p.kbt = float(cfg.get("kbt", 0.0))
    p.alpha_v = float(cfg.get("alpha_v", 1.0))
    p.alpha_o = float(cfg.get("alpha_o", 1.0))
    p.dt = float(cfg.get("dt", 0.01))
    p.a = float(cfg.get("a", 5.0))
    p.a_xi = float(cfg.get("a_xi", 2.0))
    p.mass_ratio = float(cfg.get("mass_ratio", 1.0))
    p.gravity_g = float(cfg.get("gravity_g", 0.0))
    p.gravity_dir = {"-X": 0, "-Y": 1, "-Z": 2}[cfg.get("gravity_dir", "-Z")]
    p.epsilon = float(cfg.get("epsilon", 1.0))
    p.lj_powers = {"12:6": 0, "24:12": 1, "36:18": 2}[cfg.get("lj_powers", "12:6")]
    p.lj_truncate = {"ON": 1, "OFF": 0, "NONE": -1}[cfg.get("lj_truncate", "ON")]
    p.rotation = 1 if cfg.get("rotation", "ON") == "ON" else 0
    fc = cfg.get("fix_cell", (False, False, False))
    for d in range(3):
        p.fix_cell[d] = 1 if fc[d] else 0
    p.mt_seed = int(cfg.get("mt_seed", 0))
    p.frozen = 1 if cfg.get("frozen", False) else 0
    p.neighbor_lists = int(cfg.get("neighbor_lists", 0))
    el = cfg.get("electrolyte")
    if el:
        p.dielectric = float(el["dielectric"])
        p.surface_charge = float(el["surface_charge"])
        p.debye_length = float(el["debye"])
        p.valency_p = float(el.get("val_p", 1.0))
        p.valency_n = float(el.get("val_n", -1.0))
        p.onsager_p = float(el.get("onsager_p", 1.0))
        p.onsager_n = float(el.get("onsager_n", 1.0))
        for d, e in enumerate(el.get("efield", (0.0, 0.0, 0.0))):
            p.e_ext[d] = float(e)
    return p


class Simulation:
    """One SPM box on the GPU (one kapsel_ctx)."""

    def __init__(self, cfg: dict, precision: int = FP64, init: bool = True):
        self.L = load_library()
        self.cfg = cfg
        self.precision = precision
        self._p = params_from_config(cfg, precision)
        h = _VP()
        self._check(self.L.kapsel_gpu_create(ctypes.byref(self._p), ctypes.byref(h)))
        self.h = h
        d = (ctypes.c_int * 6)()
        self._check(self.L.kapsel_gpu_get_dims(self.h, d))
        self.NX, self.NY, self.NZ, self.NZ_, self.Np, self.S = list(d)
        if self.Np > 0:
            x = np.ascontiguousarray([p["x"] for p in cfg["particles"]], dtype=np.float64)
            qs = [p.get("q") for p in cfg["particles"]]
            q = None if all(v is None for v in qs) else np.ascontiguousarray(
                [v if v is not None else (1.0, 0.0, 0.0, 0.0) for v in qs], dtype=np.float64)
            self._check(self.L.kapsel_gpu_set_particles(self.h, _ptr(x), _ptr(q) if q is not None else None))
        if init:
            self.init_state()

    def _check(self, rc: int):
        if rc != 0:
            msg = load_library().kapsel_gpu_strerror(rc).decode()
            err = KapselError(f"kapsel_gpu status {rc}: {msg}")
            err.code = rc
            raise err

    def close(self):
        if getattr(self, "h", None):
            self.L.kapsel_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state evolution
    def init_state(self):
        self._check(self.L.kapsel_gpu_init_state(self.h))

    def step(self, n: int = 1, graph: bool = False):
        f = self.L.kapsel_gpu_step_graph if graph else self.L.kapsel_gpu_step
        self._check(f(self.h, int(n)))

    def step_particles(self, n: int = 1) -> dict:
        """n graph-replayed steps, then the particle records, with one host
        synchronisation (kapsel_gpu_step_graph_particles)."""
        a = np.zeros((max(self.Np, 1), P_STRIDE))
        self._check(self.L.kapsel_gpu_step_graph_particles(self.h, int(n), _ptr(a)))
        return self._records(a)

    def step_kernel_names(self) -> list:
        """The kernel of each profiling slot (kapsel_gpu_profile_step) for
        this context's pass variants; "" for a slot with no launch."""
        return [self.L.kapsel_gpu_step_kernel_name(self.h, i).decode() for i in range(13)]

    def time(self):
        ts = ctypes.c_int()
        t = ctypes.c_double()
        self._check(self.L.kapsel_gpu_get_time(self.h, ctypes.byref(ts), ctypes.byref(t)))
        return ts.value, t.value

    # ---- state readout in the reference layouts
    def zeta(self) -> np.ndarray:
        z = np.zeros((2, self.NX, self.NY, self.NZ_))
        self._check(self.L.kapsel_gpu_get_zeta(self.h, _ptr(z), None))
        return z

    def uk_dc(self) -> np.ndarray:
        z = np.zeros((2, self.NX, self.NY, self.NZ_))
        u = np.zeros(3)
        self._check(self.L.kapsel_gpu_get_zeta(self.h, _ptr(z), _ptr(u)))
        return u

    def set_zeta(self, zeta: np.ndarray, uk_dc):
        z = np.ascontiguousarray(zeta, dtype=np.float64)
        u = np.ascontiguousarray(uk_dc, dtype=np.float64)
        self._check(self.L.kapsel_gpu_set_zeta(self.h, _ptr(z), _ptr(u)))

    def velocity(self) -> np.ndarray:
        """u = Zeta_k2u(zeta, uk_dc), shape (3, NX, NY, NZ)."""
        u = np.zeros((3, self.NX, self.NY, self.NZ_))
        self._check(self.L.kapsel_gpu_get_velocity(self.h, _ptr(u)))
        return u[..., : self.NZ].copy()

    def particles(self) -> dict:
        a = np.zeros((max(self.Np, 1), P_STRIDE))
        self._check(self.L.kapsel_gpu_get_particles(self.h, _ptr(a)))
        return self._records(a)

    def _records(self, a: np.ndarray) -> dict:
        a = a[: self.Np]
        names = ["x", "v", "omega", "f_hydro", "torque_hydro", "fr", "x_nopbc", "v_old", "omega_old"]
        out = {n: a[:, 3 * i: 3 * i + 3].copy() for i, n in enumerate(names)}
        out["q"] = a[:, 27:31].copy()
        out["q_old"] = a[:, 31:35].copy()
        return out

    def set_particle_state(self, st: dict):
        a = np.zeros((max(self.Np, 1), P_STRIDE))
        names = ["x", "v", "omega", "f_hydro", "torque_hydro", "fr", "x_nopbc", "v_old", "omega_old"]
        for i, n in enumerate(names):
            a[: self.Np, 3 * i: 3 * i + 3] = st[n]
        a[: self.Np, 27:31] = st["q"]
        a[: self.Np, 31:35] = st["q_old"]
        self._check(self.L.kapsel_gpu_set_particle_state(self.h, _ptr(a)))

    def save_restart(self, path: str):
        """Write the restart records (Save_Restart_udf paths, text)."""
        self._check(self.L.kapsel_gpu_save_restart(self.h, str(path).encode()))

    def load_restart(self, path: str):
        """Restore from restart records as Force_restore_parameters does."""
        self._check(self.L.kapsel_gpu_load_restart(self.h, str(path).encode()))

    def write_avs(self, out_dir: str, out_name: str, nstep: int, init: bool = False):
        """Append an AVS field snapshot (Output_avs, binary, uniform field)."""
        self._check(self.L.kapsel_gpu_write_avs(self.h, str(out_dir).encode(), str(out_name).encode(), int(nstep),
                                                1 if init else 0))

    def concentration(self) -> np.ndarray:
        """Ion concentrations (2, NX, NY, NZ_) in the Ooura layout (Electrolyte)."""
        c = np.zeros((2, self.NX, self.NY, self.NZ_))
        self._check(self.L.kapsel_gpu_get_concentration(self.h, _ptr(c)))
        return c

    def set_efield(self, e):
        a = np.ascontiguousarray(e, dtype=np.float64)
        self._check(self.L.kapsel_gpu_set_efield(self.h, _ptr(a)))

    def udf_record(self) -> dict:
        """One Output_udf record of the current state (avs_output.cxx:343-450):
        E (the reference writes 1.0), t = jikan.ts and, per particle, R, R_raw
        (unwrapped), v, q, omega, the previous step's f_hydro, torque_hydro and
        f_r, and zero torque_r, f_slip, torque_slip (spherical, no slip).
        Nested as the outParticle class of define.udf, for udf_io.write_records."""
        ts, _ = self.time()
        p = self.particles()
        v3 = lambda a: {"x": float(a[0]), "y": float(a[1]), "z": float(a[2])}
        zero = {"x": 0.0, "y": 0.0, "z": 0.0}
        parts = []
        for n in range(self.Np):
            q = p["q"][n]
            parts.append({"R": v3(p["x"][n]), "R_raw": v3(p["x_nopbc"][n]), "v": v3(p["v"][n]),
                          "q": {"q0": float(q[0]), "q1": float(q[1]), "q2": float(q[2]), "q3": float(q[3])},
                          "omega": v3(p["omega"][n]), "f_hydro": v3(p["f_hydro"][n]),
                          "torque_hydro": v3(p["torque_hydro"][n]), "f_r": v3(p["fr"][n]),
                          "torque_r": dict(zero), "f_slip": dict(zero), "torque_slip": dict(zero)})
        return {"E": 1.0, "t": ts, "Particles": parts}

    def oblique(self) -> dict:
        """Lees-Edwards state: degree_oblique, Shear_rate_eff, Shear_strain_realized."""
        a = np.zeros(3)
        self._check(self.L.kapsel_gpu_get_oblique(self.h, _ptr(a)))
        return {"degree_oblique": float(a[0]), "shear_rate_eff": float(a[1]), "strain": float(a[2])}

    def set_oblique(self, degree_oblique: float, shear_rate_eff: float):
        self._check(self.L.kapsel_gpu_set_oblique(self.h, float(degree_oblique), float(shear_rate_eff)))

    # ---- routine-level entry points (reference layouts, NX*NY*NZ_ doubles)
    def _padded(self, a):
        b = np.zeros((self.NX, self.NY, self.NZ_))
        b[:, :, : a.shape[2]] = a
        return b

    def A2a_k(self, a: np.ndarray) -> np.ndarray:
        b = self._padded(a)
        self._check(self.L.kapsel_gpu_A2a_k(self.h, _ptr(b)))
        return b

    def A_k2a(self, ak: np.ndarray) -> np.ndarray:
        b = np.ascontiguousarray(ak, dtype=np.float64).copy()
        self._check(self.L.kapsel_gpu_A_k2a(self.h, _ptr(b)))
        return b[:, :, : self.NZ].copy()

    def solenoidal_u(self, u: np.ndarray) -> np.ndarray:
        b = [self._padded(u[d]) for d in range(3)]
        self._check(self.L.kapsel_gpu_solenoidal_u(self.h, _ptr(b[0]), _ptr(b[1]), _ptr(b[2])))
        return np.stack([x[:, :, : self.NZ] for x in b])

    def make_phi_u(self):
        f = [np.zeros((self.NX, self.NY, self.NZ_)) for _ in range(4)]
        self._check(self.L.kapsel_gpu_make_phi_u(self.h, *[_ptr(x) for x in f]))
        return f[0][:, :, : self.NZ].copy(), np.stack([x[:, :, : self.NZ] for x in f[1:]])

    def calc_f_hydro(self, u: np.ndarray):
        b = [self._padded(u[d]) for d in range(3)]
        f = np.zeros((max(self.Np, 1), 3))
        t = np.zeros((max(self.Np, 1), 3))
        self._check(self.L.kapsel_gpu_calc_f_hydro(self.h, _ptr(b[0]), _ptr(b[1]), _ptr(b[2]), _ptr(f), _ptr(t)))
        return f[: self.Np], t[: self.Np]

    def calc_fr(self) -> np.ndarray:
        f = np.zeros((max(self.Np, 1), 3))
        self._check(self.L.kapsel_gpu_calc_fr(self.h, _ptr(f)))
        return f[: self.Np]


class Batch:
    """Independent boxes advanced together, one CUDA graph launch per step
    (kapsel_batch_*).  The Simulation objects stay owned by the caller."""

    def __init__(self, sims, autotune: bool = True):
        self.L = load_library()
        self.sims = list(sims)
        arr = (_VP * len(self.sims))(*[s.h for s in self.sims])
        h = _VP()
        rc = self.L.kapsel_batch_create(arr, len(self.sims), 1 if autotune else 0, ctypes.byref(h))
        if rc != 0:
            raise KapselError(f"kapsel_batch_create status {rc}: {self.L.kapsel_gpu_strerror(rc).decode()}")
        self.h = h

    def step(self, n: int = 1):
        rc = self.L.kapsel_batch_step(self.h, int(n))
        if rc != 0:
            raise KapselError(f"kapsel_batch_step status {rc}: {self.L.kapsel_gpu_strerror(rc).decode()}")

    def msd(self) -> np.ndarray:
        out = np.zeros(len(self.sims))
        rc = self.L.kapsel_batch_msd(self.h, _ptr(out))
        if rc != 0:
            raise KapselError(f"kapsel_batch_msd status {rc}")
        return out

    def stream(self) -> int:
        sp = _VP()
        self.L.kapsel_batch_get_stream(self.h, ctypes.byref(sp))
        return sp.value

    def variants(self) -> list:
        """The autotuner's choice per box shape: (NX, NY, NZ, z variant,
        y variant, x split); z 0 warp-level / 1 block-level, y 0 warp-level /
        1 block-level wide tile / 2 block-level narrow tile / 3 warp-level
        with the fused y/z plane kernels, x split 0 default / 1 the other
        radix factorisation of NX."""
        self.L.kapsel_batch_variants.argtypes = [_VP, _IP, ctypes.c_int]
        buf = (ctypes.c_int * (6 * 64))()
        n = self.L.kapsel_batch_variants(self.h, buf, 64)
        return [tuple(buf[6 * i: 6 * i + 6]) for i in range(max(n, 0))]

    def close(self):
        if getattr(self, "h", None):
            self.L.kapsel_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["Batch", "Simulation", "KapselError", "load_library", "params_from_config", "FP64", "MIXED", "LIB_PATH"]


def simulation_from_udf(path: str, precision: int = FP64, seed: int = 0) -> "Simulation":
    """A Simulation configured from a KAPSEL input UDF (its define.udf
    resolved through \\include); see udf_io.to_config for what is supported."""
    from . import udf_io

    return Simulation(udf_io.to_config(udf_io.read(path), seed=seed), precision=precision)
