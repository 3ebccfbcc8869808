"""ctypes access to the reference oracle built by oracle/Makefile (oracle/_ref).

TEST INFRASTRUCTURE ONLY.  Only tests/, tests/golden/make_golden.py and the
CPU arms of bench.py use this module, as a checker or a timed baseline.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

from . import udf

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
P_STRIDE = 35  # doubles per particle in kref_get_particles


def lib_path(omp: bool = False) -> str:
    return os.path.join(REF_DIR, "libkapsel_ref_omp.so" if omp else "libkapsel_ref.so")


def available(omp: bool = False) -> bool:
    return os.path.exists(lib_path(omp))


class RefSim:
    """One reference simulation.  The reference keeps global state, so each
    instance loads its own private copy of the library (copied to a temp file)."""

    def __init__(self, cfg: dict | None, omp: bool = False, workdir: str | None = None, kv_path: str | None = None):
        self._tmp = tempfile.mkdtemp(prefix="kref_", dir=workdir)
        src = lib_path(omp)
        dst = os.path.join(self._tmp, "lib.so")
        with open(src, "rb") as f, open(dst, "wb") as g:
            g.write(f.read())
        self.lib = ctypes.CDLL(dst, mode=ctypes.RTLD_LOCAL)
        L = self.lib
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.kref_init.argtypes = [ctypes.c_char_p]
        L.kref_step.argtypes = [ctypes.c_int]
        L.kref_dims.argtypes = [ip]
        L.kref_scalars.argtypes = [dp]
        L.kref_get_field.argtypes = [ctypes.c_int, dp]
        L.kref_set_field.argtypes = [ctypes.c_int, dp]
        L.kref_get_ukdc.argtypes = [dp]
        L.kref_set_ukdc.argtypes = [dp]
        L.kref_get_particles.argtypes = [dp]
        L.kref_set_efield.argtypes = [ctypes.c_double] * 3
        L.kref_sekibun.argtypes = [ip]
        L.kref_A2a_k.argtypes = [dp]
        L.kref_A_k2a.argtypes = [dp]
        L.kref_solenoidal_u.argtypes = [dp, dp, dp]
        L.kref_save_restart.argtypes = [ctypes.c_char_p]
        L.kref_output_avs.argtypes = [ctypes.c_int]
        L.kref_resume.argtypes = [ctypes.c_char_p]
        L.kref_time_steps.argtypes = [ctypes.c_int]
        L.kref_time_steps.restype = ctypes.c_double
        L.kref_oblique.argtypes = [dp]
        L.kref_output_udf.argtypes = []
        L.kref_set_particle_velocity.argtypes = [ctypes.c_int, dp, dp]
        L.kref_set_oblique.argtypes = [ctypes.c_double, ctypes.c_double]
        self.cfg = cfg
        self.kv = kv_path or udf.write_udf(os.path.join(self._tmp, "input.kv"), cfg)
        rc = L.kref_init(self.kv.encode())
        if rc != 0:
            raise RuntimeError(f"kref_init failed: {rc}")
        d = (ctypes.c_int * 8)()
        L.kref_dims(d)
        self.NX, self.NY, self.NZ, self.NZ_, self.Np, self.NPdomain, self.Nspec, self.eq = list(d)

    @staticmethod
    def _p(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def step(self, n: int = 1):
        self.lib.kref_step(n)

    def save_restart(self, path: str):
        """Save_Restart_udf through the stand-in record writer."""
        assert self.lib.kref_save_restart(str(path).encode()) == 0

    def resume(self, path: str):
        """The first pass of a resumed run: one step, then Force_restore_parameters."""
        assert self.lib.kref_resume(str(path).encode()) == 0

    def output_avs(self, init: bool = False):
        """Output_avs of the current state (needs cfg["avs"])."""
        assert self.lib.kref_output_avs(1 if init else 0) == 0

    def ts(self) -> int:
        return int(self.lib.kref_ts())

    def time_steps(self, n: int) -> float:
        return self.lib.kref_time_steps(n)

    def scalars(self):
        s = np.zeros(16)
        self.lib.kref_scalars(self._p(s))
        return dict(zip(["dt", "nu", "radius", "xi", "hxi", "mass", "moi", "kbt", "time"], s[:9]))

    def field(self, which: int) -> np.ndarray:
        a = np.zeros(self.NX * self.NY * self.NZ_)
        if self.lib.kref_get_field(which, self._p(a)) != 0:
            raise KeyError(which)
        return a.reshape(self.NX, self.NY, self.NZ_)

    def set_field(self, which: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        if self.lib.kref_set_field(which, self._p(a)) != 0:
            raise KeyError(which)

    def u(self):
        return np.stack([self.field(i)[:, :, : self.NZ] for i in range(3)])

    def zeta(self):
        return np.stack([self.field(7), self.field(8)])

    def phi(self):
        return self.field(3)[:, :, : self.NZ]

    def ucp(self):
        """Lees-Edwards: the Cartesian velocity of the last step (ucp)."""
        return np.stack([self.field(12 + i)[:, :, : self.NZ] for i in range(3)])

    def oblique(self) -> dict:
        a = np.zeros(3)
        self.lib.kref_oblique(self._p(a))
        return {"degree_oblique": float(a[0]), "shear_rate_eff": float(a[1]), "strain": float(a[2])}

    def output_udf(self):
        """Output_udf of the current state (appends one record)."""
        assert self.lib.kref_output_udf() == 0

    def udf_records(self) -> list:
        """The output records written so far: list of {path: value text},
        record 0 first (the stand-in manager's "record <n> path = value" lines)."""
        recs = []
        with open(self.kv + ".out") as f:
            for line in f:
                head, _, val = line.rstrip("\n").partition(" = ")
                _, n, path = head.split(" ", 2)
                n = int(n)
                while len(recs) <= n:
                    recs.append({})
                recs[n][path] = val
        return recs

    def set_particle_velocity(self, n: int, v, omega):
        v = np.ascontiguousarray(v, dtype=np.float64)
        w = np.ascontiguousarray(omega, dtype=np.float64)
        assert self.lib.kref_set_particle_velocity(int(n), self._p(v), self._p(w)) == 0

    def set_oblique(self, deg: float, srate: float):
        assert self.lib.kref_set_oblique(float(deg), float(srate)) == 0

    def up(self):
        return np.stack([self.field(4 + i)[:, :, : self.NZ] for i in range(3)])

    def uk_dc(self):
        a = np.zeros(3)
        self.lib.kref_get_ukdc(self._p(a))
        return a

    def set_uk_dc(self, v):
        a = np.ascontiguousarray(v, dtype=np.float64)
        self.lib.kref_set_ukdc(self._p(a))

    def particles(self) -> dict:
        a = np.zeros(max(self.Np, 1) * P_STRIDE)
        self.lib.kref_get_particles(self._p(a))
        a = a[: self.Np * P_STRIDE].reshape(self.Np, P_STRIDE)
        names = ["x", "v", "omega", "f_hydro", "torque_hydro", "fr", "x_nopbc", "v_old", "omega_old"]
        out = {n: a[:, 3 * i: 3 * i + 3].copy() for i, n in enumerate(names)}
        out["q"] = a[:, 27:31].copy()
        out["q_old"] = a[:, 31:35].copy()
        return out

    def sekibun(self) -> np.ndarray:
        n = self.lib.kref_sekibun(None)
        a = (ctypes.c_int * (3 * n))()
        self.lib.kref_sekibun(a)
        return np.frombuffer(a, dtype=np.int32).reshape(n, 3).copy()

    def A2a_k(self, a: np.ndarray) -> np.ndarray:
        b = np.zeros((self.NX, self.NY, self.NZ_))
        b[:, :, : a.shape[2]] = a
        b = np.ascontiguousarray(b)
        self.lib.kref_A2a_k(self._p(b))
        return b

    def A_k2a(self, a: np.ndarray) -> np.ndarray:
        b = np.ascontiguousarray(a, dtype=np.float64).copy()
        self.lib.kref_A_k2a(self._p(b))
        return b[:, :, : self.NZ]

    def set_efield(self, e):
        self.lib.kref_set_efield(*[float(x) for x in e])
