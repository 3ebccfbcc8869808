"""Learned near-contact correction of the SPM hydrodynamic force.

At a/dx ~ 5 the smoothed interface (xi = 2) is under-resolved, and the
force/torque the method gives two close spheres differs from the one it
gives the same geometry at twice the resolution.  This module

* generates training pairs with the method itself (two spheres held at a
  gap with prescribed velocities, the "frozen" mode of the GPU step, FP64),
  once on a coarse grid (64^3, a = 5) and once on a fine grid (128^3,
  a = 10) in dynamically similar units;
* trains a 16-128-128-128-16 SiLU network on the GPU with the library's own
  tcgen05 BF16 forward/backward kernels (kapsel_nc_train);
* attaches the trained network to a coarse simulation, whose step then
  corrects every pair inside the trained gap range and keeps the plain SPM
  force elsewhere (kapsel_gpu_set_nearcontact).

Dynamic similarity.  With rho = eta = dx = 1 on both grids, lengths scale by
2 (box 64 -> 128, a 5 -> 10), times by 4 (a^2/nu) and velocities by 1/2,
which leaves the Navier-Stokes equations and the Reynolds number unchanged;
forces are then equal and torques scale by 2.  The fine run therefore uses
dt_f = 4 dt_c, v_f = v_c / 2, omega_f = omega_c / 4, the same number of
steps, and reports F_f and T_f / 2 in coarse units.  Only the interface
thickness relative to a differs (xi/a = 0.4 vs 0.2): that is the
resolution error the network learns.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import FP64, KapselError, Simulation, _DP, _VP, load_library

NC_IN, NC_OUT, NPARAM = 16, 16, 37264
_FP = ctypes.POINTER(ctypes.c_float)

# the training protocol (coarse units)
COARSE = dict(np_xyz=(6, 6, 6), a=5.0)
FINE = dict(np_xyz=(7, 7, 7), a=10.0)
GAP_LO, GAP_HI = 0.05, 2.0   # surface gap / a, log-uniform
V_MAX = 0.1                   # |v2 - v1|
W_MAX = 0.1 / 5.0             # |omega| a <= 0.1
DT_C = 0.1                    # coarse time step; fine uses 4x
N_STEPS = 250                 # t = 25 = a^2/nu in coarse units


def _lib():
    L = load_library()
    if not getattr(L, "_nc_sig", False):
        sig = {
            "kapsel_nc_create": (ctypes.c_int, [_FP, ctypes.POINTER(_VP)]),
            "kapsel_nc_destroy": (ctypes.c_int, [_VP]),
            "kapsel_nc_get_params": (ctypes.c_int, [_VP, _FP]),
            "kapsel_nc_set_params": (ctypes.c_int, [_VP, _FP]),
            "kapsel_nc_forward": (ctypes.c_int, [_VP, _FP, ctypes.c_int, _FP]),
            "kapsel_nc_gradient": (ctypes.c_int, [_VP, _FP, _FP, _FP, ctypes.c_int, _FP, _FP]),
            "kapsel_nc_train": (ctypes.c_int, [_VP, _FP, _FP, _FP, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_float, ctypes.c_uint, _FP]),
            "kapsel_nc_set_scaling": (ctypes.c_int, [_VP, _FP, _FP, _FP, ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_double]),
            "kapsel_nc_pair_features": (ctypes.c_int, [_VP, _DP, _DP, _DP, _FP, _FP, _DP]),
            "kapsel_gpu_set_nearcontact": (ctypes.c_int, [_VP, _VP]),
            "kapsel_gpu_nearcontact_pairs": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        L._nc_sig = True
    return L


def _f32(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_FP)


def _check(rc: int):
    if rc != 0:
        raise KapselError(f"kapsel_nc status {rc}: {load_library().kapsel_gpu_strerror(rc).decode()}")


# ---------------------------------------------------------------------------
# pair features (the same arithmetic as nc_frame / nc_features on the device)
def pair_frame(d: np.ndarray) -> np.ndarray:
    """Rows e1, e2, e3 of the pair frame for centre lines d[..., 3]."""
    d = np.asarray(d, np.float64)
    e1 = d / np.linalg.norm(d, axis=-1, keepdims=True)
    near_z = np.abs(e1[..., 2]) > 0.9
    h = np.zeros_like(e1)
    h[..., 0] = np.where(near_z, 1.0, 0.0)
    h[..., 2] = np.where(near_z, 0.0, 1.0)
    e2 = np.cross(e1, h)
    e2 /= np.linalg.norm(e2, axis=-1, keepdims=True)
    e3 = np.cross(e1, e2)
    return np.stack([e1, e2, e3], axis=-2)


def raw_features(gap_over_a, e, v1, v2, w1, w2) -> np.ndarray:
    """[log(gap/a), (v2-v1).e_k, w1.e_k, w2.e_k] (10 values per pair)."""
    g = np.atleast_1d(np.asarray(gap_over_a, np.float64))
    out = np.zeros(g.shape + (10,))
    out[..., 0] = np.log(g)
    out[..., 1:4] = np.einsum("...kj,...j->...k", e, np.asarray(v2) - np.asarray(v1))
    out[..., 4:7] = np.einsum("...kj,...j->...k", e, np.asarray(w1))
    out[..., 7:10] = np.einsum("...kj,...j->...k", e, np.asarray(w2))
    return out


# ---------------------------------------------------------------------------
def init_params(seed: int) -> np.ndarray:
    """He-uniform weights (SiLU), zero biases, last layer scaled by 0.1;
    PCG64(seed).  Packed order W1 b1 W2 b2 W3 b3 W4 b4, W[out][in]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shapes = [(128, 16), (128,), (128, 128), (128,), (128, 128), (128,), (16, 128), (16,)]
    parts = []
    for i, s in enumerate(shapes):
        if len(s) == 1:
            parts.append(np.zeros(s, np.float32))
        else:
            lim = math.sqrt(6.0 / s[1]) * (0.1 if i == 6 else 1.0)
            parts.append(rng.uniform(-lim, lim, size=s).astype(np.float32))
    p = np.concatenate([a.reshape(-1) for a in parts])
    assert p.size == NPARAM
    return p


class NearContactNet:
    """The correction network on the GPU (one kapsel_nc)."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        self.L = _lib()
        p = _f32(init_params(seed) if params is None else params)
        if p.size != NPARAM:
            raise ValueError(f"expected {NPARAM} parameters")
        h = _VP()
        _check(self.L.kapsel_nc_create(_fp(p), ctypes.byref(h)))
        self.h = h
        self.scaling = None

    def close(self):
        if getattr(self, "h", None):
            self.L.kapsel_nc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(NPARAM, np.float32)
        _check(self.L.kapsel_nc_get_params(self.h, _fp(p)))
        return p

    @params.setter
    def params(self, p):
        p = _f32(p)
        _check(self.L.kapsel_nc_set_params(self.h, _fp(p)))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = _f32(x, (-1, NC_IN))
        y = np.zeros((x.shape[0], NC_OUT), np.float32)
        _check(self.L.kapsel_nc_forward(self.h, _fp(x), x.shape[0], _fp(y)))
        return y

    def gradient(self, x, y, colw):
        x = _f32(x, (-1, NC_IN))
        y = _f32(y, (-1, NC_OUT))
        w = _f32(colw, (NC_OUT,))
        g = np.zeros(NPARAM, np.float32)
        loss = np.zeros(1, np.float32)
        _check(self.L.kapsel_nc_gradient(self.h, _fp(x), _fp(y), _fp(w), x.shape[0], _fp(g), _fp(loss)))
        return g, float(loss[0])

    def train(self, x, y, colw, epochs: int, batch: int = 256, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        x = _f32(x, (-1, NC_IN))
        y = _f32(y, (-1, NC_OUT))
        w = _f32(colw, (NC_OUT,))
        hist = np.zeros(epochs, np.float32)
        _check(self.L.kapsel_nc_train(self.h, _fp(x), _fp(y), _fp(w), x.shape[0], int(epochs), int(batch),
                                      float(lr), int(seed), _fp(hist)))
        return hist

    def set_scaling(self, in_shift, in_scale, out_scale, a: float, gap_lo: float = GAP_LO,
                    gap_hi: float = GAP_HI):
        s0, s1, s2 = (_f32(np.resize(np.asarray(v, np.float32), 16)) for v in (in_shift, in_scale, out_scale))
        _check(self.L.kapsel_nc_set_scaling(self.h, _fp(s0), _fp(s1), _fp(s2), float(a), float(gap_lo),
                                            float(gap_hi)))
        self.scaling = dict(in_shift=s0, in_scale=s1, out_scale=s2, a=float(a), gap_lo=gap_lo, gap_hi=gap_hi)

    def pair_features(self, rec_i, rec_j, box):
        """Device feature arithmetic evaluated on the host (for checks)."""
        ri = np.ascontiguousarray(rec_i, np.float64)
        rj = np.ascontiguousarray(rec_j, np.float64)
        b = np.ascontiguousarray(box, np.float64)
        f = np.zeros(16, np.float32)
        e = np.zeros(9, np.float32)
        gap = ctypes.c_double()
        _check(self.L.kapsel_nc_pair_features(self.h, ri.ctypes.data_as(_DP), rj.ctypes.data_as(_DP),
                                              b.ctypes.data_as(_DP), _fp(f), _fp(e), ctypes.byref(gap)))
        return f, e.reshape(3, 3), gap.value

    def features(self, raw: np.ndarray) -> np.ndarray:
        """Scaled, zero-padded network inputs from raw_features rows."""
        s = self.scaling
        out = np.zeros(raw.shape[:-1] + (16,), np.float32)
        out[..., :10] = ((raw - s["in_shift"][:10].astype(np.float64)) * s["in_scale"][:10].astype(np.float64))
        return out

    def predict(self, raw: np.ndarray) -> np.ndarray:
        """Corrections (n, 12) in the pair frame for raw feature rows."""
        y = self.forward(self.features(raw))
        return y[:, :12] * self.scaling["out_scale"][:12]


def attach(sim: Simulation, net: NearContactNet | None):
    """Attach (or with None detach) a trained, scaled network to a simulation."""
    L = _lib()
    rc = L.kapsel_gpu_set_nearcontact(sim.h, net.h if net is not None else None)
    sim._check(rc)
    sim._nc = net  # keep the network alive while attached


def corrected_pairs(sim: Simulation) -> int:
    n = ctypes.c_int()
    sim._check(_lib().kapsel_gpu_nearcontact_pairs(sim.h, ctypes.byref(n)))
    return n.value


# ---------------------------------------------------------------------------
# training pairs
def sample_pairs(n: int, seed: int = 5) -> dict:
    """Pair configurations in coarse units, PCG64(seed): gap/a log-uniform in
    [GAP_LO, GAP_HI]; v2 - v1 uniform in the ball |v| <= V_MAX (v1 = -v/2,
    v2 = +v/2); omega1, omega2 uniform in the ball |omega| a <= 0.1; centre
    line along x; a sub-cell offset of the pair centre uniform in [0, 1)^3."""
    rng = np.random.Generator(np.random.PCG64(seed))

    def ball(r, m):
        v = rng.normal(size=(m, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        return v * (r * rng.random(m) ** (1.0 / 3.0))[:, None]

    gap = np.exp(rng.uniform(np.log(GAP_LO), np.log(GAP_HI), size=n))
    return dict(gap=gap, v=ball(V_MAX, n), w1=ball(W_MAX, n), w2=ball(W_MAX, n), offset=rng.random((n, 3)))


def _pair_cfg(level: dict, dt: float) -> dict:
    N = 1 << level["np_xyz"][0]
    a = level["a"]
    return {"eq": "Navier_Stokes", "np_xyz": level["np_xyz"], "a": a, "a_xi": 2.0, "kbt": 0.0, "dt": dt,
            "frozen": True, "lj_truncate": "NONE",
            "particles": [{"x": (N / 2 - a - 1.0, N / 2, N / 2)}, {"x": (N / 2 + a + 1.0, N / 2, N / 2)}]}


class PairRunner:
    """Runs frozen two-sphere configurations on one context per level."""

    def __init__(self, level: dict, scale: float, steps: int = N_STEPS, dt_c: float = DT_C):
        self.s = scale  # length scale of this level relative to coarse (1 or 2)
        self.steps = steps
        self.a_c = COARSE["a"]
        self.sim = Simulation(_pair_cfg(level, dt_c * scale * scale), FP64, init=False)
        self.N = 1 << level["np_xyz"][0]

    def forces(self, gap, v, w1, w2, offset) -> np.ndarray:
        """[F1, T1, F2, T2] in coarse units for one configuration."""
        s, a = self.s, self.a_c
        half = a + 0.5 * gap * a  # centre half-distance, coarse units
        c = self.N / 2 + s * np.asarray(offset)
        x = np.array([c - [s * half, 0, 0], c + [s * half, 0, 0]])
        L = self.sim.L
        xs = np.ascontiguousarray(x)
        self.sim._check(L.kapsel_gpu_set_particles(self.sim.h, xs.ctypes.data_as(_DP), None))
        self.sim.init_state()
        st = self.sim.particles()
        st["v"] = np.array([-0.5 * np.asarray(v), 0.5 * np.asarray(v)]) / s
        st["omega"] = np.array([w1, w2]) / (s * s)
        st["v_old"] = st["v"].copy()
        st["omega_old"] = st["omega"].copy()
        self.sim.set_particle_state(st)
        self.sim.step(self.steps, graph=True)
        p = self.sim.particles()
        return np.concatenate([p["f_hydro"][0], p["torque_hydro"][0] / s, p["f_hydro"][1],
                               p["torque_hydro"][1] / s])

    def close(self):
        self.sim.close()


def generate(n: int, seed: int = 5, steps: int = N_STEPS, progress=None) -> dict:
    """n training pairs: inputs and the coarse and fine forces (coarse units)."""
    cfg = sample_pairs(n, seed)
    coarse = PairRunner(COARSE, 1.0, steps)
    fine = PairRunner(FINE, 2.0, steps)
    fc = np.zeros((n, 12))
    ff = np.zeros((n, 12))
    for i in range(n):
        args = (cfg["gap"][i], cfg["v"][i], cfg["w1"][i], cfg["w2"][i], cfg["offset"][i])
        fc[i] = coarse.forces(*args)
        ff[i] = fine.forces(*args)
        if progress and (i + 1) % progress == 0:
            print(f"pairs {i + 1}/{n}", flush=True)
    coarse.close()
    fine.close()
    cfg.update(f_coarse=fc, f_fine=ff, steps=steps, dt_c=DT_C)
    return cfg


def dataset_raw(data: dict) -> np.ndarray:
    """Raw features of generated pairs (centre line along +x)."""
    n = len(data["gap"])
    e = pair_frame(np.tile([1.0, 0.0, 0.0], (n, 1)))
    v = np.asarray(data["v"])
    return raw_features(data["gap"], e, -0.5 * v, 0.5 * v, data["w1"], data["w2"])


def to_pair_frame(f12: np.ndarray, e: np.ndarray) -> np.ndarray:
    """Rotate [F1, T1, F2, T2] (box frame) into the pair frame e (rows e1..e3)."""
    f = np.asarray(f12).reshape(f12.shape[:-1] + (4, 3))
    return np.einsum("...kj,...vj->...vk", e, f).reshape(f12.shape)


def fit(data: dict, train_idx, epochs: int = 400, batch: int = 128, lr: float = 2e-3, seed: int = 0,
        init_seed: int = 0):
    """Train a network on data[train_idx]; returns (net, loss history)."""
    raw = dataset_raw(data)
    n = len(data["gap"])
    e = pair_frame(np.tile([1.0, 0.0, 0.0], (n, 1)))
    target = to_pair_frame(data["f_fine"] - data["f_coarse"], e)
    tr = np.asarray(train_idx)
    shift = np.zeros(16, np.float32)
    scale = np.ones(16, np.float32)
    shift[:10] = raw[tr].mean(0)
    scale[:10] = 1.0 / np.maximum(raw[tr].std(0), 1e-12)
    out_scale = np.ones(16, np.float32)
    out_scale[:12] = np.maximum(np.sqrt((target[tr] ** 2).mean(0)), 1e-12)
    net = NearContactNet(seed=init_seed)
    net.set_scaling(shift, scale, out_scale, a=COARSE["a"])
    x = net.features(raw[tr])
    y = np.zeros((len(tr), 16), np.float32)
    y[:, :12] = target[tr] / out_scale[:12]
    colw = np.zeros(16, np.float32)
    colw[:12] = 1.0
    hist = []
    # step decay of the learning rate over three stages
    for k, f in enumerate((1.0, 0.3, 0.1)):
        hist.append(net.train(x, y, colw, epochs // 3, batch, lr * f, seed + k))
    return net, np.concatenate(hist)


def errors(net: NearContactNet, data: dict, idx) -> dict:
    """RMS force and torque error against the fine run, plain and corrected."""
    idx = np.asarray(idx)
    n = len(data["gap"])
    e = pair_frame(np.tile([1.0, 0.0, 0.0], (n, 1)))[idx]
    raw = dataset_raw(data)[idx]
    corr = net.predict(raw)                              # pair frame
    fc = to_pair_frame(data["f_coarse"][idx], e)
    ff = to_pair_frame(data["f_fine"][idx], e)
    fl = fc + corr
    F = np.r_[0:3, 6:9]
    T = np.r_[3:6, 9:12]

    def rms(a):
        return float(np.sqrt(np.mean(a ** 2)))

    return dict(force_plain=rms(fc[:, F] - ff[:, F]), force_learned=rms(fl[:, F] - ff[:, F]),
                torque_plain=rms(fc[:, T] - ff[:, T]), torque_learned=rms(fl[:, T] - ff[:, T]),
                force_scale=rms(ff[:, F]), torque_scale=rms(ff[:, T]))
