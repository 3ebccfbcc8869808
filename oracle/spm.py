"""CPU restatement (FP64, numpy) of KAPSEL's Smoothed Profile Method time step.

TEST INFRASTRUCTURE ONLY.  This module is the oracle: tests/, the smoke check
and the CPU leg of bench.py call it to check the CUDA path.  The product never
imports it.  Its own correctness is pinned against the unmodified reference
(oracle/_ref, built by oracle/Makefile) through the golden fixtures in
tests/golden/ (tests/golden/make_golden.py).

Conventions restated from the reference:
  * k-space arrays are complex (NX, NY, NZ//2+1) with the Ooura sign: the
    forward transform is exp(+i k.x) and unnormalised, the inverse carries 1/N
    (fft_wrapper.h:432-631, fftsg3d.c:108-131).  In numpy terms
    A2a_k(a) = conj(rfftn(a)) and A_k2a(A) = irfftn(conj(A)).
  * integer wavenumbers KX = i>NX/2 ? i-NX : i, KY likewise, KZ = k
    (fft_wrapper.h:687-699); K2 and IK2 (0 at k=0) as in Init_K
    (fft_wrapper.cxx:29-62).
  * 2/3 rule keeps |kx|<TRN_X, |ky|<TRN_Y, kz<TRN_Z, TRN=(N+2)/3
    (fft_wrapper.h:723-766, input.cxx:297).
"""
from __future__ import annotations

import math

import numpy as np

KT_SNAP_V = 1.439  # input.cxx:263
KT_SNAP_O = 1.22   # input.cxx:265


class Params:
    """Derived parameters, restating Set_global_parameters (input.cxx:274-431)
    and the A/A_XI/SIGMA reads of Gourmet_file_io (input.cxx:1347-1353)."""

    def __init__(self, cfg: dict):
        self.eq = cfg.get("eq", "Navier_Stokes")
        self.N = [1 << int(p) for p in cfg["np_xyz"]]
        self.NX, self.NY, self.NZ = self.N
        self.DX = float(cfg.get("dx", 1.0))
        self.RHO = float(cfg.get("rho", 1.0))
        self.ETA = float(cfg.get("eta", 1.0))
        self.kBT = float(cfg.get("kbt", 0.0))
        self.alpha_v = float(cfg.get("alpha_v", 1.0))
        self.alpha_o = float(cfg.get("alpha_o", 1.0))
        self.DT = float(cfg.get("dt", 0.01))
        self.A = float(cfg.get("a", 5.0))
        self.A_XI = float(cfg.get("a_xi", 2.0))
        self.RADIUS = self.A * self.DX
        self.XI = self.A_XI * self.DX
        self.HXI = 0.5 * self.XI
        self.SIGMA = 2.0 * self.RADIUS
        self.MASS_RATIO = float(cfg.get("mass_ratio", 1.0))
        self.G = float(cfg.get("gravity_g", 0.0))
        self.G_direction = {"-X": 0, "-Y": 1, "-Z": 2}[cfg.get("gravity_dir", "-Z")]
        self.EPSILON = float(cfg.get("epsilon", 1.0))
        self.ROTATION = 1 if cfg.get("rotation", "ON") == "ON" else 0
        # particles held at their positions and velocities, forces still
        # measured (the GPU library's resistance mode; no reference switch)
        self.frozen = bool(cfg.get("frozen", False))
        lj = cfg.get("lj_truncate", "ON")
        self.LJ_truncate = {"ON": 1, "OFF": 0, "NONE": -1}[lj]
        self.LJ_powers = {"12:6": 0, "24:12": 1, "36:18": 2}[cfg.get("lj_powers", "12:6")]
        # input.cxx:1461-1475
        if self.LJ_truncate > 0:
            self.A_R_cutoff = 2.0 ** (1.0 / (6.0 * (self.LJ_powers + 1)))
        elif self.LJ_truncate == 0:
            self.A_R_cutoff = min(min(self.N) * self.DX * 0.5 / self.SIGMA, 2.5)
        else:
            self.A_R_cutoff = 0.0
        self.LJ_dia = self.SIGMA
        self.fix_cell = [bool(f) for f in cfg.get("fix_cell", (False, False, False))]
        self.NU = self.ETA / self.RHO
        self.IRHO = 1.0 / self.RHO
        self.DX3 = self.DX ** 3
        self.RHO_particle = self.MASS_RATIO * self.RHO
        self.MASS = self.RHO_particle * 4.0 / 3.0 * math.pi * self.RADIUS ** 3
        self.IMASS = 1.0 / self.MASS
        self.MOI = 2.0 / 5.0 * self.MASS * self.RADIUS ** 2
        self.IMOI = 1.0 / self.MOI
        el = cfg.get("electrolyte", {})
        self.Dielectric_cst = float(el.get("dielectric", 1.0))
        self.Surface_charge = float(el.get("surface_charge", 0.0))
        self.Debye_length = float(el.get("debye", 1.0))
        self.Valency = [float(el.get("val_p", 1.0)), float(el.get("val_n", -1.0))]
        self.Onsager = [float(el.get("onsager_p", 1.0)), float(el.get("onsager_n", 1.0))]
        self.E_ext = [float(e) for e in el.get("efield", (0.0, 0.0, 0.0))]
        self.Elementary_charge = 1.0  # input.cxx:247
        self.TRN = [(n + 2) // 3 for n in self.N]
        self.L = [n * self.DX for n in self.N]
        self.WAVE = [2.0 * math.pi / l for l in self.L]


def nint(a):
    """Nint (macro.h:38-46): round half away from zero."""
    return np.where(a >= 0.0, np.floor(a + 0.5), -np.floor(-a + 0.5))


class Spectral:
    """FFT and k-space tables (fft_wrapper.cxx:29-62, fft_wrapper.h:432-766)."""

    def __init__(self, P: Params):
        self.P = P
        NX, NY, NZ = P.N
        i = np.arange(NX)
        j = np.arange(NY)
        k = np.arange(NZ // 2 + 1)
        self.KX = np.where(i > NX // 2, i - NX, i)[:, None, None]
        self.KY = np.where(j > NY // 2, j - NY, j)[None, :, None]
        self.KZ = k[None, None, :]
        self.kx = self.KX * P.WAVE[0]
        self.ky = self.KY * P.WAVE[1]
        self.kz = self.KZ * P.WAVE[2]
        self.K2 = self.kx ** 2 + self.ky ** 2 + self.kz ** 2
        with np.errstate(divide="ignore"):
            self.IK2 = np.where(self.K2 > 0, 1.0 / np.where(self.K2 > 0, self.K2, 1.0), 0.0)
        tx, ty, tz = P.TRN
        self.keep = (np.abs(self.KX) < tx) & (np.abs(self.KY) < ty) & (self.KZ < tz)

    def fwd(self, a):
        """A2a_k (fft_wrapper.h:432-527)."""
        return np.conj(np.fft.rfftn(a))

    def inv(self, A):
        """A_k2a (fft_wrapper.h:534-631)."""
        return np.fft.irfftn(np.conj(A), s=self.P.N, axes=(0, 1, 2))

    def inv_ooura(self, A):
        """A_k2a on a spectrum that need not be Hermitian on the kz=0 and
        kz=NZ/2 planes: rdft3dsort(isgn<0) (fftsg3d.c:645-668) reads only one
        half of each of these planes (and the real part at the self-conjugate
        points) and the inverse assumes the other half is its conjugate."""
        X = A.copy()
        n1, n2, m1 = X.shape
        n1h, n2h = n1 // 2, n2 // 2
        I, J = np.meshgrid(np.arange(n1), np.arange(n2), indexing="ij")
        selfc = ((I == 0) | (I == n1h)) & ((J == 0) | (J == n2h))
        for kz, hi in ((0, False), (m1 - 1, True)):
            P = X[:, :, kz]
            if hi:
                keep = (J > n2h) | (((J == 0) | (J == n2h)) & (I >= n1h))
            else:
                keep = ((J > 0) & (J < n2h)) | (((J == 0) | (J == n2h)) & (I <= n1h))
            Q = np.where(keep, P, np.conj(P[(-I) % n1, (-J) % n2]))
            X[:, :, kz] = np.where(selfc, Q.real + 0j, Q)
        return self.inv(X)

    def grad_k(self, A):
        """A_k2da_k (fft_wrapper.cxx:103-135): da = -i k a per component."""
        return np.stack([-1j * self.kx * A, -1j * self.ky * A, -1j * self.kz * A])

    def div_k(self, F):
        """U_k2divergence_k (fft_wrapper.cxx:649-677): -i k.F."""
        return -1j * (self.kx * F[0] + self.ky * F[1] + self.kz * F[2])

    def truncate(self, A):
        """Truncate_two_third_rule_ooura (fft_wrapper.h:723-766)."""
        return np.where(self.keep, A, 0.0)

    def zeta_k2u_k(self, zeta, uk_dc):
        """Zeta_k2u_k (fft_wrapper.cxx:408-511): reduced vorticity -> velocity.
        The third vorticity component is rebuilt from k.omega = 0 with the
        3-case component map, then u = -i k x omega / k^2 and u(k=0) = uk_dc."""
        kx, ky, kz = self.kx, self.ky, self.kz
        z0, z1 = zeta
        cx = self.KX != 0
        cy = (~cx) & (self.KY != 0)
        with np.errstate(divide="ignore", invalid="ignore"):
            w0 = np.where(cx, -(ky * z0 + kz * z1) / np.where(cx, kx, 1.0), np.where(cy, z1, z0))
            w1 = np.where(cx, z0, np.where(cy, -(kz / np.where(cy, ky, 1.0)) * z0, z1))
            w2 = np.where(cx, z1, np.where(cy, z0, 0.0))
        ik2 = self.IK2
        u0 = -1j * (ky * w2 - kz * w1) * ik2
        u1 = -1j * (kz * w0 - kx * w2) * ik2
        u2 = -1j * (kx * w1 - ky * w0) * ik2
        u = np.stack([u0, u1, u2])
        u[:, 0, 0, 0] = np.asarray(uk_dc, dtype=np.float64)
        return u

    def _select(self, w):
        """Component map of Omega_k2zeta_k (fft_wrapper.cxx:137-173) and
        U_k2zeta_k (:258-339): kx!=0 -> (w1,w2); ky!=0 -> (w2,w0); else (w0,w1)."""
        cx = self.KX != 0
        cy = (~cx) & (self.KY != 0)
        z0 = np.where(cx, w[1], np.where(cy, w[2], w[0]))
        z1 = np.where(cx, w[2], np.where(cy, w[0], w[1]))
        return np.stack([z0, z1])

    def omega_k2zeta_k(self, w):
        return self._select(w)

    def u_k2zeta_k(self, uk):
        """U_k2zeta_k (fft_wrapper.cxx:258-339): omega = -i k x u, reduced by
        the component map; uk_dc = Re u(k=0)."""
        kx, ky, kz = self.kx, self.ky, self.kz
        w0 = -1j * (ky * uk[2] - kz * uk[1])
        w1 = -1j * (kz * uk[0] - kx * uk[2])
        w2 = -1j * (kx * uk[1] - ky * uk[0])
        zeta = self._select(np.stack([w0, w1, w2]))
        uk_dc = np.array([uk[d][0, 0, 0].real for d in range(3)])
        return zeta, uk_dc

    def solenoidal_uk(self, uk):
        """Solenoidal_uk (operate_omega.cxx:186-219): u -= k (k.u)/k^2."""
        kx, ky, kz = self.kx, self.ky, self.kz
        d = self.IK2 * (uk[0] * kx + uk[1] * ky + uk[2] * kz)
        return np.stack([uk[0] - d * kx, uk[1] - d * ky, uk[2] - d * kz])

    def solenoidal_u(self, f):
        """Solenoidal_u (operate_omega.h:96-103): FFT, 2/3 truncation,
        Solenoidal_uk, inverse FFT."""
        fk = np.stack([self.truncate(self.fwd(f[d])) for d in range(3)])
        fk = self.solenoidal_uk(fk)
        return np.stack([self.inv(fk[d]) for d in range(3)])

    def advection_k(self, u):
        """U2advection_k (operate_omega.cxx:14-100): the 5 real-space products,
        their forward FFTs, the k-space curl-divergence combine into Omega and
        the reduction Omega_k2zeta_k."""
        u1, u2, u3 = u
        a23 = self.fwd(u2 * u3)
        a31 = self.fwd(u3 * u1)
        a12 = self.fwd(u1 * u2)
        b22_33 = self.fwd((u2 - u3) * (u2 + u3))
        b33_11 = self.fwd((u3 - u1) * (u3 + u1))
        b11_22 = -b33_11 - b22_33
        k1, k2, k3 = self.kx, self.ky, self.kz
        k1k2, k2k3, k3k1 = k1 * k2, k2 * k3, k3 * k1
        w0 = -(k2k3 * b22_33 + (k3 - k2) * (k3 + k2) * a23 + k3k1 * a12 - k1k2 * a31)
        w1 = -(k3k1 * b33_11 + (k1 - k3) * (k1 + k3) * a31 + k1k2 * a23 - k2k3 * a12)
        w2 = -(k1k2 * b11_22 + (k2 - k1) * (k2 + k1) * a12 + k2k3 * a31 - k3k1 * a23)
        return self.omega_k2zeta_k(np.stack([w0, w1, w2]))

    def zeta_k2u(self, zeta, uk_dc):
        """Zeta_k2u (operate_omega.h:124-128)."""
        uk = self.zeta_k2u_k(zeta, uk_dc)
        return np.stack([self.inv(uk[d]) for d in range(3)])

    def u2zeta_k(self, u):
        """U2zeta_k (operate_omega.h:186-189)."""
        uk = np.stack([self.fwd(u[d]) for d in range(3)])
        return self.u_k2zeta_k(uk)


class MT19937Gauss:
    """Thermostat normals: the reference MT19937 stream seeded by
    init_genrand(0) (sp_3d_ns.cxx:477, fluct.h:34-46), genrand_real3
    (mt19937ar.c:168-172) and polar Box-Muller Gauss2 (fluct.h:48-60).
    numpy's legacy RandomState seeding is the same init_genrand; its
    random_raw yields genrand_int32."""

    def __init__(self, seed: int = 0):
        self.bg = np.random.RandomState(seed)._bit_generator
        self.buf = np.empty(0, dtype=np.uint64)

    def _u32(self):
        if self.buf.size == 0:
            self.buf = self.bg.random_raw(4096)
        v = int(self.buf[0])
        self.buf = self.buf[1:]
        return v

    def real3(self):
        return (float(self._u32()) + 0.5) * (1.0 / 4294967296.0)

    def gauss2(self):
        while True:
            x1 = 2.0 * self.real3() - 1.0
            x2 = 2.0 * self.real3() - 1.0
            rsq = x1 * x1 + x2 * x2
            if not (rsq >= 1.0 or rsq == 0.0):
                break
        f = math.sqrt(-2.0 * math.log(rsq) / rsq)
        return f * x1, f * x2

    def normals6(self, n_particles: int) -> np.ndarray:
        out = np.empty((n_particles, 6))
        for n in range(n_particles):
            for c in range(3):
                out[n, 2 * c], out[n, 2 * c + 1] = self.gauss2()
        return out


def sekibun_cells(P: Params) -> np.ndarray:
    """Particle_domain (profile.cxx:25-74): integer offsets within
    RADIUS + HXI + 1.7321 DX of the cell origin, scanned i, j, k from -nh."""
    nh = int(P.A) + int(P.A_XI) + 2
    max_r = P.RADIUS + P.HXI + 1.7321 * P.DX
    r = np.arange(-nh, nh + 1)
    I, J, K = np.meshgrid(r, r, r, indexing="ij")
    d = np.sqrt((I * P.DX) ** 2 + (J * P.DX) ** 2 + (K * P.DX) ** 2)
    m = d < max_r
    return np.stack([I[m], J[m], K[m]], axis=1).astype(np.int64)


def phi_profile(x, radius, P: Params):
    """Phi (profile.h:46-49) with H(x) = exp(-(DX/x)^2) for x > 0 (profile.h:29-32)."""
    x = np.asarray(x, dtype=np.float64)

    def H(y):
        with np.errstate(divide="ignore", over="ignore"):
            return np.where(y > 0, np.exp(-np.square(P.DX / np.where(y > 0, y, 1.0))), 0.0)

    h1 = H(radius + P.HXI - x)
    return h1 / (h1 + H(x - radius + P.HXI))


class Particles:
    """Particle SoA (the subset of variable.h:27-75 the SPM step touches)."""

    FIELDS = ["x", "x_previous", "x_nopbc", "v", "v_old", "omega", "omega_old", "f_hydro",
              "f_hydro_previous", "torque_hydro", "torque_hydro_previous", "fr", "fr_previous"]

    def __init__(self, n: int):
        for f in self.FIELDS:
            setattr(self, f, np.zeros((n, 3)))
        self.q = np.tile([1.0, 0.0, 0.0, 0.0], (n, 1))
        self.q_old = self.q.copy()
        self.n = n


def qprod(a, b, alpha=1.0):
    """qtn_prod (quaternion.h:173-186) on (..., 4) arrays (s, v0, v1, v2)."""
    s = alpha * (a[..., 0] * b[..., 0] - (a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2] + a[..., 3] * b[..., 3]))
    v0 = alpha * (a[..., 0] * b[..., 1] + b[..., 0] * a[..., 1] + a[..., 2] * b[..., 3] - a[..., 3] * b[..., 2])
    v1 = alpha * (a[..., 0] * b[..., 2] + b[..., 0] * a[..., 2] + a[..., 3] * b[..., 1] - a[..., 1] * b[..., 3])
    v2 = alpha * (a[..., 0] * b[..., 3] + b[..., 0] * a[..., 3] + a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1])
    return np.stack([s, v0, v1, v2], axis=-1)


def qconj(q):
    return q * np.array([1.0, -1.0, -1.0, -1.0])


def vec_q(v):
    return np.concatenate([np.zeros(v.shape[:-1] + (1,)), v], axis=-1)


def space2body(v, q):
    """rigid_body_rotation SPACE2BODY (rigid_body.cxx:10-33): conj(q).(0,v).q"""
    qx = qprod(vec_q(v), q)
    return qprod(qconj(q), qx)[..., 1:]


def qnormalize(q):
    """qtn_normalize (quaternion.h:237-245)."""
    n = np.sqrt(np.sum(q * q, axis=-1, keepdims=True))
    return q * (1.0 / n)


class SpmOracle:
    """One SPM box in the Navier_Stokes mode: state (zeta, uk_dc, particles)
    and the step Time_evolution_hydro (sp_3d_ns.cxx:61-212)."""

    def __init__(self, cfg: dict):
        self.P = P = Params(cfg)
        self.S = Spectral(P)
        self.cells = sekibun_cells(P)
        parts = cfg["particles"]
        self.p = Particles(len(parts))
        for n, pd in enumerate(parts):
            # positions and orientations are read; velocities and angular
            # velocities are reset to 0 afterwards (init_particle.cxx:357-370)
            self.p.x[n] = pd["x"]
            q = np.asarray(pd.get("q", (1.0, 0.0, 0.0, 0.0)), dtype=np.float64)
            self.p.q[n] = qnormalize(q)  # init_particle.cxx:281-286 (user_dir)
        self.p.q_old[:] = self.p.q
        self.p.x_nopbc[:] = self.p.x
        self.ts = 0
        self.time = 0.0
        self.rng = MT19937Gauss(0)
        self.noise_override = None
        self.zeta, self.uk_dc = self._initial_state()

    # ---- particle <-> grid stencils (make_phi.h:102-160, make_phi.cxx:221-298, md_force.cxx:263-389)
    def stencil(self, x):
        """For particle centres x (Np,3): grid index (Np,S,3), the vector r
        from the centre to the point (Np,S,3) and the min-image distance (Np,S).
        Particle_cell (make_phi.h:102-130), Relative_coord (:143-160),
        Distance (interaction.h:110-133)."""
        P = self.P
        N = np.array(P.N)
        L = np.array(P.L)
        xi = x / P.DX
        x_int = xi.astype(np.int64)  # (int) truncation, x >= 0
        residue = (xi - x_int) * P.DX
        cells = self.cells[None, :, :]
        r_mesh = (x_int[:, None, :] + cells + N) % N
        r = cells * P.DX - residue[:, None, :]
        d = r_mesh * P.DX - x[:, None, :]
        d = d - nint(d / L) * L
        dist = np.sqrt(np.sum(d * d, axis=-1))
        return r_mesh, r, dist

    def phi_up(self, x, v, omega):
        """Make_phi_u_particle with the phi>1 clamp (make_phi.cxx:221-298)."""
        P = self.P
        r_mesh, r, dist = self.stencil(x)
        ph = phi_profile(dist, P.RADIUS, P)
        vr = np.cross(omega[:, None, :], r) if P.ROTATION else np.zeros_like(r)
        vel = (v[:, None, :] + vr) * ph[..., None]
        flat = (r_mesh[..., 0] * P.NY + r_mesh[..., 1]) * P.NZ + r_mesh[..., 2]
        n = P.NX * P.NY * P.NZ
        phi = np.bincount(flat.ravel(), weights=ph.ravel(), minlength=n)
        up = np.stack([np.bincount(flat.ravel(), weights=vel[..., d].ravel(), minlength=n) for d in range(3)])
        over = phi > 1.0
        inv = np.where(over, 1.0 / np.where(over, phi, 1.0), 1.0)
        up = up * inv
        phi = np.where(over, 1.0, phi)
        return phi.reshape(P.N), up.reshape((3,) + tuple(P.N))

    def hydro_force(self, u):
        """Calc_f_hydro_correct_precision (md_force.cxx:263-389), DBG_MASS_GRID off."""
        P = self.P
        p = self.p
        r_mesh, r, dist = self.stencil(p.x)
        ph = phi_profile(dist, P.RADIUS, P)
        vr = np.cross(p.omega[:, None, :], r) if P.ROTATION else np.zeros_like(r)
        ug = u[:, r_mesh[..., 0], r_mesh[..., 1], r_mesh[..., 2]]  # (3,Np,S)
        fp = ((p.v[:, None, :] + vr) - np.moveaxis(ug, 0, -1)) * ph[..., None]
        force = fp.sum(axis=1)
        torque = np.cross(r, fp).sum(axis=1)
        c = -P.DX3 * P.RHO / P.DT
        p.f_hydro[:] = c * force
        if P.ROTATION:
            p.torque_hydro[:] = c * torque

    # ---- particle forces (md_force.cxx:23-191, interaction.h:110-181)
    def lj_force(self):
        """Calc_f_Lennard_Jones_shear_cap_primitive_lnk (md_force.cxx:23-134),
        cap = DBL_MAX, including the cell-list multiplicity: a pair is met
        once per neighbour offset (-1..1 per axis) that wraps onto the
        partner's cell, so with fewer than 3 cells on an axis it is counted
        more than once (lc=NX/16 cells of 16 DX)."""
        P = self.P
        p = self.p
        n = p.n
        if n < 2 or P.LJ_truncate < 0:
            return
        lc = np.array([P.NX // 16, P.NY // 16, P.NZ // 16])
        mc = (p.x / (16 * P.DX)).astype(np.int64)
        L = np.array(P.L)
        cutoff = P.A_R_cutoff * P.LJ_dia
        ii, jj = np.triu_indices(n, 1)
        a, b = jj, ii  # i > j in the reference loop: i=a (larger), j=b
        mult = np.ones(len(a), dtype=np.int64)
        for d in range(3):
            cnt = np.zeros(len(a), dtype=np.int64)
            for o in (-1, 0, 1):
                c = mc[a, d] + o
                c = np.where(c < 0, lc[d] - 1, np.where(c > lc[d] - 1, 0, c))
                cnt += (c == mc[b, d])
            mult *= cnt
        x12 = p.x[b] - p.x[a]
        x12 = x12 - nint(x12 / L) * L
        r = np.sqrt(np.sum(x12 * x12, axis=1))
        m = (r < cutoff) & (mult > 0)
        ps = 6 * (P.LJ_powers + 1)
        coeff = 24.0 * (P.LJ_powers + 1) * P.EPSILON
        rr = r[m]
        dmy = (P.LJ_dia / rr) ** ps
        f = coeff / rr ** 2 * (2.0 * dmy * dmy - dmy)
        contrib = (f[:, None] * -x12[m]) * mult[m][:, None]
        np.add.at(p.fr, a[m], contrib)
        np.add.at(p.fr, b[m], -contrib)

    def force(self):
        """Force (particle_solver.h:97-109): LJ and gravity (md_force.cxx:181-191)."""
        P = self.P
        if P.LJ_truncate >= 0:
            self.lj_force()
        if P.G != 0.0:
            g = P.G * P.RHO * 4.0 / 3.0 * math.pi * P.RADIUS ** 2 * P.RADIUS
            self.p.fr[:, P.G_direction] -= g * (P.MASS_RATIO - 1.0)

    def reset_forces(self):
        """reset_Forces (particle_solver.cxx:11-34)."""
        p = self.p
        p.fr_previous[:] = p.fr
        p.fr[:] = 0
        p.f_hydro_previous[:] = p.f_hydro
        p.f_hydro[:] = 0
        p.torque_hydro_previous[:] = p.torque_hydro
        p.torque_hydro[:] = 0

    # ---- integrators (particle_solver.cxx:36-147, 247-289; particle_rotation_solver.h:15-39)
    def position_update(self):
        P = self.P
        p = self.p
        p.x_previous[:] = p.x
        if self.ts == 0:
            dx = P.DT * p.v
        else:
            dx = 0.5 * P.DT * (3.0 * p.v - p.v_old)
        p.x_nopbc += dx
        p.x += dx
        L = np.array(P.L)
        p.x[:] = np.fmod(p.x + L, L)  # PBC (periodic_boundary.h:9-15)
        if P.ROTATION:
            if self.ts == 0:
                p.q_old[:] = p.q
                dq = qprod(vec_q(p.omega), p.q, 0.5)  # qdot SPACE_FRAME (rigid_body.cxx:50-63)
                p.q[:] = qnormalize(p.q + dq * P.DT)
            else:
                wb = space2body(p.omega, p.q)
                wb_old = space2body(p.omega_old, p.q_old)
                wb = 3.0 * wb - wb_old
                p.q_old[:] = p.q
                dq = qprod(p.q, vec_q(wb), 0.5)  # qdot BODY_FRAME
                p.q[:] = qnormalize(p.q + dq * (0.5 * P.DT))

    def velocity_update(self):
        P = self.P
        p = self.p
        self.force()
        p.v_old[:] = p.v
        p.omega_old[:] = p.omega
        if self.ts == 0:
            p.v += P.DT * P.IMASS * (p.f_hydro + p.fr)
            p.omega += P.DT * P.IMOI * p.torque_hydro
        else:
            h = 0.5 * P.DT
            p.v += h * P.IMASS * (2.0 * p.f_hydro + p.fr + p.fr_previous)
            p.omega += h * P.IMOI * 2.0 * p.torque_hydro
        self.reset_forces()

    def noise_factors(self):
        """Add_random_force_thermostat amplitudes (fluct.cxx:10-19)."""
        P = self.P
        zeta_drag = 6.0 * math.pi * P.ETA * P.RADIUS
        zeta_drag_rot = 8.0 * math.pi * P.ETA * P.RADIUS ** 3
        nv = KT_SNAP_V * math.sqrt(zeta_drag * P.DT * P.kBT * P.alpha_v)
        no = KT_SNAP_O * math.sqrt(zeta_drag_rot * P.DT * P.kBT * P.alpha_o)
        return nv, no

    def thermostat(self):
        """Add_random_force_thermostat (fluct.cxx:10-36), spherical particles."""
        P = self.P
        p = self.p
        g = self.rng.normals6(p.n)
        nv, no = self.noise_factors()
        p.v += g[:, 0:3] * nv * P.IMASS
        if P.ROTATION:
            p.omega += g[:, 3:6] * no * P.IMOI

    # ---- the step
    def _initial_state(self):
        """Initial state of main() (sp_3d_ns.cxx:508-524): Init_zeta_k gives
        zeta = 0 (init_fluid.cxx:10-26), then one rigidity projection, then
        uk_dc = 0."""
        S = self.S
        P = self.P
        shape_k = (2, P.NX, P.NY, P.NZ // 2 + 1)
        zeta = np.zeros(shape_k, dtype=np.complex128)
        uk_dc = np.zeros(3)
        if self.p.n > 0:
            phi, up = self.phi_up(self.p.x, self.p.v, self.p.omega)
            u = S.zeta_k2u(zeta, uk_dc)
            f = S.solenoidal_u(up - phi * u)
            zeta, uk_dc = S.u2zeta_k(u + f)
        return zeta, np.zeros(3)

    def step(self):
        """Time_evolution_hydro (sp_3d_ns.cxx:61-212), Navier_Stokes branch."""
        P = self.P
        S = self.S
        # NS_solver_slavedEuler (fluid_solver.cxx:328-354)
        zeta = np.stack([S.truncate(self.zeta[d]) for d in range(2)])
        u = S.zeta_k2u(zeta, self.uk_dc)
        fns = S.advection_k(u)
        dmy = np.exp(-P.NU * P.DT * S.K2) - 1.0
        upd = zeta + dmy * (zeta - (1.0 / P.NU) * S.IK2 * fns)
        zeta = np.where(S.keep, upd, zeta)
        # FIX_CELL (sp_3d_ns.cxx:67-73)
        for d in range(3):
            if P.fix_cell[d]:
                self.uk_dc[d] = 0.0
        zeta = np.stack([S.truncate(zeta[d]) for d in range(2)])
        u = S.zeta_k2u(zeta, self.uk_dc)
        if self.p.n > 0:
            if P.frozen:
                self.hydro_force(u)
                self.force()
                self.reset_forces()
            else:
                self.position_update()
                self.hydro_force(u)
                self.velocity_update()
                if P.kBT > 0.0:
                    self.thermostat()
            phi, up = self.phi_up(self.p.x, self.p.v, self.p.omega)
            f = S.solenoidal_u(up - phi * u)
            u = u + f
        self.u = u
        self.zeta, self.uk_dc = S.u2zeta_k(u)
        self.ts += 1
        self.time += P.DT

    def run(self, n: int):
        for _ in range(n):
            self.step()

    # ---- accessors in the reference's padded Ooura layout
    @staticmethod
    def to_ooura(A: np.ndarray) -> np.ndarray:
        """complex (NX,NY,NZ/2+1) -> float (NX,NY,NZ_) interleaved (re,im)."""
        out = np.empty(A.shape[:-1] + (2 * A.shape[-1],))
        out[..., 0::2] = A.real
        out[..., 1::2] = A.imag
        return out

    @staticmethod
    def from_ooura(a: np.ndarray) -> np.ndarray:
        return a[..., 0::2] + 1j * a[..., 1::2]


def dphi_compact_sin(x, P: Params):
    """DPhi_compact_sin (profile.h:168-181) with radius RADIUS and xi XI."""
    hxi = 0.5 * P.XI
    d = P.RADIUS - np.asarray(x, dtype=np.float64)
    return np.where(np.abs(d) < hxi, math.pi * 0.5 * (1.0 / P.XI) * np.cos(math.pi * d * (1.0 / P.XI)), 0.0)


class ElectrolyteOracle(SpmOracle):
    """The Electrolyte branch (salt, two ion species, INIT_profile Uniform) of
    Time_evolution_hydro (sp_3d_ns.cxx:61-212) with NSsolute_solver_Euler
    (fluid_solver.cxx:306-326)."""

    def __init__(self, cfg: dict):
        super().__init__(cfg)
        self.init_rho_ion()

    # ---- particle-grid helpers
    def _scatter(self, values_per_point):
        P = self.P
        r_mesh, r, dist = self.stencil(self.p.x)
        flat = (r_mesh[..., 0] * P.NY + r_mesh[..., 1]) * P.NZ + r_mesh[..., 2]
        n = P.NX * P.NY * P.NZ
        return np.bincount(flat.ravel(), weights=values_per_point(r, dist).ravel(), minlength=n).reshape(P.N)

    def phi_particle(self):
        """Make_phi_particle (make_phi.cxx:388-400): scatter without the clamp."""
        return self._scatter(lambda r, dist: phi_profile(dist, self.P.RADIUS, self.P))

    def phi_qq(self):
        """Make_phi_qq_particle (operate_electrolyte.cxx:179-242): phi and the
        surface charge Z_e DPhi_compact_sin, rescaled so that its absolute
        integral is sum |Z_e|."""
        P = self.P
        phi = self.phi_particle()
        ze = P.Surface_charge * P.Elementary_charge
        surf = self._scatter(lambda r, dist: ze * dphi_compact_sin(dist, P))
        total = abs(ze) * self.p.n
        surf = surf * (total / (np.sum(np.abs(surf)) * P.DX3))
        return phi, surf

    def surface_normal(self):
        """Make_surface_normal (make_phi.cxx:17-58): sum of r/|r| over
        interface points (| |r| - RADIUS | < HXI) of every particle."""
        P = self.P
        r_mesh, r, dist = self.stencil(self.p.x)
        rr = np.sqrt(np.sum(r * r, axis=-1))
        m = np.abs(rr - P.RADIUS) < P.HXI
        flat = ((r_mesh[..., 0] * P.NY + r_mesh[..., 1]) * P.NZ + r_mesh[..., 2])[m]
        n = P.NX * P.NY * P.NZ
        out = np.stack([np.bincount(flat, weights=(r[..., d] / np.where(m, rr, 1.0))[m], minlength=n)
                        for d in range(3)])
        return out.reshape((3,) + tuple(P.N))

    def charge_field(self):
        """Conc_k2charge_field (operate_electrolyte.cxx:45-74)."""
        P = self.P
        phi, surf = self.phi_qq()
        charge = surf.copy()
        for n in range(2):
            c = self.S.inv(self.conc_k[n])
            charge += P.Valency[n] * P.Elementary_charge * c * (1.0 - phi)
        return charge

    def count_solute(self, conc_x, phi):
        """Count_single_solute (solute_rhs.cxx:130-148)."""
        return float(np.sum((1.0 - phi) * conc_x) * self.P.DX3)

    def init_rho_ion(self):
        """Init_rho_ion (operate_electrolyte.cxx:692-815), salt, Uniform:
        Set_uniform_ion_charge_density_salt (:516-575) then Count_solute_each
        (solute_rhs.h:143-157)."""
        P = self.P
        phi = self.phi_particle()
        Z, Np = P.Surface_charge, self.p.n
        pos = abs(Z * Np / P.Valency[0]) if Z < 0 else 0.0
        neg = abs(Z * Np / P.Valency[1]) if Z > 0 else 0.0
        vol = float(np.sum(1.0 - phi))
        rho_inf = P.kBT * P.Dielectric_cst / (P.Elementary_charge * P.Debye_length) ** 2
        v0, v1 = P.Valency
        c0 = pos / (vol * P.DX3) + rho_inf / (v0 * (v0 - v1))
        c1 = neg / (vol * P.DX3) - rho_inf / (v1 * (v0 - v1))
        conc = [np.full(P.N, c0), np.full(P.N, c1)]
        self.conc_k = np.stack([self.S.fwd(c) for c in conc])
        phi = self.phi_particle()
        self.total_solute = [self.count_solute(self.S.inv(self.conc_k[n]), phi) for n in range(2)]

    def set_efield(self, e):
        self.P.E_ext = [float(x) for x in e]

    # ---- the step
    def step(self):
        P = self.P
        S = self.S
        N = P.NX * P.NY * P.NZ
        ext_on = any(e != 0.0 for e in P.E_ext)
        # Rhs_NS_Nernst_Planck (fluid_solver.cxx:243-280): potential gradient
        charge = self.charge_field()
        psi = S.truncate(S.fwd(charge) * S.IK2 * (1.0 / P.Dielectric_cst))
        gk = S.grad_k(psi)
        for d in range(3):  # Add_constant_field_k (fluid_solver.cxx:228-241)
            gk[d][0, 0, 0] -= P.E_ext[d] * float(N)
        grad = np.stack([S.inv(gk[d]) for d in range(3)])
        # Rhs_NS_solute (fluid_solver.cxx:181-227)
        zeta = np.stack([S.truncate(self.zeta[d]) for d in range(2)])
        u = S.zeta_k2u(zeta, self.uk_dc)
        normal = self.surface_normal()
        n2 = np.sum(normal * normal, axis=0)
        rhs_sol = []
        for n in range(2):
            self.conc_k[n] = S.truncate(self.conc_k[n])
            L = P.Onsager[n]
            flux = np.stack([S.inv(g) for g in S.grad_k(P.kBT * L * self.conc_k[n])])  # Diffusion_flux_single
            c = S.inv(self.conc_k[n])
            flux = flux + c * (L * (grad * (P.Valency[n] * P.Elementary_charge)))  # Solute_solver_rhs_nonlinear_x_single
            # Solute_impermeability (solute_rhs.cxx:42-97): project out the normal part
            dn = np.where(n2 > 0, np.sum(flux * normal, axis=0) / np.where(n2 > 0, n2, 1.0), 0.0)
            flux = flux - normal * dn
            flux = flux + c * -u  # Add_advection_flux
            fk = np.stack([S.fwd(flux[d]) for d in range(3)])
            rhs_sol.append(S.div_k(fk))
        rhs_ns = S.advection_k(u)
        rhs_ns = np.where(S.keep, rhs_ns - P.NU * S.K2 * zeta, rhs_ns)  # Add_zeta_viscous_term
        # Field_solver_Euler on the retained modes
        zeta = np.where(S.keep, zeta + P.DT * rhs_ns, zeta)
        for n in range(2):
            self.conc_k[n] = np.where(S.keep, self.conc_k[n] + P.DT * rhs_sol[n], self.conc_k[n])
        for d in range(3):
            if P.fix_cell[d]:
                self.uk_dc[d] = 0.0
        zeta = np.stack([S.truncate(zeta[d]) for d in range(2)])
        u = S.zeta_k2u(zeta, self.uk_dc)
        if self.p.n > 0:
            self.position_update()
        # Rescale_solute (solute_rhs.cxx:99-128)
        phi = self.phi_particle()
        for n in range(2):
            fac = self.total_solute[n] / self.count_solute(S.inv(self.conc_k[n]), phi)
            self.conc_k[n] = self.conc_k[n] * fac
        # Make_Coulomb_force_x_on_fluid (operate_electrolyte.cxx:90-177): no truncation
        charge = self.charge_field()
        gk = S.grad_k(S.fwd(charge) * S.IK2 * (1.0 / P.Dielectric_cst))
        grad = np.stack([S.inv_ooura(gk[d]) for d in range(3)])
        f = np.stack([charge * (-grad[d] + (P.E_ext[d] if ext_on else 0.0)) for d in range(3)])
        u = u + f * (P.DT * P.IRHO)
        u = S.solenoidal_u(u)
        if self.p.n > 0:
            self.hydro_force(u)
            self.velocity_update()
            phi, up = self.phi_up(self.p.x, self.p.v, self.p.omega)
            f = S.solenoidal_u(up - phi * u)
            u = u + f
        self.u = u
        self.zeta, self.uk_dc = S.u2zeta_k(u)
        self.ts += 1
        self.time += P.DT
