/*
 * kapsel_ref_shim.cxx -- the GPU library behind KAPSEL's own function names.
 *
 * This translation unit is compiled INTO a KAPSEL build (against the
 * reference's headers: variable.h, input.h, ... via sp_3d_ns.h) and linked
 * with libkapsel_gpu.so.  It defines, with the reference's exact signatures,
 *
 *   whole step (KAPSEL_SHIM_STEP):
 *     Time_evolution_hydro       sp_3d_ns.cxx:61-212  (Navier_Stokes, Electrolyte)
 *     Time_evolution_hydro_OBL   sp_3d_ns.cxx:214-390 (Lees-Edwards)
 *   routines (KAPSEL_SHIM_ROUTINES):
 *     NS_solver_slavedEuler                        fluid_solver.h:80
 *     Make_phi_particle, Make_phi_u_particle       make_phi.h:51,70
 *     Calc_f_hydro_correct_precision               md_force.h:60
 *     Calc_f_Lennard_Jones_shear_cap_primitive_lnk md_force.h:67 (what the
 *                                                   inline Calc_f_Lennard_Jones,
 *                                                   md_force.h:75, calls)
 *     MD_solver_position_Euler / _AB2              particle_solver.h:38,55
 *     MD_solver_velocity_Euler / _AB2_hydro        particle_solver.h:62,71
 *     NSsolute_solver_Euler                        fluid_solver.h:116 (with
 *                                                   the solute_rhs.cxx routines
 *                                                   it calls)
 *     Rescale_solute                               solute_rhs.h:107
 *     Make_Coulomb_force_x_on_fluid                operate_electrolyte.h:78
 *
 * so that the reference's main loop (sp_3d_ns.cxx:442-657) runs unchanged on
 * the GPU once the reference's own definitions of these names are removed
 * from the link or made weak (objcopy --weaken-symbol=<name> on the object
 * that defines it).  Both groups are on by default; a build that wants only
 * one defines the other's macro to 0.
 *
 * Handle registry.  The reference keeps its state in host arrays that its
 * main allocates once (zeta, uk_dc, the Particle array, the global field
 * pointers).  The shim keys GPU contexts by those host base pointers:
 *   - the whole-step shims: one context per zeta[0] (the run's state lives
 *     on the device between steps; the first call uploads zeta, uk_dc, the
 *     particles (and the ion concentrations) and the step counter);
 *   - the routine shims: one work context per process (and a second one,
 *     of the Electrolyte kind, for the Electrolyte routines), whose particle
 *     and field state every call uploads from the arguments and whose
 *     results every call writes back (the routines have no state of their
 *     own).
 * Host mirrors of the whole-step state: the particles after every step; zeta,
 * uk_dc (and the concentrations) after the steps whose state the main loop
 * reads -- ts+1 a multiple of GTS (Output_udf / Output_avs at the top of the
 * next iteration) and ts == MSTEP (Save_Restart_udf) -- or after every step
 * with KAPSEL_SHIM_MIRROR=every in the environment.  If the host changes the
 * state between steps (a particle position differs from the last mirror, or
 * jikan.ts from the device counter, as after Force_restore_parameters), the
 * next call uploads it again; kapsel_shim_invalidate(zeta) forces that.
 *
 * Errors: a non-zero status of the library is reported on stderr and ends the
 * run through the reference's exit_job (macro.h:194), as the reference does
 * on invalid state.  Configurations the GPU library does not model (several
 * particle species, chains, rigid bodies, Janus particles, fixed particles,
 * the zig-zag Shear_Navier_Stokes branch) stop the same way.
 *
 * Precision: FP64 (KAPSEL_FP64) unless KAPSEL_SHIM_PRECISION=mixed.
 */
#include "sp_3d_ns.h"

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "kapsel_gpu.h"

#ifndef KAPSEL_SHIM_STEP
#define KAPSEL_SHIM_STEP 1
#endif
#ifndef KAPSEL_SHIM_ROUTINES
#define KAPSEL_SHIM_ROUTINES 1
#endif

// Time_evolution_hydro_OBL's Lees-Edwards state (sp_3d_ns.cxx, input.cxx:271)
extern double degree_oblique;
// the ion concentrations of the Electrolyte branch (solute_rhs.cxx:16)
extern double **Concentration;

namespace {

void shim_fail(const char *what, int rc) {
  fprintf(stderr, "kapsel shim: %s failed: %s (%d)\n", what, rc ? kapsel_gpu_strerror(rc) : "unsupported", rc);
  exit_job(EXIT_FAILURE);
}

void check(int rc, const char *what) {
  if (rc) shim_fail(what, rc);
}

int ilog2i(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

int shim_precision() {
  const char *e = getenv("KAPSEL_SHIM_PRECISION");
  return e && strcmp(e, "mixed") == 0 ? KAPSEL_MIXED : KAPSEL_FP64;
}

// The GPU library models one species of free spherical particles.
void check_supported() {
  if (SW_EQ == Shear_Navier_Stokes) shim_fail("Shear_Navier_Stokes (zig-zag) branch", 0);
  if (Particle_Number > 0) {
    if (Component_Number != 1) shim_fail("more than one particle species", 0);
    if (SW_PT != spherical_particle) shim_fail("chains / rigid bodies", 0);
    if (SW_JANUS || SW_JANUS_MOTOR || SW_JANUS_SLIP) shim_fail("Janus particles", 0);
    if (Fixed_particle) shim_fail("fixed particles", 0);
    if (PINNING) shim_fail("pinned particles", 0);
  }
  if (DBG_MASS_GRID) shim_fail("DBG_MASS_GRID", 0);
  if (SW_EQ == Electrolyte) {
    if (N_spec != 2) shim_fail("an ion model other than two species (salt)", 0);
    if (External_field && AC) shim_fail("an AC external electric field", 0);
  }
}

// kapsel_params from the reference's globals (set by Gourmet_file_io and
// Set_global_parameters, input.cxx:274-1818).
kapsel_params params_from_globals() {
  check_supported();
  kapsel_params p;
  kapsel_params_default(&p);
  p.np_xyz[0] = ilog2i(NX);
  p.np_xyz[1] = ilog2i(NY);
  p.np_xyz[2] = ilog2i(NZ);
  p.eq = SW_EQ == Navier_Stokes ? KAPSEL_EQ_NAVIER_STOKES
         : SW_EQ == Shear_Navier_Stokes_Lees_Edwards ? KAPSEL_EQ_SHEAR_LE
                                                      : KAPSEL_EQ_ELECTROLYTE;
  p.precision = shim_precision();
  p.n_particles = Particle_Number;
  p.dx = DX;
  p.rho = RHO;
  p.eta = ETA;
  p.kbt = kBT;
  p.alpha_v = alpha_v;
  p.alpha_o = alpha_o;
  p.dt = DT;
  p.a = A;
  p.a_xi = A_XI;
  p.mass_ratio = Particle_Number > 0 ? MASS_RATIOS[0] : 1.0;
  p.gravity_g = G;
  p.gravity_dir = G_direction;
  p.epsilon = EPSILON;
  p.lj_powers = LJ_powers;
  p.lj_truncate = LJ_truncate;
  p.rotation = ROTATION;
  for (int d = 0; d < DIM; d++) p.fix_cell[d] = FIX_CELL ? FIX_CELLxyz[d] : 0;
  p.mt_seed = (unsigned int)GIVEN_SEED;  // MT_seed(GIVEN_SEED, 0) in main
  if (SW_EQ == Electrolyte) {
    p.dielectric = Dielectric_cst;
    p.surface_charge = Particle_Number > 0 ? Surface_charge[0] : 0.0;
    p.debye_length = Debye_length;
    p.valency_p = Valency_positive_ion;
    p.valency_n = Valency_negative_ion;
    p.onsager_p = Onsager_coeff_positive_ion;
    p.onsager_n = Onsager_coeff_negative_ion;
    for (int d = 0; d < DIM; d++) p.e_ext[d] = E_ext[d];
  }
  p.shear_rate = Shear_rate;
  return p;
}

// Particle <-> the library's particle record (KAPSEL_P_*).
void to_records(const Particle *p, std::vector<double> &rec) {
  rec.assign((size_t)KAPSEL_P_STRIDE * (Particle_Number > 0 ? Particle_Number : 1), 0.0);
  for (int n = 0; n < Particle_Number; n++) {
    double *o = rec.data() + (size_t)KAPSEL_P_STRIDE * n;
    for (int d = 0; d < DIM; d++) {
      o[KAPSEL_P_X + d] = p[n].x[d];
      o[KAPSEL_P_V + d] = p[n].v[d];
      o[KAPSEL_P_OMEGA + d] = p[n].omega[d];
      o[KAPSEL_P_FHYDRO + d] = p[n].f_hydro_previous[d];
      o[KAPSEL_P_THYDRO + d] = p[n].torque_hydro_previous[d];
      o[KAPSEL_P_FR + d] = p[n].fr_previous[d];
      o[KAPSEL_P_XNOPBC + d] = p[n].x_nopbc[d];
      o[KAPSEL_P_VOLD + d] = p[n].v_old[d];
      o[KAPSEL_P_OMEGAOLD + d] = p[n].omega_old[d];
    }
    o[KAPSEL_P_Q + 0] = p[n].q.s;
    o[KAPSEL_P_QOLD + 0] = p[n].q_old.s;
    for (int d = 0; d < DIM; d++) {
      o[KAPSEL_P_Q + 1 + d] = p[n].q.v[d];
      o[KAPSEL_P_QOLD + 1 + d] = p[n].q_old.v[d];
    }
  }
}

// The state after a whole step or a velocity update: positions, velocities,
// orientations and the forces reset_Forces moved into *_previous (the
// current forces are zero after it, particle_solver.cxx:11-34).
void from_records_step(const std::vector<double> &rec, Particle *p) {
  for (int n = 0; n < Particle_Number; n++) {
    const double *o = rec.data() + (size_t)KAPSEL_P_STRIDE * n;
    for (int d = 0; d < DIM; d++) {
      p[n].x[d] = o[KAPSEL_P_X + d];
      p[n].x_nopbc[d] = o[KAPSEL_P_XNOPBC + d];
      p[n].v[d] = o[KAPSEL_P_V + d];
      p[n].v_old[d] = o[KAPSEL_P_VOLD + d];
      p[n].omega[d] = o[KAPSEL_P_OMEGA + d];
      p[n].omega_old[d] = o[KAPSEL_P_OMEGAOLD + d];
      p[n].f_hydro_previous[d] = o[KAPSEL_P_FHYDRO + d];
      p[n].torque_hydro_previous[d] = o[KAPSEL_P_THYDRO + d];
      p[n].fr_previous[d] = o[KAPSEL_P_FR + d];
      p[n].f_hydro[d] = p[n].torque_hydro[d] = p[n].fr[d] = 0.0;
      p[n].f_slip_previous[d] = p[n].f_slip[d];
      p[n].torque_slip_previous[d] = p[n].torque_slip[d];
      p[n].f_slip[d] = p[n].torque_slip[d] = 0.0;
    }
    p[n].q.s = o[KAPSEL_P_Q];
    p[n].q_old.s = o[KAPSEL_P_QOLD];
    for (int d = 0; d < DIM; d++) {
      p[n].q.v[d] = o[KAPSEL_P_Q + 1 + d];
      p[n].q_old.v[d] = o[KAPSEL_P_QOLD + 1 + d];
    }
  }
}

size_t field_len() { return (size_t)NX * NY * NZ_; }

void pack2(double *const *a, std::vector<double> &buf) {
  const size_t n = field_len();
  buf.resize(2 * n);
  memcpy(buf.data(), a[0], sizeof(double) * n);
  memcpy(buf.data() + n, a[1], sizeof(double) * n);
}
void unpack2(const std::vector<double> &buf, double **a) {
  const size_t n = field_len();
  memcpy(a[0], buf.data(), sizeof(double) * n);
  memcpy(a[1], buf.data() + n, sizeof(double) * n);
}

#if KAPSEL_SHIM_STEP
// ---- whole-step registry ----------------------------------------------------
struct StepCtx {
  kapsel_ctx *ctx = nullptr;
  std::vector<double> x_mirror;  // particle positions as last mirrored
  bool dirty = true;             // upload the host state before the next step
};
std::map<const double *, StepCtx> g_step;

bool mirror_every() {
  const char *e = getenv("KAPSEL_SHIM_MIRROR");
  return e && strcmp(e, "every") == 0;
}

bool host_changed(const StepCtx &s, const Particle *p) {
  if (s.x_mirror.size() != (size_t)DIM * Particle_Number) return true;
  for (int n = 0; n < Particle_Number; n++)
    for (int d = 0; d < DIM; d++)
      if (p[n].x[d] != s.x_mirror[(size_t)DIM * n + d]) return true;
  return false;
}

// the ion concentrations and the Rescale_solute targets of the host run
// (Electrolyte branch)
void upload_concentrations(kapsel_ctx *c) {
  if (SW_EQ != Electrolyte) return;
  std::vector<double> buf;
  pack2(Concentration, buf);
  check(kapsel_gpu_set_concentration(c, buf.data(), Total_solute), "kapsel_gpu_set_concentration");
}

void upload(StepCtx &s, double **zeta, const double *uk_dc, Particle *p, const CTime &jikan) {
  std::vector<double> buf, rec;
  if (Particle_Number > 0) {
    to_records(p, rec);
    check(kapsel_gpu_set_particle_state(s.ctx, rec.data()), "kapsel_gpu_set_particle_state");
  }
  pack2(zeta, buf);
  check(kapsel_gpu_set_zeta(s.ctx, buf.data(), uk_dc), "kapsel_gpu_set_zeta");
  upload_concentrations(s.ctx);
  if (SW_EQ == Shear_Navier_Stokes_Lees_Edwards)
    check(kapsel_gpu_set_oblique(s.ctx, degree_oblique, Shear_rate_eff), "kapsel_gpu_set_oblique");
  check(kapsel_gpu_set_time(s.ctx, jikan.ts, jikan.time), "kapsel_gpu_set_time");
  s.dirty = false;
}

void remember_positions(StepCtx &s, const Particle *p) {
  s.x_mirror.resize((size_t)DIM * Particle_Number);
  for (int n = 0; n < Particle_Number; n++)
    for (int d = 0; d < DIM; d++) s.x_mirror[(size_t)DIM * n + d] = p[n].x[d];
}

StepCtx &attach(double **zeta, double *uk_dc, Particle *p, const CTime &jikan) {
  auto it = g_step.find(zeta[0]);
  if (it == g_step.end()) {
    StepCtx s;
    kapsel_params prm = params_from_globals();
    check(kapsel_gpu_create(&prm, &s.ctx), "kapsel_gpu_create");
    if (Particle_Number > 0) {
      std::vector<double> x((size_t)DIM * Particle_Number), q((size_t)4 * Particle_Number);
      for (int n = 0; n < Particle_Number; n++) {
        for (int d = 0; d < DIM; d++) x[DIM * n + d] = p[n].x[d];
        q[4 * n] = p[n].q.s;
        for (int d = 0; d < DIM; d++) q[4 * n + 1 + d] = p[n].q.v[d];
      }
      check(kapsel_gpu_set_particles(s.ctx, x.data(), q.data()), "kapsel_gpu_set_particles");
    }
    // the device's own initialisation (its fields are replaced by the host's
    // below)
    check(kapsel_gpu_init_state(s.ctx), "kapsel_gpu_init_state");
    fprintf(stderr, "kapsel shim: Time_evolution on the GPU (%dx%dx%d, %d particles, %s)\n", NX, NY, NZ,
            Particle_Number, prm.precision == KAPSEL_FP64 ? "FP64" : "mixed");
    it = g_step.emplace(zeta[0], s).first;
    // then the host's fluid and particle state and step counter
    StepCtx &a = it->second;
    std::vector<double> buf, rec;
    if (Particle_Number > 0) {
      to_records(p, rec);
      check(kapsel_gpu_set_particle_state(a.ctx, rec.data()), "kapsel_gpu_set_particle_state");
    }
    pack2(zeta, buf);
    check(kapsel_gpu_set_zeta(a.ctx, buf.data(), uk_dc), "kapsel_gpu_set_zeta");
    upload_concentrations(a.ctx);
    if (SW_EQ == Shear_Navier_Stokes_Lees_Edwards)
      check(kapsel_gpu_set_oblique(a.ctx, degree_oblique, Shear_rate_eff), "kapsel_gpu_set_oblique");
    check(kapsel_gpu_set_time(a.ctx, jikan.ts, jikan.time), "kapsel_gpu_set_time");
    remember_positions(a, p);
    a.dirty = false;
  }
  StepCtx &s = it->second;
  int ts = 0;
  check(kapsel_gpu_get_time(s.ctx, &ts, nullptr), "kapsel_gpu_get_time");
  if (s.dirty || ts != jikan.ts || host_changed(s, p)) {
    upload(s, zeta, uk_dc, p, jikan);
    remember_positions(s, p);
  }
  return s;
}

void mirror(StepCtx &s, double **zeta, double *uk_dc, Particle *p, const CTime &jikan) {
  std::vector<double> rec, buf;
  if (Particle_Number > 0) {
    rec.resize((size_t)KAPSEL_P_STRIDE * Particle_Number);
    check(kapsel_gpu_get_particles(s.ctx, rec.data()), "kapsel_gpu_get_particles");
    from_records_step(rec, p);
    remember_positions(s, p);
  }
  if (SW_EQ == Shear_Navier_Stokes_Lees_Edwards) {
    double ob[3];
    check(kapsel_gpu_get_oblique(s.ctx, ob), "kapsel_gpu_get_oblique");
    degree_oblique = ob[0];
    Shear_rate_eff = ob[1];
  }
  // the main loop reads the fields before Output_* (top of the iteration
  // whose ts is a multiple of GTS) and in Save_Restart_udf (ts == MSTEP)
  const bool wanted = mirror_every() || (jikan.ts + 1) % GTS == 0 || jikan.ts == MSTEP;
  if (!wanted) return;
  buf.resize(2 * field_len());
  check(kapsel_gpu_get_zeta(s.ctx, buf.data(), uk_dc), "kapsel_gpu_get_zeta");
  unpack2(buf, zeta);
  if (SW_EQ == Electrolyte) {
    check(kapsel_gpu_get_concentration(s.ctx, buf.data()), "kapsel_gpu_get_concentration");
    unpack2(buf, Concentration);
  }
}

void gpu_step(double **zeta, double *uk_dc, Particle *p, CTime &jikan) {
  StepCtx &s = attach(zeta, uk_dc, p, jikan);
  check(kapsel_gpu_step_graph(s.ctx, 1), "kapsel_gpu_step_graph");
  mirror(s, zeta, uk_dc, p, jikan);
}
#endif  // KAPSEL_SHIM_STEP

#if KAPSEL_SHIM_ROUTINES
// ---- routine work context -----------------------------------------------------
kapsel_ctx *g_work = nullptr;

kapsel_ctx *work_ctx() {
  if (!g_work) {
    kapsel_params prm = params_from_globals();
    prm.eq = KAPSEL_EQ_NAVIER_STOKES;  // the routines below are the Navier_Stokes ones
    check(kapsel_gpu_create(&prm, &g_work), "kapsel_gpu_create");
    fprintf(stderr, "kapsel shim: solver routines on the GPU (%dx%dx%d, %d particles)\n", NX, NY, NZ,
            Particle_Number);
  }
  return g_work;
}

kapsel_ctx *g_work_el = nullptr;

// true when every mode of the two k-space fields outside the 2/3 box
// (Truncate_two_third_rule_ooura, fft_wrapper.h:723-766) is zero: the
// library keeps only the box, so a field with modes outside it (an initial
// profile other than Uniform, operate_electrolyte.cxx:490-515) is refused
bool truncated2(double *const *a) {
  for (int f = 0; f < 2; f++)
    for (int i = 0; i < NX; i++)
      for (int j = 0; j < NY; j++) {
        const bool row_in = (i < TRN_X || i > NX - TRN_X) && (j < TRN_Y || j > NY - TRN_Y);
        const double *r = a[f] + ((size_t)i * NY + j) * NZ_;
        for (int k = row_in ? 2 * TRN_Z : 0; k < NZ_; k++)
          if (r[k] != 0.0) return false;
      }
  return true;
}

kapsel_ctx *work_ctx_el() {
  if (SW_EQ != Electrolyte) shim_fail("an Electrolyte routine outside the Electrolyte branch", 0);
  if (!g_work_el) {
    kapsel_params prm = params_from_globals();
    check(kapsel_gpu_create(&prm, &g_work_el), "kapsel_gpu_create");
    fprintf(stderr, "kapsel shim: Electrolyte routines on the GPU (%dx%dx%d, %d particles)\n", NX, NY, NZ,
            Particle_Number);
  }
  return g_work_el;
}

void upload_particles(kapsel_ctx *c, const Particle *p) {
  if (Particle_Number == 0) return;
  std::vector<double> rec;
  to_records(p, rec);
  check(kapsel_gpu_set_particle_state(c, rec.data()), "kapsel_gpu_set_particle_state");
}

std::vector<double> download_particles(kapsel_ctx *c) {
  std::vector<double> rec((size_t)KAPSEL_P_STRIDE * (Particle_Number > 0 ? Particle_Number : 1));
  if (Particle_Number > 0) check(kapsel_gpu_get_particles(c, rec.data()), "kapsel_gpu_get_particles");
  return rec;
}

void position_update(Particle *p, const CTime &jikan, int euler) {
  if (jikan.dt_md != DT) shim_fail("a particle time step other than DT", 0);
  kapsel_ctx *c = work_ctx();
  upload_particles(c, p);
  check(kapsel_gpu_md_position(c, euler), "kapsel_gpu_md_position");
  const std::vector<double> rec = download_particles(c);
  for (int n = 0; n < Particle_Number; n++) {
    const double *o = rec.data() + (size_t)KAPSEL_P_STRIDE * n;
    for (int d = 0; d < DIM; d++) {
      p[n].x_previous[d] = p[n].x[d];
      p[n].x[d] = o[KAPSEL_P_X + d];
      p[n].x_nopbc[d] = o[KAPSEL_P_XNOPBC + d];
    }
    if (ROTATION) {
      p[n].q.s = o[KAPSEL_P_Q];
      p[n].q_old.s = o[KAPSEL_P_QOLD];
      for (int d = 0; d < DIM; d++) {
        p[n].q.v[d] = o[KAPSEL_P_Q + 1 + d];
        p[n].q_old.v[d] = o[KAPSEL_P_QOLD + 1 + d];
      }
    }
  }
}

void velocity_update(Particle *p, const CTime &jikan, int euler) {
  if (jikan.dt_md != DT) shim_fail("a particle time step other than DT", 0);
  kapsel_ctx *c = work_ctx();
  upload_particles(c, p);
  std::vector<double> fh((size_t)DIM * Particle_Number), th((size_t)DIM * Particle_Number);
  for (int n = 0; n < Particle_Number; n++)
    for (int d = 0; d < DIM; d++) {
      fh[DIM * n + d] = p[n].f_hydro[d];
      th[DIM * n + d] = p[n].torque_hydro[d];
    }
  check(kapsel_gpu_md_velocity(c, fh.data(), th.data(), euler), "kapsel_gpu_md_velocity");
  from_records_step(download_particles(c), p);
}
#endif  // KAPSEL_SHIM_ROUTINES

}  // namespace

extern "C" {
// Marks the whole-step state of the run whose zeta is `zeta` as changed on
// the host: the next step uploads it again.
void kapsel_shim_invalidate(double **zeta) {
#if KAPSEL_SHIM_STEP
  auto it = g_step.find(zeta[0]);
  if (it != g_step.end()) it->second.dirty = true;
#else
  (void)zeta;
#endif
}
}

#if KAPSEL_SHIM_STEP
void Time_evolution_hydro(double **zeta, double uk_dc[DIM], double **f, Particle *p, CTime &jikan) {
  (void)f;  // the rigidity force field stays on the device
  if (SW_EQ != Navier_Stokes && SW_EQ != Electrolyte) shim_fail("Time_evolution_hydro branch", 0);
  gpu_step(zeta, uk_dc, p, jikan);
}

void Time_evolution_hydro_OBL(double **zeta, double uk_dc[DIM], double **f, Particle *p, CTime &jikan) {
  (void)f;
  if (SW_EQ != Shear_Navier_Stokes_Lees_Edwards) shim_fail("Time_evolution_hydro_OBL branch", 0);
  gpu_step(zeta, uk_dc, p, jikan);
}
#endif

#if KAPSEL_SHIM_ROUTINES
void NS_solver_slavedEuler(double **zeta, const CTime &jikan, double uk_dc[DIM], const Index_range *ijk_range,
                           const int &n_ijk_range, Particle *p) {
  // the ranges are the 2/3 box of Truncate_two_third_rule (the only ranges
  // the reference passes, sp_3d_ns.cxx:15-21); the library keeps exactly
  // those modes
  (void)ijk_range;
  (void)n_ijk_range;
  (void)p;
  if (jikan.dt_fluid != DT) shim_fail("a fluid time step other than DT", 0);
  kapsel_ctx *c = work_ctx();
  std::vector<double> buf;
  pack2(zeta, buf);
  check(kapsel_gpu_ns_slaved_euler(c, buf.data(), uk_dc), "kapsel_gpu_ns_slaved_euler");
  unpack2(buf, zeta);
}

void Make_phi_particle(double *phi, Particle *p, const double radius) {
  // phi is overwritten with the profile sum (the reference adds it to a
  // field its callers have reset)
  if (radius != RADIUS) shim_fail("Make_phi_particle with a radius other than RADIUS", 0);
  kapsel_ctx *c = work_ctx();
  upload_particles(c, p);
  check(kapsel_gpu_make_phi(c, phi), "kapsel_gpu_make_phi");
}

void Make_phi_u_particle(double *phi, double **up, Particle *p) {
  // phi and up are overwritten (the reference adds to fields its callers
  // have reset with Reset_phi_u), then clamped where phi > 1
  kapsel_ctx *c = work_ctx();
  upload_particles(c, p);
  check(kapsel_gpu_make_phi_u(c, phi, up[0], up[1], up[2]), "kapsel_gpu_make_phi_u");
}

void Calc_f_hydro_correct_precision(Particle *p, double const *const *u, const CTime &jikan) {
  if (jikan.dt_fluid != DT) shim_fail("a fluid time step other than DT", 0);
  kapsel_ctx *c = work_ctx();
  upload_particles(c, p);
  std::vector<double> f((size_t)DIM * (Particle_Number > 0 ? Particle_Number : 1)), t(f.size());
  if (Particle_Number > 0)
    check(kapsel_gpu_calc_f_hydro(c, u[0], u[1], u[2], f.data(), t.data()), "kapsel_gpu_calc_f_hydro");
  for (int n = 0; n < Particle_Number; n++) {
    for (int d = 0; d < DIM; d++) {
      p[n].f_hydro[d] = f[DIM * n + d];
      p[n].f_slip[d] = 0.0;
    }
    if (ROTATION)
      for (int d = 0; d < DIM; d++) {
        p[n].torque_hydro[d] = t[DIM * n + d];
        p[n].torque_slip[d] = 0.0;
      }
  }
}

double Calc_f_Lennard_Jones_shear_cap_primitive_lnk(Particle *p,
                                                    void (*distance0_func)(const double *x1, const double *x2,
                                                                           double &r12, double *x12),
                                                    const double cap) {
  // the minimum-image pair distance and no cap: what Calc_f_Lennard_Jones
  // (md_force.h:75-78) passes.  The return value (the pairs' xy stress
  // sum, read by no Navier_Stokes caller) and the Min_rij / Max_force
  // diagnostics are not computed: 0 is returned.
  if (distance0_func != Distance0 || cap != DBL_MAX) shim_fail("LJ with another distance or a force cap", 0);
  kapsel_ctx *c = work_ctx();
  upload_particles(c, p);
  std::vector<double> fr((size_t)DIM * (Particle_Number > 0 ? Particle_Number : 1));
  check(kapsel_gpu_calc_lj(c, fr.data()), "kapsel_gpu_calc_lj");
  for (int n = 0; n < Particle_Number; n++)
    for (int d = 0; d < DIM; d++) p[n].fr[d] += fr[DIM * n + d];
  return 0.0;
}

void MD_solver_position_Euler(Particle *p, const CTime &jikan) { position_update(p, jikan, 1); }
void MD_solver_position_AB2(Particle *p, const CTime &jikan) { position_update(p, jikan, 0); }
void MD_solver_velocity_Euler(Particle *p, const CTime &jikan) { velocity_update(p, jikan, 1); }
void MD_solver_velocity_AB2_hydro(Particle *p, const CTime &jikan) { velocity_update(p, jikan, 0); }

void NSsolute_solver_Euler(double **zeta, const CTime &jikan, double uk_dc[DIM], double **concentration_k,
                           Particle *p, const Index_range *ijk_range, const int &n_ijk_range) {
  // the ranges are the 2/3 box (sp_3d_ns.cxx:46-58), the only ones the
  // reference passes; zeta and the concentrations come back truncated to it,
  // as the reference leaves them (Rhs_NS_solute truncates both first)
  (void)ijk_range;
  (void)n_ijk_range;
  if (jikan.dt_fluid != DT) shim_fail("a fluid time step other than DT", 0);
  kapsel_ctx *c = work_ctx_el();
  upload_particles(c, p);
  std::vector<double> z, conc;
  pack2(zeta, z);
  pack2(concentration_k, conc);
  check(kapsel_gpu_ns_solute_euler(c, z.data(), uk_dc, conc.data()), "kapsel_gpu_ns_solute_euler");
  unpack2(z, zeta);
  unpack2(conc, concentration_k);
}

void Rescale_solute(double *rescale_factor, double *total_solute, double **conc_k, Particle *p, double *phi,
                    double *conc_x) {
  // phi and conc_x are the reference's working memory; no caller reads them
  // afterwards (sp_3d_ns.cxx:89-95 resets phi next; fluid_solver.cxx:296-301)
  (void)phi;
  (void)conc_x;
  kapsel_ctx *c = work_ctx_el();
  if (!truncated2(conc_k)) shim_fail("Rescale_solute on concentrations with modes outside the 2/3 box", 0);
  upload_particles(c, p);
  std::vector<double> conc;
  pack2(conc_k, conc);
  check(kapsel_gpu_rescale_solute(c, total_solute, conc.data(), rescale_factor), "kapsel_gpu_rescale_solute");
  unpack2(conc, conc_k);
}

void Make_Coulomb_force_x_on_fluid(double **force, Particle *p, double **conc_k, double *charge_density,
                                   double *potential, const CTime &jikan) {
  // charge_density and potential are working memory (up[0], up[1] in
  // Time_evolution_hydro, reset before their next use); the DC field only
  (void)charge_density;
  (void)potential;
  (void)jikan;
  kapsel_ctx *c = work_ctx_el();
  if (!truncated2(conc_k)) shim_fail("the Coulomb force of concentrations with modes outside the 2/3 box", 0);
  upload_particles(c, p);
  std::vector<double> conc;
  pack2(conc_k, conc);
  check(kapsel_gpu_coulomb_force(c, conc.data(), force[0], force[1], force[2]), "kapsel_gpu_coulomb_force");
}
#endif  // KAPSEL_SHIM_ROUTINES
