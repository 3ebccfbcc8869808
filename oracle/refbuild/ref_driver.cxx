/*
 * Driver that runs the UNMODIFIED KAPSEL reference sources as a CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY: it is linked against the reference translation
 * units (compiled from their original location by oracle/Makefile) and is
 * used by tests/golden/make_golden.py to produce golden vectors, and by
 * bench.py as the timed CPU reference arm.  Nothing in the product links it.
 *
 * The initialisation sequence follows the reference main()
 * (sp_3d_ns.cxx:442-540): file_get/Gourmet_file_io, Time_evolution binding,
 * MT_seed(GIVEN_SEED,0), Init_fft, Mem_alloc_var, Init_Particle, Init_zeta_k,
 * the initial rigidity projection and (electrolyte) Init_rho_ion.  Each step
 * is Time_evolution(...) followed by jikan.time += dt (sp_3d_ns.cxx:593-594).
 * UDF/AVS snapshot output is not called; restart records are written and
 * read back on request (kref_save_restart, kref_resume).
 */
#include "sp_3d_ns.h"

#include <sys/time.h>

extern void (*Time_evolution)(double **zeta, double uk_dc[DIM], double **f, Particle *p, CTime &jikan);
void Time_evolution_hydro(double **zeta, double uk_dc[DIM], double **f, Particle *p, CTime &jikan);
void Time_evolution_hydro_OBL(double **zeta, double uk_dc[DIM], double **f, Particle *p, CTime &jikan);
extern double **ucp;
/* emitted from sp_3d_ns.cxx by -fkeep-inline-functions */
void Mem_alloc_var(double **zeta);

namespace {
double **g_zeta = NULL;
double g_uk_dc[DIM];
Particle *g_particles = NULL;
CTime g_jikan;
int g_ready = 0;
std::string g_out, g_res;
}

extern "C" {

/* Initialise the reference from a flat `path = value` UDF stand-in file. */
int kref_init(const char *kv_path) {
  if (g_ready) return -1;
  g_out = std::string(kv_path) + ".out";
  g_res = std::string(kv_path) + ".res";
  std::string a0 = "kapsel", aI = std::string("-I") + kv_path, aO = "-O" + g_out,
              aD = std::string("-D") + kv_path, aR = "-R" + g_res;
  char *argv[5] = {&a0[0], &aI[0], &aO[0], &aD[0], &aR[0]};
  file_get(5, argv);
  Gourmet_file_io(In_udf, Out_udf, Sum_udf, Def_udf, Ctrl_udf, Res_udf);
  if (SW_EQ == Shear_Navier_Stokes) return -2; /* not driven here */
  Time_evolution = SW_EQ == Shear_Navier_Stokes_Lees_Edwards ? Time_evolution_hydro_OBL : Time_evolution_hydro;

  MT_seed(GIVEN_SEED, 0);
  Init_fft();
  g_zeta = (double **)malloc(sizeof(double *) * (DIM - 1));
  Mem_alloc_var(g_zeta);
  CTime j0 = {0, 0.0, DT, DT * 0.5, DT, DT * 0.5};
  g_jikan = j0;

  g_particles = new Particle[Particle_Number > 0 ? Particle_Number : 1];
  if (Particle_Number > 0) Init_Particle(g_particles);
  Init_zeta_k(g_zeta, g_uk_dc);
  {
    Reset_phi_u(phi, up);
    Make_phi_u_particle(phi, up, g_particles);
    Zeta_k2u(g_zeta, g_uk_dc, u);
    Make_f_particle_dt_sole(f_particle, u, up, phi);
    Add_f_particle(u, f_particle);
    U2zeta_k(g_zeta, g_uk_dc, u);
    for (int d = 0; d < DIM; d++) g_uk_dc[d] = 0.0;
  }
  if (SW_EQ == Electrolyte) Init_rho_ion(Concentration, g_particles, g_jikan);
  if (SW_EQ == Shear_Navier_Stokes_Lees_Edwards && !Fixed_particle) {
    /* the v_x / omega_z reset that Show_parameter applies in the sheared
       branches (init_particle.cxx:666-677), without its report */
    for (int n = 0; n < Particle_Number; n++) {
      g_particles[n].v[0] = 0.0;
      g_particles[n].v_old[0] = 0.0;
      g_particles[n].omega[2] = 0.0;
      g_particles[n].omega_old[2] = 0.0;
    }
  }
  g_ready = 1;
  return 0;
}

int kref_step(int n) {
  if (!g_ready) return -1;
  for (int s = 0; s < n; s++) {
    Time_evolution(g_zeta, g_uk_dc, f_particle, g_particles, g_jikan);
    g_jikan.time += g_jikan.dt_fluid;
    /* main loop bookkeeping of the Lees-Edwards branch (sp_3d_ns.cxx:599-601;
       Mean_shear_stress only reports) */
    if (SW_EQ == Shear_Navier_Stokes_Lees_Edwards) Shear_strain_realized += Shear_rate_eff * g_jikan.dt_fluid;
    g_jikan.ts++;
  }
  return 0;
}

/* Output_udf of the current state into the output record file (the stand-in
   manager writes "record <n> path = value" lines to <input>.out, record 0
   holding the input values Gourmet_file_io echoed); as the step loop calls
   it (sp_3d_ns.cxx:568-570). */
int kref_output_udf(void) {
  if (!g_ready || !ufout) return -1;
  Output_udf(ufout, Avs_parameters, g_zeta, g_uk_dc, g_particles, g_jikan);
  ufout->write();
  return 0;
}

/* Set the velocity and angular velocity of particle n (and their previous
   values, as a fresh start has them equal). */
int kref_set_particle_velocity(int n, const double *v, const double *w) {
  if (!g_ready || n < 0 || n >= Particle_Number) return -1;
  for (int d = 0; d < DIM; d++) {
    g_particles[n].v[d] = g_particles[n].v_old[d] = v[d];
    g_particles[n].omega[d] = g_particles[n].omega_old[d] = w[d];
  }
  return 0;
}

/* Lees-Edwards state: out = degree_oblique, Shear_rate_eff, Shear_strain_realized. */
void kref_oblique(double *out) {
  out[0] = degree_oblique;
  out[1] = Shear_rate_eff;
  out[2] = Shear_strain_realized;
}

/* Set degree_oblique and Shear_rate_eff and rebuild K2/IK2 for the new
   degree_oblique, as the resume path does (resume.cxx:333-360). */
int kref_set_oblique(double deg, double srate) {
  if (!g_ready || SW_EQ != Shear_Navier_Stokes_Lees_Edwards) return -1;
  degree_oblique = deg;
  Shear_rate_eff = srate;
  for (int i = 0; i < NX; i++)
    for (int j = 0; j < NY; j++)
      for (int k = 0; k < NZ_; k++) {
        const int im = (i * NY * NZ_) + (j * NZ_) + k;
        K2[im] = SQ(WAVE_X * KX_int[im]) + SQ(WAVE_Y * KY_int[im] - WAVE_X * degree_oblique * KX_int[im]) +
                 SQ(WAVE_Z * KZ_int[im]);
        IK2[im] = K2[im] > 0.0 ? 1.0 / K2[im] : 0.0;
      }
  return 0;
}

/* dims[0..7] = NX, NY, NZ, NZ_, Particle_Number, NP_domain, N_spec, SW_EQ */
void kref_dims(int *dims) {
  dims[0] = NX; dims[1] = NY; dims[2] = NZ; dims[3] = NZ_;
  dims[4] = Particle_Number; dims[5] = NP_domain; dims[6] = N_spec; dims[7] = (int)SW_EQ;
}

/* scal[0..] = DT, NU, RADIUS, XI, HXI, MASS[0], MOI[0], kBT, time */
void kref_scalars(double *s) {
  s[0] = DT; s[1] = NU; s[2] = RADIUS; s[3] = XI; s[4] = HXI;
  s[5] = Particle_Number > 0 ? MASS[0] : 0.0;
  s[6] = Particle_Number > 0 ? MOI[0] : 0.0;
  s[7] = kBT; s[8] = g_jikan.time;
}

int kref_ts(void) { return g_jikan.ts; }

/* Copy a NX*NY*NZ_ field.  which: 0-2 u, 3 phi, 4-6 up, 7-8 zeta, 9-11 f_particle,
   12-14 ucp (Lees-Edwards: the Cartesian velocity of the step), 20+n
   Concentration[n] (k-space), 30-32 work_v3 */
int kref_get_field(int which, double *out) {
  double *src = NULL;
  if (which >= 0 && which < 3) src = u[which];
  else if (which == 3) src = phi;
  else if (which >= 4 && which < 7) src = up[which - 4];
  else if (which >= 7 && which < 9) src = g_zeta[which - 7];
  else if (which >= 9 && which < 12) src = f_particle[which - 9];
  else if (which >= 12 && which < 15 && ucp) src = ucp[which - 12];
  else if (which >= 20 && which < 20 + N_spec && SW_EQ == Electrolyte) src = Concentration[which - 20];
  else if (which >= 30 && which < 33) src = work_v3[which - 30];
  if (!src) return -1;
  memcpy(out, src, sizeof(double) * (size_t)NX * NY * NZ_);
  return 0;
}

int kref_set_field(int which, const double *in) {
  double *dst = NULL;
  if (which >= 7 && which < 9) dst = g_zeta[which - 7];
  else if (which >= 20 && which < 20 + N_spec && SW_EQ == Electrolyte) dst = Concentration[which - 20];
  if (!dst) return -1;
  memcpy(dst, in, sizeof(double) * (size_t)NX * NY * NZ_);
  return 0;
}

void kref_get_ukdc(double *out) { for (int d = 0; d < DIM; d++) out[d] = g_uk_dc[d]; }
void kref_set_ukdc(const double *in) { for (int d = 0; d < DIM; d++) g_uk_dc[d] = in[d]; }

/* 35 doubles per particle: x v omega f_hydro_previous torque_hydro_previous
   fr_previous x_nopbc v_old omega_old (3 each) q(s,v0,v1,v2) q_old(4) */
void kref_get_particles(double *out) {
  for (int n = 0; n < Particle_Number; n++) {
    const Particle &p = g_particles[n];
    double *o = out + 35 * n;
    for (int d = 0; d < DIM; d++) {
      o[0 + d] = p.x[d]; o[3 + d] = p.v[d]; o[6 + d] = p.omega[d];
      o[9 + d] = p.f_hydro_previous[d]; o[12 + d] = p.torque_hydro_previous[d];
      o[15 + d] = p.fr_previous[d]; o[18 + d] = p.x_nopbc[d];
      o[21 + d] = p.v_old[d]; o[24 + d] = p.omega_old[d];
    }
    o[27] = p.q.s; o[28] = p.q.v[0]; o[29] = p.q.v[1]; o[30] = p.q.v[2];
    o[31] = p.q_old.s; o[32] = p.q_old.v[0]; o[33] = p.q_old.v[1]; o[34] = p.q_old.v[2];
  }
}

void kref_set_efield(double ex, double ey, double ez) {
  E_ext[0] = ex; E_ext[1] = ey; E_ext[2] = ez;
  External_field = (ex != 0.0 || ey != 0.0 || ez != 0.0) ? 1 : 0;
}

/* Sekibun stencil: writes NP_domain*3 ints (if out != NULL), returns NP_domain */
int kref_sekibun(int *out) {
  if (out)
    for (int m = 0; m < NP_domain; m++)
      for (int d = 0; d < DIM; d++) out[3 * m + d] = Sekibun_cell[m][d];
  return NP_domain;
}

/* Primitive-level hooks on the reference's own spectral wrappers */
void kref_A2a_k(double *a) { A2a_k(a); }
void kref_A_k2a(double *a) { A_k2a(a); }
void kref_solenoidal_u(double *f0, double *f1, double *f2) {
  double *f[3] = {f0, f1, f2};
  Solenoidal_u(f);
}

/* Save_Restart_udf as the step loop calls it after its last step
   (sp_3d_ns.cxx:606-616: jikan.ts is the index of the step just done),
   written through the stand-in record writer. */
int kref_save_restart(const char *path) {
  if (!g_ready) return -1;
  UDFManager res(path, "", 0);
  UDFManager *old = ufres;
  ufres = &res;
  CTime j = g_jikan;
  j.ts -= 1;
  Save_Restart_udf(g_zeta, g_uk_dc, g_particles, j, Concentration);
  res.write();
  ufres = old;
  return 0;
}

/* The first pass of a resumed run's step loop (sp_3d_ns.cxx:545-627): one
   Time_evolution at ts = last_ts, then Force_restore_parameters from the
   restart file, then ts++. */
int kref_resume(const char *path) {
  if (!g_ready) return -1;
  UDFManager in(path);
  int last_ts = 0;
  if (!in.get("resume.CONTINUE.Saved_Data.jikan.ts", last_ts)) return -2;
  g_jikan.ts = last_ts;
  Time_evolution(g_zeta, g_uk_dc, f_particle, g_particles, g_jikan);
  g_jikan.time += g_jikan.dt_fluid;
  UDFManager *old = ufin;
  ufin = &in;
  Force_restore_parameters(g_zeta, g_uk_dc, g_particles, g_jikan, Concentration);
  ufin = old;
  g_jikan.ts += 1;
  return 0;
}

/* Output_avs_p and Output_avs (Output_avs_charge in the Electrolyte branch)
   of the current state as the step loop calls them (sp_3d_ns.cxx:553-566,
   BINARY); init writes the .fld headers and the .cod file first (Init_avs,
   Init_avs_p).  Needs output.AVS = ON in the input. */
int kref_output_avs(int init) {
  if (!g_ready || !SW_AVS || (SW_EQ != Navier_Stokes && SW_EQ != Electrolyte)) return -1;
  Set_avs_parameters(Avs_parameters);
  if (init) {
    Init_avs(Avs_parameters);
    if (Particle_Number > 0) Init_avs_p(Avs_parameters);
  }
  // as the main loop writes them (sp_3d_ns.cxx:555-566)
  if (Particle_Number > 0) Output_avs_p(Avs_parameters, g_particles, g_jikan);
  if (SW_EQ == Electrolyte)
    Output_avs_charge(Avs_parameters, g_zeta, g_uk_dc, Concentration, g_particles, g_jikan);
  else
    Output_avs(Avs_parameters, g_zeta, g_uk_dc, g_particles, g_jikan);
  return 0;
}

/* Wall-clock seconds of n steps (excludes initialisation). */
double kref_time_steps(int n) {
  struct timeval a, b;
  gettimeofday(&a, NULL);
  kref_step(n);
  gettimeofday(&b, NULL);
  return (double)(b.tv_sec - a.tv_sec) + 1e-6 * (double)(b.tv_usec - a.tv_usec);
}

} /* extern "C" */

#ifdef KREF_CLI
/* kapsel_ref <kv-file> <warmup> <steps>: prints {"s_per_step": ...} */
int main(int argc, char **argv) {
  if (argc < 4) { fprintf(stderr, "usage: %s kv warmup steps\n", argv[0]); return 2; }
  if (kref_init(argv[1]) != 0) return 3;
  kref_step(atoi(argv[2]));
  int n = atoi(argv[3]);
  double t = kref_time_steps(n);
  printf("{\"steps\": %d, \"seconds\": %.6f, \"s_per_step\": %.6f}\n", n, t, t / n);
  return 0;
}
#endif
