/*
 * kapsel_gpu.h -- C ABI of the B200 (sm_100a) Smoothed Profile Method step.
 *
 * The library replaces KAPSEL's SPM time step, Time_evolution_hydro
 * (sp_3d_ns.cxx:61-212), and the solver routines it calls.  State (reduced
 * vorticity, k=0 velocity, particles) lives on the GPU between calls; host
 * buffers cross the boundary only in the reference's own layouts:
 *
 *   - k-space fields in the Ooura layout of the reference: NX*NY*NZ_ doubles,
 *     NZ_ = NZ+2, index (i*NY + j)*NZ_ + 2*kz (+1 for the imaginary part),
 *     forward sign exp(+i k.x) (fft_wrapper.h:432-631);
 *   - real-space fields as NX*NY*NZ_ doubles with the same padded stride
 *     (sp_3d_ns.cxx:392-440 allocates every field this way);
 *   - particles as the reference Particle fields, see KAPSEL_P_* below
 *     (variable.h:27-75).
 *
 * Every entry point returns 0 on success or a negative KAPSEL_E* status; the
 * library never exits the process (the reference calls exit_job, macro.h:194).
 * One context owns one CUDA stream; contexts are independent.
 *
 * Failure detection: parameters and particle records are checked on the
 * host (a NaN or Inf, a position outside the box: KAPSEL_EINVAL /
 * KAPSEL_ERANGE, nothing is sent to the device).  During a step the device
 * flags a non-finite particle velocity (KAPSEL_ENONFINITE), a particle
 * outside the box or a full neighbour list (KAPSEL_ERANGE) and a bounded
 * wait that ran out (KAPSEL_ETIMEOUT); the step's status returns it, and it
 * stays until the state is replaced (kapsel_gpu_set_zeta,
 * kapsel_gpu_set_particles / _set_particle_state, kapsel_gpu_load_restart).
 */
#ifndef KAPSEL_GPU_H
#define KAPSEL_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define KAPSEL_OK 0
#define KAPSEL_EINVAL -1     /* bad argument or unsupported configuration */
#define KAPSEL_ECUDA -2      /* a CUDA runtime call failed */
#define KAPSEL_ENOMEM -3     /* device allocation failed */
#define KAPSEL_ESTATE -4     /* call out of order (e.g. step before init) */
#define KAPSEL_ENONFINITE -5 /* a NaN/Inf was detected in the particle state */
#define KAPSEL_ERANGE -6     /* a particle left the box or a size limit was exceeded */
#define KAPSEL_ETIMEOUT -7   /* a bounded device wait ran out */

#define KAPSEL_FP64 0  /* all fields and FFTs in double precision */
#define KAPSEL_MIXED 1 /* fields/FFTs/stencils in float, particles and reductions in double */

#define KAPSEL_EQ_NAVIER_STOKES 0 /* EQ::Navier_Stokes (input.h:46) */
#define KAPSEL_EQ_SHEAR_LE 2      /* EQ::Shear_Navier_Stokes_Lees_Edwards (input.h:48) */
#define KAPSEL_EQ_ELECTROLYTE 3   /* EQ::Electrolyte (input.h:49) */

/* Per-particle record layout used by kapsel_gpu_get_particles (doubles). */
#define KAPSEL_P_X 0         /* x[3]                      */
#define KAPSEL_P_V 3         /* v[3]                      */
#define KAPSEL_P_OMEGA 6     /* omega[3]                  */
#define KAPSEL_P_FHYDRO 9    /* f_hydro_previous[3]       */
#define KAPSEL_P_THYDRO 12   /* torque_hydro_previous[3]  */
#define KAPSEL_P_FR 15       /* fr_previous[3]            */
#define KAPSEL_P_XNOPBC 18   /* x_nopbc[3]                */
#define KAPSEL_P_VOLD 21     /* v_old[3]                  */
#define KAPSEL_P_OMEGAOLD 24 /* omega_old[3]              */
#define KAPSEL_P_Q 27        /* q (s, v0, v1, v2)         */
#define KAPSEL_P_QOLD 31     /* q_old (s, v0, v1, v2)     */
#define KAPSEL_P_STRIDE 35

/* Physical and numerical parameters: the values Gourmet_file_io reads from
   the UDF (input.cxx:438-1818) for one spherical-particle species. */
typedef struct kapsel_params {
  int np_xyz[3];       /* grid N = 1 << np per axis, np 4..8 (input.cxx:1392-1397) */
  int eq;              /* KAPSEL_EQ_* */
  int precision;       /* KAPSEL_FP64 or KAPSEL_MIXED */
  int n_particles;     /* Particle_Number (one species) */
  double dx, rho, eta, kbt, alpha_v, alpha_o, dt;
  double a, a_xi;      /* radius and interface thickness in units of DX */
  double mass_ratio;   /* MASS_RATIO of the species */
  double gravity_g;    /* G (gravity.G) */
  int gravity_dir;     /* 0,1,2 for "-X","-Y","-Z" */
  double epsilon;      /* LJ EPSILON */
  int lj_powers;       /* 0: 12:6, 1: 24:12, 2: 36:18 */
  int lj_truncate;     /* 1 ON, 0 OFF, -1 NONE */
  int rotation;        /* switch.ROTATION */
  int fix_cell[3];     /* switch.FIX_CELL.{x,y,z} */
  unsigned int mt_seed;/* MT19937 seed of the thermostat (reference: 0) */
  /* Electrolyte branch (ignored for Navier_Stokes) */
  double dielectric, surface_charge, debye_length;
  double valency_p, valency_n, onsager_p, onsager_n;
  double e_ext[3];
  /* Particles held at their positions and velocities while the hydrodynamic
     force and torque are still measured each step (a resistance
     measurement, as used to generate near-contact training pairs; no
     counterpart in the reference).  0 for the reference dynamics. */
  int frozen;
  /* Shear_Navier_Stokes_Lees_Edwards: Shear_rate of the DC external field
     (constitutive_eq.Shear_Navier_Stokes_Lees_Edwards.External_field.DC,
     input.cxx:634-645); ignored by the other branches. */
  double shear_rate;
  /* Pair searches (LJ forces, the overlap test of the phi/up scatter, the
     near-contact pairs): 0 chooses by particle count (per-step cell and
     neighbour lists above 1024 particles, a scan of all particles below),
     1 always uses the lists, -1 never.  Results do not depend on it. */
  int neighbor_lists;
} kapsel_params;

typedef struct kapsel_ctx kapsel_ctx;

/* Fill p with the reference defaults (input.udf; 64^3, a=5, xi=2, dt=0.01). */
void kapsel_params_default(kapsel_params *p);

/* Create a context on the current CUDA device.  Replaces the allocations of
   Mem_alloc_var (sp_3d_ns.cxx:392-440) and Init_fft (fft_wrapper.cxx:92-101). */
int kapsel_gpu_create(const kapsel_params *p, kapsel_ctx **out);
int kapsel_gpu_destroy(kapsel_ctx *ctx);

/* Particle positions (n*3) and orientations (n*4 quaternions s,v0,v1,v2, or
   NULL for identity) as read by the user_specify initialiser
   (init_particle.cxx:226-288); velocities start at zero (:357-370). */
int kapsel_gpu_set_particles(kapsel_ctx *ctx, const double *x, const double *q);

/* Initial fluid state of main(): Init_zeta_k and the initial rigidity
   projection, then uk_dc = 0 (sp_3d_ns.cxx:508-524). */
int kapsel_gpu_init_state(kapsel_ctx *ctx);

/* n calls of Time_evolution_hydro (sp_3d_ns.cxx:61-212) with
   jikan.time += dt after each (sp_3d_ns.cxx:593-594). */
int kapsel_gpu_step(kapsel_ctx *ctx, int n);

/* As kapsel_gpu_step, but the step sequence is captured once into a CUDA
   graph and replayed (same results). */
int kapsel_gpu_step_graph(kapsel_ctx *ctx, int n);

/* Reduced vorticity zeta[2] in the Ooura layout (2*NX*NY*NZ_ doubles) and
   uk_dc[3]; modes outside the 2/3 box are zero.  (Save_Restart_udf data,
   resume.cxx:10-78.) */
int kapsel_gpu_get_zeta(kapsel_ctx *ctx, double *zeta, double *uk_dc);
int kapsel_gpu_set_zeta(kapsel_ctx *ctx, const double *zeta, const double *uk_dc);

/* Real velocity field u = Zeta_k2u(zeta, uk_dc) (operate_omega.h:124-128)
   of the current state, 3*NX*NY*NZ_ doubles (padding left untouched). */
int kapsel_gpu_get_velocity(kapsel_ctx *ctx, double *u);

/* Particle records, n_particles * KAPSEL_P_STRIDE doubles. */
int kapsel_gpu_get_particles(kapsel_ctx *ctx, double *out);
/* kapsel_gpu_step_graph(ctx, n) followed by kapsel_gpu_get_particles(ctx,
   out) with one host synchronisation instead of two: one pass of the
   reference main loop (sp_3d_ns.cxx:547-594, Output_udf of the particles
   every GTS steps, Time_evolution) with GTS = n.  Same status codes; the
   records are filled also when the status is non-zero. */
int kapsel_gpu_step_graph_particles(kapsel_ctx *ctx, int n, double *out);
int kapsel_gpu_set_particle_state(kapsel_ctx *ctx, const double *in);

/* Restart records.  save writes the state that Save_Restart_udf
   (resume.cxx:10-78, 166-272) records -- zeta over all NX*NY*NZ_ Ooura
   entries, uk_dc, the particles, jikan, and the concentrations in the
   Electrolyte branch -- as `<path> = <value>` text lines with the
   reference's record paths (resume.CONTINUE.Saved_Data.Zeta[i][j][k].zeta0,
   ...Particles[n].R.x, ...jikan.ts, ...).  load reads such a file (lines may
   carry a leading `record <n> `) into an initialised context as
   Force_restore_parameters does (resume.cxx:274-365, 366-512): quaternions
   normalised, x_nopbc reset to x, the step counter continuing after the
   saved jikan.ts, and the thermostat stream seeded afresh and advanced by
   the one step the reference's resumed run takes before it restores. */
int kapsel_gpu_save_restart(kapsel_ctx *ctx, const char *path);
int kapsel_gpu_load_restart(kapsel_ctx *ctx, const char *path);

/* AVS/Express field snapshot of a Navier_Stokes context, as Output_avs
   writes it in its BINARY mode on a uniform field (avs_output.cxx:20-342):
   with init != 0 the header <out_dir>/<out_name>.fld (nstep snapshots) and
   the coordinate file <out_name>.cod are (re)written and <out_dir>/avs is
   created; every call appends the snapshot's description to the .fld file
   and writes <out_dir>/avs/<out_name>_<ts>.dat: float32 columns ux uy uz phi
   pressure tau_xy tau_yz tau_zx tau_xx tau_yy, x fastest.  phi is the
   unclamped profile sum of Make_phi_particle; tau is ETA times the
   symmetric strain rate of the velocity by the spectral formula of
   Zeta_k2Strain_k; the pressure column is zero (the step computes none).
   On an Electrolyte context the snapshot is Output_avs_charge's
   (avs_output.cxx:451-549): columns ux uy uz phi surface_charge rho
   e_potential -- phi and the normalised surface charge density (times
   4 pi a^2) of Make_phi_qq_particle, the ionic charge density (1 - phi)
   sum_n z_n c_n, and the Coulomb potential of the total charge over the
   full spectrum.  Unlike the reference, which transforms its concentrations
   to real space and back in place, the state is not changed.  With
   particles, every call also writes the particle snapshot of Output_avs_p
   (avs_output_p.cxx:13-142), as the main loop does beside it:
   <out_dir>/<out_name>p.fld (header with init) and avs/<out_name>p_<ts>.cod
   / .dat (float32 positions; radius and body axes). */
int kapsel_gpu_write_avs(kapsel_ctx *ctx, const char *out_dir, const char *out_name, int nstep, int init);

/* Time step counter jikan.ts and time jikan.time. */
int kapsel_gpu_get_time(kapsel_ctx *ctx, int *ts, double *time);

/* Grid sizes: dims[0..5] = NX, NY, NZ, NZ_, n_particles, sekibun points. */
int kapsel_gpu_get_dims(kapsel_ctx *ctx, int *dims);

/* External electric field E_ext (operate_electrolyte.cxx:90-177), Electrolyte
   only: the reference reads it from the UDF (input.cxx:743-790); switching it
   mid-run replaces a restart with a new Electric_field. */
int kapsel_gpu_set_efield(kapsel_ctx *ctx, const double *e);

/* Lees-Edwards branch: out[0] = degree_oblique (the strain of the oblique
   grid, input.cxx:271), out[1] = Shear_rate_eff (Calc_shear_rate_eff,
   sp_3d_ns.h:174-196), out[2] = Shear_strain_realized (sp_3d_ns.cxx:600). */
int kapsel_gpu_get_oblique(kapsel_ctx *ctx, double *out);
/* Sets degree_oblique and Shear_rate_eff, as a resumed run restores
   degree_oblique (resume.cxx:333-360).  KAPSEL_EINVAL outside the branch. */
int kapsel_gpu_set_oblique(kapsel_ctx *ctx, double degree_oblique, double shear_rate_eff);

/* Ion concentrations conc_k[2] in the Ooura layout (2*NX*NY*NZ_ doubles;
   the Concentration array of solute_rhs.cxx:16), Electrolyte only. */
int kapsel_gpu_get_concentration(kapsel_ctx *ctx, double *conc);
/* Sets them (the retained 2/3 box is kept; a restored or host-modified
   state, as Force_restore_parameters leaves it, resume.cxx:274-365) and,
   when total_solute is not NULL, the target totals of Rescale_solute
   (Total_solute[2], solute_rhs.cxx:20), which Init_rho_ion computed at the
   start of the run. */
int kapsel_gpu_set_concentration(kapsel_ctx *ctx, const double *conc, const double *total_solute);

/* ---- Batched ensemble of independent boxes. ---- */

/* Many independent boxes of any sizes advanced together, one CUDA graph
   launch per step.  The reference runs each box as its own process (one
   main() per UDF); boxes keep their own parameters, particles and thermostat
   streams.  `boxes` must be initialised contexts at the same time step; the
   batch does not own them.  With autotune != 0 the z- and y-pass variants
   are chosen per box shape by timing whole steps of one box of the shape
   with each variant on a copy of its state (the state is restored). */
typedef struct kapsel_batch kapsel_batch;
int kapsel_batch_create(kapsel_ctx *const *boxes, int n, int autotune, kapsel_batch **out);
int kapsel_batch_step(kapsel_batch *b, int nsteps);
/* Per-box mean-square displacement of the unwrapped positions x_nopbc since
   kapsel_batch_create (the R_raw records of Output_udf, avs_output.cxx:361-363). */
int kapsel_batch_msd(kapsel_batch *b, double *msd);
int kapsel_batch_get_stream(kapsel_batch *b, void **stream);
/* The autotuner's choice per box shape, 6 ints each (up to cap shapes):
   NX, NY, NZ, the z-pass variant (0 warp-level line groups, 1 block-level
   row tiles) and the y-pass variant (0 warp-level, 1 block-level wide kz
   tile, 2 block-level narrow kz tile, 3 warp-level with the inverse y + z
   c2r and the force's z + y passes fused over (component, x) planes held in
   shared memory; 3 needs z variant 0, NY = 32..128 and particles) and the
   radix split of the x transforms (kapsel_gpu_set_x_split); returns the
   number of shapes. */
int kapsel_batch_variants(kapsel_batch *b, int *out, int cap);
/* Radix split of the block-level x transforms of one context: 0 the default
   factorisation of NX into two radix-2 networks, 1 the other one (32 = 4 x 8
   instead of 8 x 4, 64 = 16 x 4 instead of 8 x 8, 128 = 16 x 8 instead of
   8 x 16; NX = 256 has only the default).  Same results to roundoff; the
   batch autotuner times both per box shape.  KAPSEL_EINVAL where NX has no
   other split. */
int kapsel_gpu_set_x_split(kapsel_ctx *ctx, int split);
/* Sets the pass variants (as above) of one Navier_Stokes context; results
   are the same to roundoff, speed differs by shape.  KAPSEL_EINVAL for a
   variant the shape does not allow. */
int kapsel_gpu_set_pass_variant(kapsel_ctx *ctx, int zmode, int ymode);
int kapsel_batch_destroy(kapsel_batch *b);

/* ---- Routine-level entry points on host arrays (reference layouts). ---- */

/* A2a_k / A_k2a (fft_wrapper.h:432-631): in-place forward / inverse 3D real
   FFT of one NX*NY*NZ_ field with the Ooura sign and scaling. */
int kapsel_gpu_A2a_k(kapsel_ctx *ctx, double *a);
int kapsel_gpu_A_k2a(kapsel_ctx *ctx, double *a);

/* Solenoidal_u (operate_omega.h:96-103) on three real NX*NY*NZ_ fields. */
int kapsel_gpu_solenoidal_u(kapsel_ctx *ctx, double *u0, double *u1, double *u2);

/* Make_phi_u_particle (make_phi.cxx:401-409, with the phi>1 clamp of
   :278-297) for the context's particles: phi and up[3] as NX*NY*NZ_ fields. */
int kapsel_gpu_make_phi_u(kapsel_ctx *ctx, double *phi, double *up0, double *up1, double *up2);

/* Calc_f_hydro_correct_precision (md_force.cxx:263-389) for the context's
   particles on the given velocity field; writes f_hydro[n*3], torque[n*3]. */
int kapsel_gpu_calc_f_hydro(kapsel_ctx *ctx, const double *u0, const double *u1, const double *u2,
                            double *f_hydro, double *torque_hydro);

/* Calc_f_Lennard_Jones + Add_f_gravity (particle_solver.h:97-109) for the
   context's particles; writes fr[n*3]. */
int kapsel_gpu_calc_fr(kapsel_ctx *ctx, double *fr);

/* Calc_f_Lennard_Jones_shear_cap_primitive_lnk with the minimum-image
   Distance0 and no cap (md_force.cxx:23-134, md_force.h:75-78): the LJ force
   alone, cell-list pair multiplicity included; writes fr[n*3]. */
int kapsel_gpu_calc_lj(kapsel_ctx *ctx, double *fr);

/* Make_phi_particle (make_phi.cxx:180-219; no phi > 1 clamp) for the
   context's particles: phi as an NX*NY*NZ_ field. */
int kapsel_gpu_make_phi(kapsel_ctx *ctx, double *phi);

/* NS_solver_slavedEuler (fluid_solver.cxx:328-354): the advection term of the
   2/3-truncated zeta (Zeta_k2advection_k, operate_omega.cxx:102-113) and the
   slaved-Euler update of the retained modes, on zeta[2] in the Ooura layout
   (2*NX*NY*NZ_ doubles, updated in place; the modes outside the 2/3 box keep
   their values, as in the reference) with the k=0 velocity uk_dc[3].  The
   context's own fluid state is replaced by the result. */
int kapsel_gpu_ns_slaved_euler(kapsel_ctx *ctx, double *zeta, const double *uk_dc);

/* The Electrolyte routines, on an Electrolyte context whose particle state
   (kapsel_gpu_set_particle_state) gives the positions; concentrations are
   conc_k[2] in the Ooura layout (2*NX*NY*NZ_ doubles, species 0 then 1), as
   the reference's Concentration.  KAPSEL_ESTATE on another kind of context.

   NSsolute_solver_Euler (fluid_solver.cxx:306-326, replaces the call of
   fluid_solver.h:116): Rhs_NS_Nernst_Planck (the potential gradient of the
   charge, the advection term, and per species Diffusion_flux_single,
   Solute_solver_rhs_nonlinear_x_single, Solute_impermeability,
   Add_advection_flux and the flux divergence, solute_rhs.cxx:42-234) and the
   explicit Euler update of zeta and of both concentrations, in place.  As in
   the reference, which truncates zeta and conc_k to the 2/3 box before using
   them, the modes outside the box come back zero; uk_dc is not changed (its
   right-hand side is zero).  The context's own fluid state is replaced. */
int kapsel_gpu_ns_solute_euler(kapsel_ctx *ctx, double *zeta, const double *uk_dc, double *conc_k);

/* Rescale_solute (solute_rhs.cxx:99-128, replaces solute_rhs.h:107): the
   factors total_solute[n] / (DX3 sum (1 - phi) c_n) at the current positions
   into rescale_factor[2], and conc_k scaled by them in place (2/3-truncated
   input, as NSsolute_solver_Euler leaves it; modes outside the box come back
   zero).  The context's own target totals are not changed. */
int kapsel_gpu_rescale_solute(kapsel_ctx *ctx, const double *total_solute, double *conc_k, double *rescale_factor);

/* Make_Coulomb_force_x_on_fluid (operate_electrolyte.cxx:90-177, replaces
   the call of operate_electrolyte.h:78) at the current positions: the force
   density rho_e (-grad psi + E_ext) of the charge field of Conc_k2charge_field
   (operate_electrolyte.cxx:45-74) and conc_k, with the potential of the full
   (untruncated) spectrum, as three NX*NY*NZ_ fields (row padding zero). */
int kapsel_gpu_coulomb_force(kapsel_ctx *ctx, const double *conc_k, double *f0, double *f1, double *f2);

/* MD_solver_position_Euler (euler != 0) / MD_solver_position_AB2
   (particle_solver.cxx:36-88) on the context's particle state (set it with
   kapsel_gpu_set_particle_state, read it with kapsel_gpu_get_particles). */
int kapsel_gpu_md_position(kapsel_ctx *ctx, int euler);

/* MD_solver_velocity_Euler (euler != 0) / MD_solver_velocity_AB2_hydro
   (particle_solver.cxx:106-147, 247-289) on the context's particle state,
   with this step's hydrodynamic force and torque given (the f_hydro and
   torque_hydro that Calc_f_hydro_correct_precision left, n*3 each): Force
   (LJ + gravity), the velocity update and reset_Forces, after which the
   records' f_hydro / torque_hydro / fr hold the step's values (the
   reference's *_previous). */
int kapsel_gpu_md_velocity(kapsel_ctx *ctx, const double *f_hydro, const double *torque_hydro, int euler);

/* Sets the step counter jikan.ts and time jikan.time (a host program that
   attaches a context to a run in progress); the thermostat stream keeps its
   position. */
int kapsel_gpu_set_time(kapsel_ctx *ctx, int ts, double time);

/* Solenoidal_u on three real fields that are already in device memory,
   packed as NX*NY*NZ doubles each (no NZ_ padding), written to three device
   output fields of the same shape, on `stream` (a cudaStream_t; NULL for the
   default stream).  Unlike every other entry point it allocates nothing:
   its spectra and twiddle tables live in one static device array of about
   6.2 MiB (64*64*33 complex values per component plus tables) that each GPU
   loading this library keeps until exit.  It is meant for callers that
   cannot call cudaMalloc (a caller whose device memory is owned by another
   allocator, or one that must not synchronise or fail on allocation in the
   middle of a step).  Grids are powers of two, 16..128 per axis, with
   NX*NY*(NZ/2+1) <= 64*64*33; larger grids return KAPSEL_ERANGE.  The first
   call on a device looks up the array's device address (once per device,
   with that device current); make that first call before any stream
   capture.  All calls share the one array, so calls that overlap on the GPU
   (different streams or threads at the same time) race; serialise them.
   The call is asynchronous on `stream`: its status covers the arguments
   and the launch configuration only (a fault while the kernels run shows
   up at the caller's next synchronising call), and it returns
   KAPSEL_ECUDA without launching anything when an earlier CUDA error is
   still pending on the calling thread (that error is left in place).  No
   counterpart in the reference: it is an addition of this library. */
int kapsel_gpu_solenoidal_u_noalloc(const int *np_xyz, double dx, const double *u0, const double *u1,
                                    const double *u2, double *o0, double *o1, double *o2, void *stream);

/* ---- UDF files (host only, no GPU needed). ----

   KAPSEL reads its input and writes its records through OCTA's UDFManager
   (Gourmet_file_io, input.cxx:438-1818; Output_udf avs_output.cxx:343-450;
   Save_Restart_udf resume.cxx:10-78), which is not part of the reference.
   kapsel_udf_read parses a UDF file without it: the definition blocks
   (\begin{def}, \begin{global_def}, files pulled in by \include) and every
   \begin{data} block, each flattened into one record of `path = value`
   entries with the paths the reference asks for
   (constitutive_eq.Navier_Stokes.DX, object_type.spherical_particle.
   Particle_spec[0].Particle_number, Particles[3].R.x, ...).  An input file
   has one record; an Output_udf file one per snapshot.  Strings returned
   stay valid until kapsel_udf_destroy. */
typedef struct kapsel_udf kapsel_udf;
int kapsel_udf_read(const char *path, kapsel_udf **out);
int kapsel_udf_destroy(kapsel_udf *u);
/* Number of records (data blocks). */
int kapsel_udf_records(const kapsel_udf *u);
/* Number of entries of a record; entry i in file order: its path, its
   value as written (strings without their quotes) and whether it is a
   string (select values are strings). */
int kapsel_udf_size(const kapsel_udf *u, int record);
int kapsel_udf_entry(const kapsel_udf *u, int record, int i, const char **path, const char **text, int *is_string);
/* A numeric or string value by path (KAPSEL_EINVAL when absent). */
int kapsel_udf_get_double(const kapsel_udf *u, int record, const char *path, double *value);
int kapsel_udf_get_string(const kapsel_udf *u, int record, const char *path, const char **text);
/* kapsel_params of an input file (record 0), one spherical-particle
   species: the values Gourmet_file_io reads and the automatic time step of
   Set_global_parameters (input.cxx:316-362).  With user_specify placement
   the positions (n*3) and quaternions (n*4) go to x and q when they are not
   NULL and *n_user is the particle count; otherwise *n_user is 0 (the
   reference places them with rand(): the caller chooses positions).
   KAPSEL_EINVAL for inputs the library does not model. */
int kapsel_udf_to_params(const kapsel_udf *u, int precision, kapsel_params *p, double *x, double *q, int *n_user);

/* ---- Host-only helpers (no GPU needed). ---- */

/* n normals (n even) of the thermostat stream Add_random_force_thermostat
   draws (fluct.cxx:21-35): Gauss2 pairs (fluct.h:48-60) from MT19937 seeded by
   init_genrand(seed) (mt19937ar.c), after skipping `skip` normals. */
int kapsel_thermostat_normals(unsigned int seed, long long skip, long long n, double *out);

/* Sekibun stencil offsets of Particle_domain (profile.cxx:25-74): returns the
   point count; writes 3 ints per point when out != NULL (cap = points room). */
int kapsel_sekibun_cells(double a, double a_xi, double dx, int *out, int cap);

/* ---- Measurement hooks. ---- */

/* Number of kernel launches of one step, counted from a capture of the step
   (nothing is executed); KAPSEL_N_STEP_KERNELS is the number of timing slots
   of kapsel_gpu_profile_step. */
#define KAPSEL_N_STEP_KERNELS 13
int kapsel_gpu_launches_per_step(kapsel_ctx *ctx);
const char *kapsel_gpu_kernel_name(int i);
/* The kernel of timing slot i for this context's pass variants: with the
   fused y/z plane kernels (pass variant y = 3) slot 6 is k_yzw_c2r, slot 10
   k_zyw_force, and slots 5 and 11 are empty ("", no launch). */
const char *kapsel_gpu_step_kernel_name(kapsel_ctx *ctx, int i);

/* The context's CUDA stream (a cudaStream_t), for recording events around
   its work. */
int kapsel_gpu_get_stream(kapsel_ctx *ctx, void **stream);

/* One step with a CUDA event between consecutive launches on the context's
   stream; ms[i] receives the duration of launch i (KAPSEL_N_STEP_KERNELS
   floats).  Advances the state exactly like kapsel_gpu_step(ctx, 1). */
int kapsel_gpu_profile_step(kapsel_ctx *ctx, float *ms);

/* Checks, on the current device, that the library's bounded device waits end
   instead of hanging: a one-block kernel waits on a barrier that nothing
   arrives at, gives up after 0.5 s as the network kernels' waits do, and
   records the timeout.  Returns KAPSEL_ETIMEOUT when that worked (the device
   stays usable), KAPSEL_ECUDA or KAPSEL_ENOMEM otherwise.  No counterpart in
   the reference (it has no device waits). */
int kapsel_gpu_check_bounded_wait(void);

/* Human-readable text of a status code. */
const char *kapsel_gpu_strerror(int status);

/* ---- Learned near-contact correction (no counterpart in the reference;
   the reference's force is the plain SPM momentum exchange of
   Calc_f_hydro_correct_precision, md_force.cxx:263-389). ----

   A 4-layer MLP, 16 -> 128 -> 128 -> 128 -> 16 with SiLU activations, BF16
   weights and activations on the tensor cores (tcgen05, FP32 accumulation),
   predicts the force/torque correction of a close pair of spheres:
   inputs  log(gap/a), v2 - v1, omega1, omega2 in the pair frame (10 values,
           shifted and scaled, zero-padded to 16);
   outputs F1, T1, F2, T2 in the pair frame (12 values, scaled, 4 unused).
   Parameters are one packed FP32 vector of KAPSEL_NC_NPARAM floats:
   W1[128][16] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] W4[16][128] b4[16]
   (W[out][in]).  All buffers below are host memory. */
#define KAPSEL_NC_IN 16
#define KAPSEL_NC_HIDDEN 128
#define KAPSEL_NC_OUT 16
#define KAPSEL_NC_NPARAM 37264

typedef struct kapsel_nc kapsel_nc;

int kapsel_nc_create(const float *params, kapsel_nc **out);
int kapsel_nc_destroy(kapsel_nc *nc);
int kapsel_nc_get_params(kapsel_nc *nc, float *params);
int kapsel_nc_set_params(kapsel_nc *nc, const float *params);

/* y[n][16] = network(x[n][16]). */
int kapsel_nc_forward(kapsel_nc *nc, const float *x, int n, float *y);

/* Gradient of L = (1/n) sum_rows sum_c colw[c] (net(x)[c] - y[c])^2 with
   respect to the packed parameters (grad: KAPSEL_NC_NPARAM floats), and L. */
int kapsel_nc_gradient(kapsel_nc *nc, const float *x, const float *y, const float *colw, int n, float *grad,
                       float *loss);

/* Adam (0.9, 0.999, 1e-8) on minibatches of `batch` rows, `epochs` passes
   over the n samples in MT19937(seed) shuffled order; loss_per_epoch (may be
   NULL) receives the mean minibatch loss of each epoch. */
int kapsel_nc_train(kapsel_nc *nc, const float *x, const float *y, const float *colw, int n, int epochs, int batch,
                    float lr, unsigned int seed, float *loss_per_epoch);

/* Input shift/scale (16 each: feature = (raw - shift) * scale), output
   scale (16: correction = output * scale), the radius a the network was
   trained for, and the trained gap range [gap_lo, gap_hi] in units of a.
   Pairs outside the range keep the plain SPM force. */
int kapsel_nc_set_scaling(kapsel_nc *nc, const float *in_shift, const float *in_scale, const float *out_scale,
                          double a, double gap_lo, double gap_hi);

/* Host evaluation of the network input of one pair of particle records
   (KAPSEL_P_STRIDE doubles each) in a periodic box of side lengths box[3]:
   feat[16], frame[9] (e1, e2, e3; may be NULL), and the surface gap. */
int kapsel_nc_pair_features(const kapsel_nc *nc, const double *rec_i, const double *rec_j, const double *box,
                            float *feat, float *frame, double *gap);

/* Attach a trained, scaled network to a Navier_Stokes context (NULL
   detaches): each step then finds the pairs in the trained gap range after
   the position update, evaluates the network on them and adds the
   corrections to the hydrodynamic force and torque before the velocity
   update.  The network must outlive its use by the context. */
int kapsel_gpu_set_nearcontact(kapsel_ctx *ctx, const kapsel_nc *nc);

/* Number of pairs the last step corrected. */
int kapsel_gpu_nearcontact_pairs(kapsel_ctx *ctx, int *n_pairs);

#ifdef __cplusplus
}
#endif

#endif /* KAPSEL_GPU_H */
