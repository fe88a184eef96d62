/*
 * lesgpu.h -- C ABI of the B200 LES time-step library (liblesgpu.so).
 *
 * Drop-in boundary for the Fortran module entry points of the reference
 * pseudo-spectral ABL LES (fmargairaz/new-repo, src/).  The reference's
 * operators are Fortran subroutines that read and write module-global arrays
 * (system.f90:21-43); here the same arrays live in HBM inside an opaque
 * les_state and every entry point acts on them.  Fields are addressed by
 * les_field ids and moved with les_upload / les_download in the Fortran
 * layout (nx, ny, 0:nz+1), x fastest, as real(8).
 *
 * Every function returns 0 on success or a nonzero status that mirrors the
 * reference's decomp_2d_abort codes (1 invalid option, 3 out of memory,
 * 9 numerical failure, 22 I/O; 4 for other CUDA errors); les_last_error()
 * gives the message.  Calls
 * on one state are not re-entrant; each state owns one CUDA stream (and two
 * copy streams once les_step_host is used).
 */
#ifndef LESGPU_H
#define LESGPU_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (decomp_2d_abort codes of the reference). */
#define LES_OK 0
#define LES_ERR_INVALID 1
#define LES_ERR_NOMEM 3
/* any other CUDA error (no reference counterpart: the reference has no
 * device); les_last_error says whether it is sticky, i.e. a device fault
 * after which the CUDA context is lost */
#define LES_ERR_DEVICE 4
#define LES_ERR_NUMERICAL 9
#define LES_ERR_IO 22

/* sgs_model (compute_sgs.f90:124-175) */
#define LES_SGS_CST_SMAG 0
#define LES_SGS_DYN_SMAG 1
#define LES_SGS_LASD 2
/* learned closure: Cs^2 from the 8 -> 64 -> 64 -> 1 network (no reference
 * counterpart; stands in for the dynamic procedure of compute_sgs.f90:171) */
#define LES_SGS_MLP 3
/* wall_model (compute_wall_law.f90:119-151) */
#define LES_WALL_FILTER 0
#define LES_WALL_INST 1
#define LES_WALL_HOMOG 2
/* dealiasing build option (src/Makefile:16-26) */
#define LES_DEALIAS_PADD 0
#define LES_DEALIAS_TRUNC 1
/* halo of the Lagrangian interpolation */
#define LES_HALO_REFERENCE_1X1 0
#define LES_HALO_PERIODIC 1
/* precision */
#define LES_FP64 0
#define LES_MIXED 1

/* Non-dimensional run parameters, as parameters_IO.f90:238-277 leaves them
 * after read_parameters (lengths divided by zi, lx/ly already times pi). */
typedef struct les_params {
  int nx, ny, nz;
  double dt;
  double lx, ly, lz;
  double z0;        /* lbc_dz0 / zi (set_bc_surface) */
  double pfx, pfy;  /* mean pressure-gradient forcing */
  double cs0;       /* constant Smagorinsky coefficient */
  int sgs_model;
  int cs_count, dyn_init;
  int wall_law;     /* lbc_special == 'wall_law' */
  int wall_model;
  int dealias;
  int lag_halo;
  int precision;
  int device;
} les_params;

/* Field ids: the global arrays of system.f90:21-43 and the SGS module state
 * (compute_sgs.f90:31, compute_LagScaleDep.f90:33-36).  All are stored as
 * (nx, ny, 0:nz+1); arrays the reference dimensions (nx,ny,nz) or
 * (nx,ny,nz+1) use levels 1..nz or 1..nz+1 of that storage. */
typedef enum les_field {
  LES_U = 0, LES_V, LES_W,
  LES_DUDX, LES_DUDY, LES_DUDZ, LES_DVDX, LES_DVDY, LES_DVDZ, LES_DWDX, LES_DWDY, LES_DWDZ,
  LES_P, LES_DPDX, LES_DPDY, LES_DPDZ,
  LES_RHSX, LES_RHSY, LES_RHSZ, LES_RHSX_F, LES_RHSY_F, LES_RHSZ_F,
  LES_TXX, LES_TXY, LES_TXZ, LES_TYY, LES_TYZ, LES_TZZ,
  LES_CS_OPT2, LES_NU_T,
  LES_F_LM, LES_F_MM, LES_F_QN, LES_F_NN, LES_BETA,
  LES_U_LAG, LES_V_LAG, LES_W_LAG,
  /* scalar transport (allocated by les_scalar_init): theta on uvp nodes,
   * its gradients (d/dz on w nodes), right-hand sides and SGS fluxes
   * pi_j = nu_theta d_j theta (pi_x, pi_y on uvp nodes, pi_z on w nodes) */
  LES_THETA, LES_DTDX, LES_DTDY, LES_DTDZ, LES_RHS_T, LES_RHS_T_F, LES_QX, LES_QY, LES_QZ,
  LES_NFIELDS
} les_field;

/* Plane ids (nx, ny): boundary values, pressure-BC layers, roughness, u*. */
typedef enum les_plane {
  LES_LBC_U = 0, LES_LBC_V, LES_LBC_W, LES_UBC_U, LES_UBC_V, LES_UBC_W,
  LES_BOTTOM_WK_PRESS, LES_TOP_WK_PRESS, LES_LBC_Z0, LES_U_STAR_AVG,
  LES_NPLANES
} les_plane;

typedef struct les_state les_state;

/* --- lifetime (replaces create_system system.f90:66, the *_init routines
 *     LES_engine.f90:130-153 and clean_system system.f90:214) ----------- */
int les_create(const les_params* p, les_state** out);
int les_destroy(les_state* s);
const char* les_last_error(void);

/* --- data movement: host pointers are borrowed for the call ------------ */
/* levels k0..k1 (inclusive) of field id, host array (nx, ny, k1-k0+1) */
int les_upload(les_state* s, int field, const double* host, int k0, int k1);
int les_download(les_state* s, int field, double* host, int k0, int k1);
int les_upload_plane(les_state* s, int plane, const double* host);
int les_download_plane(les_state* s, int plane, double* host);
/* Initial state: the ic_type='files' path (initial_conditions.f90:130-212):
 * u, v, w as (nx, ny, nz) arrays, then the initial boundary conditions. */
int les_set_initial_conditions(les_state* s, const double* u, const double* v, const double* w);
/* Boundary-condition types of set_bc (0 none, 1 'drc', 2 'neu') for u,v,w. */
int les_set_bc_types(les_state* s, const int lbc_typ[3], const int ubc_typ[3]);
/* Flags of the Lagrangian model: F_coeff_init and Lagran_init
 * (compute_LagScaleDep.f90:31,66,288). */
int les_set_lagrangian_init(les_state* s, int f_coeff_init);
int les_get_lagrangian_init(les_state* s, int* f_coeff_init);

/* Switch an existing state between LES_FP64 and LES_MIXED (the precision
 * chosen at creation): every field and plane, the boundary-condition types
 * and the Lagrangian flags move to a new state of the other precision (FP32
 * fields round to nearest; statistics sums and profiles restart).  Refused
 * (1) while the learned closure is the SGS model: its normalisation and
 * training data belong to the state it was trained in.  Replaces the
 * les_set_precision(mode) of the boundary; the reference runs in FP64 only. */
int les_set_precision(les_state* s, int precision);

/* --- module entry points ------------------------------------------------ */
/* compute_derivatives.f90:94-137 grad_velocity_filt(f, dfdx, dfdy) */
int les_grad_velocity_filt(les_state* s, int f, int dfdx, int dfdy);
/* compute_derivatives.f90:375-400 ddz_uv(dfdz, f) */
int les_ddz_uv(les_state* s, int dfdz, int f);
/* compute_derivatives.f90:413-441 ddz_w(dfdz, f) */
int les_ddz_w(les_state* s, int dfdz, int f);
/* compute_derivatives.f90:464-577 div_stress(rhs, tx, ty, tz, stag[, bottom, top]);
 * with stag == 0 the bottom_wk_press/top_wk_press planes are written. */
int les_div_stress(les_state* s, int rhs, int tx, int ty, int tz, int stag);
/* compute_convective_padd.f90:115-262 / compute_convective_trunc.f90:115-235
 * compute_dealias_convec(cx, cy, cz) */
int les_compute_dealias_convec(les_state* s, int cx, int cy, int cz);
/* compute_pressure.f90:116-242 press_stag_array(tadv1) */
int les_press_stag_array(les_state* s, double tadv1);
/* compute_pressure.f90:116-242 press_stag_array(tadv1) in increment form,
 * for the state les_ab2_advance(tadv1, tadv2) just left: u* / (dt tadv1) =
 * u^n / (dt tadv1) + rhs + (tadv2/tadv1) rhs_f, whose divergence is formed
 * from this step's dudx + dvdy + dwdz (les_compute_vel_grad before the
 * advance) and the transforms of rhs, rhs_f; the same pressure in exact
 * arithmetic, without the cancellation of transforming u* (values ~ u
 * against increments ~ dt rhs), so the transforms run in the state's
 * precision (the kx = ky = 0 column from FP64 plane means).  les_step keeps
 * the reference's formulation.  Preconditions: rhs, rhs_f and the gradients
 * unchanged since the advance, w(nz+1) = 0. */
int les_press_from_increment(les_state* s, double tadv1, double tadv2);
/* z-slab decomposition of the pressure solve, emulated on this GPU: with
 * nslabs > 1 the tridiagonal systems of press_stag_array (and of les_step)
 * are solved by the partition method over nslabs blocks of rows, the blocks
 * a z-slab rank holding levels b nz/G + 1 .. (b+1) nz/G would own: each
 * block eliminates its rows with the right-hand side and the two unit
 * couplings to its neighbours, the 2 nslabs boundary unknowns of every
 * (kx, ky) column solve a 2 x 2 block-tridiagonal system, and each block
 * back-substitutes.  Replaces the Y <-> Z transposes around
 * tridiag_solver_parallel (compute_pressure.f90:265,290) of the reference's
 * pencil decomposition; the same solution up to rounding.  nslabs = 1 (the
 * default) is the single sweep.  Errors: 1 unless 1 <= nslabs <= 64 and nz
 * is a multiple of nslabs with at least two levels per slab. */
int les_set_pressure_slabs(les_state* s, int nslabs);
/* compute_wall_law.f90:198-254 obukhov(u_star_avg, wl_type) */
int les_obukhov(les_state* s);
/* compute_wall_law.f90:107-185 wallstress(lbc_u, lbc_v, wl_type) */
int les_wallstress(les_state* s);
/* The wl_type argument of obukhov / wallstress: the wall model (LES_WALL_*)
 * that they and les_step use from now on (les_params.wall_model at
 * creation). */
int les_set_wall_model(les_state* s, int wall_model);
/* compute_sgs.f90:105-247 sgs_stress(jt, jtt) */
int les_sgs_stress(les_state* s, int jt, int jtt);
/* testfilter.f90:144-184 test_filter(f, G) on levels 1..nz+1;
 * which = 2 for G_test (2 Delta), 4 for G_test_test (4 Delta). */
int les_test_filter(les_state* s, int f, int which);
/* boundary_condition_mpi.f90:33-63 set_bc for u, v, w at bottom and top */
int les_set_bc(les_state* s);
/* LES_engine.f90:449-498 compute_vel_grad() */
int les_compute_vel_grad(les_state* s);
/* LES_engine.f90:509-572 compute_RHS_adv() */
int les_compute_rhs_adv(les_state* s);
/* LES_engine.f90:262-283 Adams-Bashforth advance and w(0)=w(nz+1)=0 */
int les_ab2_advance(les_state* s, double tadv1, double tadv2);
/* LES_engine.f90:300-331 projection, rhs update, w(1)=w(nz+1)=0 */
int les_projection(les_state* s, double tadv1);
/* LES_engine.f90:189-360: one whole time step (wall law .. BCs and the
 * running diagnostics).  jt is the loop counter, jt_total the global step. */
int les_step(les_state* s, int jt, int jt_total);
/* running_diagnostics.f90:80-136 of the last step: cfl, mke, u_star, rms div u
 * (FP64, compensated sums). */
int les_diagnostics(les_state* s, double out[4]);
/* Sticky device status bits, cleared on read: 1 NaN in the velocity, 2 zero
 * pivot in the tridiagonal solve, 4 closure inputs outside the training range,
 * 8 kernel argument check failed, 16 a closure kernel's tensor-core wait ran
 * out, 32 a spectral pass's bulk-copy wait ran out (the pass left its CTA's
 * work undone). */
int les_get_status(les_state* s, unsigned* bits);
/* The reference's numerical aborts as a status: check_NaN(jt)
 * (LES_engine.f90:583-616, called every NaN_check steps, :363-365) and the
 * zero-pivot abort of the tridiagonal solve (compute_pressure.f90:411-418),
 * both decomp_2d_abort code 9.  Synchronises the state's stream, reads and
 * clears the status bits (into *bits, may be NULL) and returns
 * LES_ERR_NUMERICAL with the reference's message ("I got a NaN" /
 * "tridiag solver: error bet(i,j)=0, dividing by 0!") when the NaN or pivot
 * bit was set since the last read, else 0.  The state stays usable: a caller
 * can reload a checkpoint (les_checkpoint_read) and continue. */
int les_check_status(les_state* s, unsigned* bits);
/* Synchronise the state's stream. */
int les_sync(les_state* s);
/* Device time of the kernels of the last les_step, per reference profiling
 * bucket (LES_engine.f90:100-107): grad, stress, rhs, press, loop (ms). */
int les_timers(les_state* s, double out[5]);

/* --- measurement (replaces the mpi_wtime timers of LES_engine.f90:100-107,
 *     428-435 with device-side events) ------------------------------------ */
/* Per-launch profiling: with enable != 0 every kernel launch is bracketed by
 * CUDA events on the state's stream.  les_profile_report writes a JSON object
 * {"<operator>/<kernel>": {"launches", "ms", "bytes_per_launch"}, ...} where
 * bytes_per_launch is the launch's algorithmic traffic (inputs read once,
 * outputs written once). */
int les_profile(les_state* s, int enable);
int les_profile_report(les_state* s, char* buf, int buflen);
/* Number of kernels launched on this state since creation. */
int les_launch_count(les_state* s, long long* n);
/* Record timing event slot (0..15) on the state's stream / elapsed ms b - a. */
int les_event_record(les_state* s, int slot);
int les_event_elapsed(les_state* s, int a, int b, double* ms);
/* Asynchronous FP64 transfers from/to page-locked host memory on the state's
 * stream (converted on the device in mixed precision); les_sync completes
 * them. */
int les_upload_async(les_state* s, int field, const double* pinned, int k0, int k1);
int les_download_async(les_state* s, int field, double* pinned, int k0, int k1);
int les_diagnostics_async(les_state* s, double* pinned_out4);
/* One time step of the LES_engine.f90:189-360 loop body with the velocity
 * state held in host memory, as a caller whose arrays stay authoritative
 * (the reference's u, v, w of system.f90:21-43) would step it: copies
 * u, v, w (FP64, levels 0..nz+1, the les_upload layout) to the device,
 * runs les_step(jt, jt_total), and copies the new u, v, w and the step's
 * four diagnostics (les_diagnostics order; diag_out4 may be NULL) back into
 * the same arrays.  Asynchronous: the call returns once the work is queued,
 * and the arrays must be neither read nor written until les_sync (or any
 * other entry point, which orders itself after these copies).  Successive
 * calls overlap the copies back of one step with the copies in of the next,
 * per chunk of levels, one in each direction of the host link; page-locked
 * arrays are needed for that overlap (pageable ones work, serialised). */
int les_step_host(les_state* s, int jt, int jt_total, double* u, double* v, double* w, double* diag_out4);
/* Page-lock (and release) caller-allocated host memory, e.g. the Fortran
 * u, v, w handed to les_step_host, so that its copies can overlap. */
int les_host_register(void* p, size_t bytes);
int les_host_unregister(void* p);

/* Checkpoint file of write_checkpoint_file / read_checkpoint_file
 * (IO_checkpoint.f90:119-256) on one rank, byte for byte: native FP64
 * records of nx*ny*(nz+1) values (levels 1..nz+1, x fastest) for u, v, w,
 * rhsx, rhsy, rhsz, cs_opt2 and, when the Lagrangian averages exist
 * (Lagran_init), F_LM, F_MM, F_QN, F_NN.  Reading with lagran_init = 1 also
 * sets the Lagrangian-init flag (compute_LagScaleDep.f90:66); the Lagrangian
 * accumulators restart at zero, w(0) takes its allocation value and the
 * wall law sets the lower u, v conditions to Neumann (LES_engine.f90:160-171).  Errors: 1 cannot open / short file (the
 * reference aborts with 1), 22 read or write failure. */
int les_checkpoint_write(les_state* s, const char* path);
int les_checkpoint_read(les_state* s, const char* path, int lagran_init);

/* ---- post-step statistics (one rank) ------------------------------------
 * Running sums of IO_statistics.f90.  les_stat_init replaces io_stat_init
 * (:40-250): it allocates (or zeroes) 26 FP64 volumes of nx*ny*nz and one
 * u* plane.  les_stat_averages replaces io_stat_averages(jt, jt_total)
 * (:265-291 with io_2D_stat_averages :300-354 and io_3D_stat_averages
 * :363-518): it adds the current state to the sums and, when
 * mod(jt_total, running_period) == 0 and jt_total > start_stats, writes
 * <out_path>RAV_<jt_total:09>_info.txt ("%6d%6d%6d%10d": nx, ny, nz,
 * iterations), _2D.dat (the u* sum, nx*ny FP64) and _3D.dat (the 26 sums in
 * the order u v w p u2 v2 w2 u3 v3 w3 u4 v4 w4 uv uw vw txx tyy tzz txy txz
 * tyz dudz dvdz nu_t cs, nx*ny*nz FP64 each, x fastest), then restarts the
 * sums.  out_path is prefixed as is (the reference's trim(out_path)).  The
 * caller applies the driver's condition stat_flag .and. jt_total >
 * start_stats (LES_engine.f90:368-370).  les_stat_sums copies sum index
 * 0..25 (nx*ny*nz values) or 26 (the u* plane) to the host.
 * les_stat_spectra replaces io_stat_spectra (:566-620): inside the four
 * fixed jt_total windows and every 10th jt it writes
 * <out_path>SP_<jt_total:09>.dat with u, v, w on levels 1..nz.
 * Errors: 1 not initialised / invalid period, 22 file open or write. */
int les_stat_init(les_state* s);
int les_stat_averages(les_state* s, int jt, int jt_total, int start_stats, int running_period, const char* out_path);
int les_stat_sums(les_state* s, int index, double* out);
int les_stat_iterations(les_state* s, int* out);
int les_stat_spectra(les_state* s, int jt, int jt_total, const char* out_path);

/* Plane-averaged TKE budget of tke_budget1D.f90.  les_tke_init replaces
 * tke_budget_init (:61-160): it creates <out_path>ta1_profiles/ (an existing
 * folder is fine) and zeroes 61 FP64 profiles of nz levels; the record
 * counter starts at 1.  les_tke_budget replaces compute_tke_budget(jt)
 * (:209-390): it adds the plane averages of the 61 quantities (names and
 * order of its avg_var calls: u v w dudx dudy dudz dvdx dvdy dvdz dwdx dwdy
 * dwdz uu vv ww uv uw vw txx tyy tzz txy txz tyz cs uuw vvw www uww wtzz
 * utxz vtyz dxx dyy dzz dxy dxz dyz dudx2 dudy2 dudz2 dvdx2 dvdy2 dvdz2 dwdx2
 * dwdy2 dwdz2 dudxdwdx dudydwdy dudzdwdz p dpdx dpdy dpdz pw pu pdudx pdvdy
 * pdwdz pdwdx pdudz) and, when mod(jt, tke_period) == 0, writes record ii
 * (nz FP64 values at byte offset (ii-1)*8*nz: direct access with recl = 2*nz
 * in 4-byte units) of ta1_profiles/<name>.out holding profile / tke_period,
 * then restarts the profiles and advances ii.  The caller applies
 * tke_flag .and. jt_total > start_tke (LES_engine.f90:377-380).
 * les_tke_sums copies the 61 x nz profiles (name-major) and the next record
 * number.  Errors: 1 not initialised / invalid period, 22 file open or write. */
int les_tke_init(les_state* s, const char* out_path);
int les_tke_budget(les_state* s, int jt, int tke_period);
int les_tke_sums(les_state* s, double* out, int* record);

/* ---- scalar transport, buoyancy and momentum forcing ---------------------
 * The reference's scalar module is a stub (compute_scalars.f90:80-151: the
 * AB2 update of step_scalars and its ghost values only) and its sponge layer
 * is built, zeroed and disconnected (sponge_damping.f90:83,
 * LES_engine.f90:565).  Here theta (uvp nodes, stored as the departure from
 * a reference value) is advected with the momentum's 3/2-padded (or 2/3
 * truncated) products, -(u d_x + v d_y) theta - (w d_z theta at k, k+1)/2,
 * diffuses with the SGS flux pi_j = nu_theta d_j theta (rhs += div pi, the
 * sign convention of the reference's stresses) and steps with AB2
 * (step_scalars :111-125).  nu_theta = nu_t / pr_t (LES_SCALAR_SGS_CONST) or
 * |S| kappa(z) Delta^2 with kappa = Cs^2/Pr_t from the plane-averaged
 * Germano identity at the 2 Delta test filter (LES_SCALAR_SGS_DYN: the
 * dynamic Prandtl model, K_j = filt(u_j theta) - filt(u_j) filt(theta),
 * X_j = Delta^2 (filt(|S| d_j theta) - 4 |S~| d_j theta~), kappa =
 * max(0, <K.X>/<X.X>), updated every cs_count steps from dyn_init, 0.03/pr_t
 * before), on the nodes of compute_dynamic_mum.  Boundary conditions: the
 * wall flux pi_z(1) = -surface_flux and d theta/dz(1) = -surface_flux /
 * (kappa_vk u* dz/2) (0 where u* = 0), theta(0) = 0 (step_scalars), theta(nz+1)
 * = theta(nz) + top_gradient dz.  With buoyancy != 0 (g/theta_0) the w
 * equation gains buoyancy (theta_w - <theta_w>) on w nodes 2..nz, theta_w
 * the mean of the two uvp levels around the node (the stub's
 * compute_beta_scalars, :143-148). */
#define LES_SCALAR_SGS_CONST 0
#define LES_SCALAR_SGS_DYN 1
typedef struct les_scalar_params {
  double surface_flux;  /* kinematic flux at the wall, positive upward */
  double top_gradient;  /* d theta / dz at the lid */
  double buoyancy;      /* g / theta_0 in model units; 0 = passive scalar */
  double pr_t;          /* turbulent Prandtl number (constant model; initial kappa = 0.03 / pr_t) */
  int sgs;              /* LES_SCALAR_SGS_CONST or LES_SCALAR_SGS_DYN */
} les_scalar_params;
/* scalars_module_init (compute_scalars.f90:40-57): allocates the scalar
 * fields (zero) and turns the scalar on for les_step. */
int les_scalar_init(les_state* s, const les_scalar_params* sp);
/* theta (nx, ny, nz) of levels 1..nz, then the ghost values */
int les_scalar_set_initial(les_state* s, const double* theta);
/* kappa = Cs^2 / Pr_t per level 0..nz+1 (out[nz+2]) of the scalar SGS model */
int les_scalar_kappa(les_state* s, double* out, int n);
/* sponge_damping_init (sponge_damping.f90:42-101) with the layer fraction of
 * the domain height below the sponge (0.8: the top 20 %) and without the
 * zeroing of :83; add_sponge_damping (:131-161) then runs at the end of
 * compute_RHS_adv (the call LES_engine.f90:565 leaves commented out).
 * fraction <= 0 turns it off. */
int les_sponge_init(les_state* s, double layer_fraction);
/* Optional upper bound on the dynamic SGS coefficient Cs^2 of the LASD update,
 * the plane-averaged dynamic Smagorinsky model and the learned closure
 * (0, the default, applies none: the reference has no upper clip,
 * compute_LagScaleDep.f90:651-707).  A stabiliser for grids whose lid
 * region is nearly laminar: there the Lagrangian averages' ratio
 * F_LM/F_MM of tiny test-filtered strains can grow without bound and the
 * explicit SGS diffusion then loses stability (seen at 512 x 512 x 256 from
 * the synthetic initial field within ~100 steps). */
int les_set_cs2_max(les_state* s, double cs2_max);
/* Coriolis forcing of compute_RHS_adv (LES_engine.f90:553-561): rhs_x +=
 * coriol (v - v_g), rhs_y -= coriol (u - u_g); coriol = 0 turns it off. */
int les_set_coriolis(les_state* s, double coriol, double ug, double vg);

/* ---- learned SGS closure (no reference counterpart) ---------------------
 * Cs^2 = Cs^2_prev * exp(net(features)) from an 8 -> 64 -> 64 -> 1 GELU network with
 * BF16 weights and FP32 accumulation (tcgen05 tensor cores), evaluated at
 * the dynamic-update cadence of compute_sgs.f90:171 (every cs_count steps
 * after dyn_init).  Training data are (invariants, log Cs^2) pairs of the
 * Lagrangian scale-dependent procedure (LASD, compute_sgs.f90:286) collected
 * from a running state.  Features: log1p |S|, log1p S:S, log1p W:W, signed
 * log1p tr(S^3), log1p(z / Delta), log Cs^2 before the update (the memory
 * the Lagrangian averages carry), signed log1p of the vortex stretching
 * w_i S_ij w_j, log(Delta / z0).  Columns
 * whose features leave the training range take one Lagrangian relaxation
 * step of the dynamic procedure from the previous coefficient; every
 * `check_every` updates that step also runs on the whole domain and the RMS
 * of log Cs^2 - log Cs^2_dyn is recorded.
 * Parameters: float[LES_MLP_NPARAM + LES_MLP_NSTATS] = W1[8][64], b1[64],
 * W2[64][64], b2[64], w3[64], b3, then feature mean[8], std[8],
 * min[8], max[8] (normalised units), target mean, target std, target
 * min, max (normalised units; the output is clamped to them). */
#define LES_MLP_NPARAM 4801
#define LES_MLP_NSTATS 36
int les_set_sgs_model(les_state* s, int model);
int les_mlp_init(les_state* s, unsigned seed);
int les_mlp_set_params(les_state* s, const float* params, int n);
int les_mlp_get_params(les_state* s, float* params, int n);
/* (re)allocate room for `cap` training and `cap` validation samples, empty */
int les_mlp_reset_data(les_state* s, long cap);
/* append the current state's (features, log cs_opt2) pairs, one point in
 * `stride` (seeded hash) and every point of levels 1..dense_levels, 10 % of
 * them to the validation set, the training pairs of levels 1 and 2
 * wall_repeat (1..16) times; pairs beyond the capacity are dropped.  Call
 * it right after consecutive dynamic-update steps: the previous coefficient
 * of a pair is the one the previous call saw (the first call only records
 * it). */
int les_mlp_collect(les_state* s, int stride, int dense_levels, int wall_repeat, unsigned seed);
int les_mlp_counts(les_state* s, long long out2[2]);
/* feature/target statistics of the collected data; normalises it in place */
int les_mlp_fit_stats(les_state* s);
/* Adam on the mean squared error in normalised log Cs^2; batches of
 * 128 * tiles_per_step samples; loss_epochs[epochs] (may be NULL) gets the
 * last batch loss of each epoch, val_loss the validation loss (or -1) */
int les_mlp_train(les_state* s, int epochs, int tiles_per_step, double lr, double* loss_epochs,
                  double* val_loss);
/* network output (normalised units) for n host feature rows x[n][8] */
int les_mlp_forward(les_state* s, const float* x, long n, float* y);
/* gradient of mean((y - t)^2) over n host rows into grad[LES_MLP_NPARAM] */
int les_mlp_grad(les_state* s, const float* x, const float* t, long n, float* grad, float* loss);
/* out12: last check's RMS log error (-1 if none), flagged columns of the
 * last update, number of updates, weights loaded (1/0), then for each of the
 * 8 features the columns where it left the training range at the last update */
int les_mlp_info(les_state* s, double out12[12]);
/* dynamic-procedure check every `every` closure updates (0 = never) */
int les_mlp_set_check_every(les_state* s, int every);
/* levels 1..nlev next to the wall keep the plain LASD procedure (with its
 * Lagrangian averages) under the learned closure; 0 (default) = none */
int les_mlp_set_wall_levels(les_state* s, int nlev);
/* per level 1..nz+1 (out[0..nz]), the RMS of log Cs^2 - log Cs^2_dyn at the
 * last check (-1 before the first); n >= nz + 1 */
int les_mlp_check_profile(les_state* s, double* out, int n);

/* ---- allocation-free variant (no reference counterpart) ----------------
 * The horizontal derivatives of les_grad_velocity_filt (the ddx/ddy of
 * compute_derivatives.f90 on one field) for a field already on the device:
 * f [nlev][ny][nx] (FP64) is replaced by its Nyquist-filtered version and
 * dfdx, dfdy receive the derivatives (domain lengths lx, ly); the three
 * pointers must be 16-byte aligned (rejected otherwise).  nx is one of
 * 16 24 32 48 64 96 128 192 256 384 512 768 and ny one of 16 32 64 128 256
 * 512 (other sizes are rejected before anything is queued).  Its kernel
 * launches are not counted by les_profile / les_launch_count of a state used
 * on the calling thread (the launch observer is per host thread and is
 * suspended for the duration of the call only).  It allocates
 * nothing: the tables and spectra live in one static device buffer of
 * LES_NOALLOC_SCRATCH_BYTES, for callers that must not change the device
 * memory footprint (an in-situ hook in a coupled run whose memory is fully
 * committed, a process whose free memory a caching allocator holds).
 * Sizes needing more scratch than the buffer are rejected (LES_ERR_INVALID,
 * message in les_noalloc_last_error).  The first call on a device looks up
 * the buffer's address and sets kernel attributes; make it before any stream
 * capture.  All calls share the buffer of their device: calls in flight at
 * the same time on one device race.  Asynchronous on `stream` (a
 * cudaStream_t; NULL is the default stream). */
#define LES_NOALLOC_SCRATCH_BYTES (32u << 20)
int les_grad_xy_noalloc(double* f, double* dfdx, double* dfdy, int nx, int ny, int nlev, double lx, double ly,
                        void* stream);
const char* les_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* LESGPU_H */
