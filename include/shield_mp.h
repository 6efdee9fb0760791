/*
 * shield_mp.h -- C-ABI of the B200 GFDL cloud-microphysics step and its
 * physics-to-dynamics column coupling (libshield_mp.so).
 *
 * pySHiELD has no native FFI: its interface is the Python object API. Each
 * entry point below replaces one call of that API:
 *
 *   shield_mp_create   Microphysics.__init__(stencil_factory, quantity_factory,
 *                      grid_data, namelist)     pySHiELD/stencils/microphysics.py:1624-1804
 *   shield_mp_step     Microphysics.__call__(state, timestep)
 *                                                pySHiELD/stencils/microphysics.py:1981-2263
 *   shield_physics_prestep
 *                      Physics.__call__ before the microphysics:
 *                      atmos_phys_driver_statein, get_prs_fv3, get_phi_fv3,
 *                      prepare_microphysics  pySHiELD/stencils/physics.py:26-143, 276-330;
 *                                            get_prs_fv3.py:7-20; get_phi_fv3.py:7-25
 *   shield_physics_prestep_from_dycore
 *                      DycoreToPhysics.__call__ then the pre-steps above, fused
 *   shield_copy_dycore_to_physics
 *                      DycoreToPhysics.__call__ (without the dry convective
 *                      adjustment)              pySHiELD/update/update_atmos_state.py:95-232
 *   shield_agrid_to_dgrid
 *                      AGrid2DGridPhysics.__call__(u, v, u_dt, v_dt)
 *                                                pySHiELD/update/update_dwind_phys.py:12-161, 490-701
 *   shield_update_physics_state
 *                      update_physics_state_with_tendencies
 *                                                pySHiELD/stencils/physics.py:151-194
 *   shield_update_atmos_state
 *                      UpdateAtmosphereState.__call__ column stencils:
 *                      fill_gfs_delp, prepare_tendencies_and_update_tracers
 *                                                pySHiELD/update/update_atmos_state.py:21-92, 301-349
 *                      and ApplyPhysicsToDycore's moist_cv and
 *                      update_pressure_and_surface_winds
 *                                                pySHiELD/update/fv_update_phys.py:32-75, 152-188
 *
 * Conventions
 *  - All arrays are device pointers to double. A 3-D field is described by
 *    the address of its compute-domain origin and element strides (i, j, k);
 *    any layout works, i-fastest (GPU storage) and k-fastest (C-order numpy
 *    storage) layouts are both read with coalesced loads. k = 0 is the model
 *    top. Column c of a (nx, ny) domain is (i, j) = (c % nx, c / nx).
 *  - Return codes: 0 on success, negative on error (see SHIELD_E*); the
 *    message is kept per handle (shield_mp_last_error) or per thread
 *    (shield_last_error for the handle-free calls). Nothing throws across the
 *    ABI. There is no CPU fallback: without a usable CUDA device every call
 *    fails with SHIELD_ECUDA.
 *  - Work is enqueued on the given CUDA stream (NULL = legacy default stream)
 *    and is asynchronous with respect to the host.
 *  - A handle is not thread safe; use one handle per host thread.
 */
#ifndef SHIELD_MP_H
#define SHIELD_MP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SHIELD_OK 0
#define SHIELD_EINVAL (-1)   /* bad argument (null pointer, size, timestep) */
#define SHIELD_ELAYOUT (-2)  /* unsupported size or layout */
#define SHIELD_ECUDA (-3)    /* CUDA runtime error (launch, allocation, device) */
#define SHIELD_EDEVICE (-4)  /* the kernel flagged a bad value */

/* precision modes of shield_mp_step */
#define SHIELD_MP_PLAIN 0 /* everything in FP64 */
#define SHIELD_MP_MIXED 1 /* process rates in FP32, saturation adjustment, fall and budgets in FP64 */

/* The PhysicsConfig fields the microphysics path reads
 * (pySHiELD/_config.py:22-109, same names and meaning; booleans as int). */
typedef struct {
  double dt_atmos;
  int hydrostatic;
  int do_qa;
  double c_cracw, c_paut, c_pgacs, c_psaci, ccn_l, ccn_o;
  int const_vg, const_vi, const_vr, const_vs;
  double vs_fac, vg_fac, vi_fac, vr_fac;
  int de_ice;
  double tau_imlt, tau_i2s, tau_g2v, tau_v2g, ql_mlt, qs_mlt, t_sub, qi_gen, qi_lim, qi0_max;
  int rad_snow, rad_rain;
  double dw_ocean, dw_land, tau_l2v;
  int do_sedi_heat, do_sedi_w, fast_sat_adj;
  double qc_crt;
  int fix_negative, irain_f;
  double mp_time;
  int prog_ccn;
  double qi0_crt, qs0_crt, rh_inc, rh_inr, rthresh;
  int sedi_transport, use_ppm;
  double vg_max, vi_max, vr_max, vs_max;
  int z_slope_ice, z_slope_liq;
  double tice, alin, clin;
} ShieldMpConfig;

typedef struct {
  double* ptr; /* address of element (i, j, k) = (0, 0, 0) of the compute domain */
  int64_t si, sj, sk;
} ShieldField3D;

typedef struct {
  const double* ptr;
  int64_t si, sj;
} ShieldField2D;

/* MicrophysicsState (pySHiELD/stencils/microphysics.py:1556-1620) as
 * pointers. Inputs: the 13 state fields and land. In/out: the ten
 * tendencies (accumulated, as the reference does), wmp (updated when
 * do_sedi_w holds and hydrostatic does not) and, with de_ice, qice/qsnow.
 * Outputs: the surface precipitation totals of the step in mm/day, ncol
 * contiguous doubles each (column c = j*nx + i); any of them may be NULL. */
typedef struct {
  ShieldField3D pt, qvapor, qliquid, qrain, qice, qsnow, qgraupel, qcld, ua, va, delprsi, delz, wmp;
  ShieldField3D pt_dt, qv_dt, ql_dt, qr_dt, qi_dt, qs_dt, qg_dt, qa_dt, udt, vdt;
  ShieldField2D land;
  double *rain, *snow, *ice, *graupel;
} ShieldMpFields;

/* Microphysics.__init__: computes the process constants (setupm) and the
 * sub-step for cfg->dt_atmos, copies grid_data.area (nx*ny cells, strides
 * in elements) and allocates the persistent cloud-fraction accumulator
 * (the reference's never-reset self._qaz, zero at construction). */
int shield_mp_create(const ShieldMpConfig* cfg, int nx, int ny, int nz, ShieldField2D area, void** handle);

/* Microphysics.__call__(state, timestep): one full step. A timestep that
 * differs from the previous one recomputes the sub-step (_set_timestep). */
int shield_mp_step(void* handle, const ShieldMpFields* fields, double timestep, int precision, void* stream);

int shield_mp_destroy(void* handle);

/* Copies the handle's last error message (NUL terminated) into buf. */
int shield_mp_last_error(void* handle, char* buf, size_t n);

/* ---------------------------------------------------------------------------
 * Adjoint of the step. pySHiELD has no adjoint; this is the vector-Jacobian
 * product (VJP) of one Microphysics.__call__ (microphysics.py:1981-2263),
 * evaluated in FP64 by hand-written reverse kernels after a replay of the
 * step from its inputs. The replay's records live in a workspace the handle
 * allocates on the first call (about 100 doubles per grid point and
 * sub-step) and keeps, grown as needed, until shield_mp_destroy. VJP calls
 * on one handle share that workspace: calls that overlap on the GPU (other
 * streams) race; calls on one stream, or on different handles, do not.
 *
 * Outputs of the step, whose cotangents are given: the ten tendencies
 * (as written by the step: udt and vdt for levels k >= 1 only), wmp (which
 * the step leaves unchanged without do_sedi_w), the persistent
 * cloud-fraction accumulator (the reference's never-reset self._qaz, so
 * that windows of several steps differentiate through it) and the four
 * surface totals. Inputs, whose adjoints are written (assigned): the 13
 * state fields of ShieldMpFields (pt, the six species, qcld, ua, va,
 * delprsi, delz, wmp) and the accumulator. The incoming tendencies only add
 * to the outputs and are not differentiated.
 *
 * Branches follow the forward at the given input. Supported: the plain form,
 * every configuration of the step (do_sedi_heat and de_ice included) and any
 * number of sub-steps. The state fields of `state` are the step's inputs as
 * they were before the step; with de_ice, state->qi_dt (NULL: zero) is the
 * incoming qi_dt the step read (de_ice rewrites qice, qsnow, qi_dt and
 * qs_dt in place, so pass copies taken before the step). No other tendency
 * is read. */
typedef struct {
  ShieldField3D pt_dt, qv_dt, ql_dt, qr_dt, qi_dt, qs_dt, qg_dt, qa_dt, udt, vdt, wmp, qaz; /* NULL ptr: zero */
  const double *rain, *snow, *ice, *graupel; /* ncol each (column c = j*nx + i), or NULL for zero */
} ShieldMpCotangents;

typedef struct {
  ShieldField3D pt, qvapor, qliquid, qrain, qice, qsnow, qgraupel, qcld, ua, va, delprsi, delz, wmp, qaz;
} ShieldMpGradients;

/* The plain FP64 step of shield_mp_step that also records, per column and
 * sub-step, the scheme's column-wide branch decisions, so that they can be
 * compared bit for bit with the reference's (its no_fall and stop_k
 * temporaries, microphysics.py:349-368, :706-754, :773-1168). Word
 * flags[s * nx * ny + (i + nx * j)] of sub-step s < ntimes holds:
 *   bit 0 / 1  rain falls in the first / second warm_rain pass (no_fall == 0)
 *   bit 2      cloud ice falls (no_fall == 0 and vi_fac >= 1e-5)
 *   bit 3 / 4  snow / graupel fall
 *   bits 16-23 the melting level: the first level k whose stop_k is 1.
 * nflags: words available (at least ntimes * nx * ny, see
 * shield_mp_substeps). Otherwise identical to shield_mp_step. */
int shield_mp_step_flags(void* handle, const ShieldMpFields* fields, double timestep, int32_t* flags, int64_t nflags,
                         void* stream);
/* ntimes, the number of sub-steps a step of `timestep` takes
 * (microphysics.py:1964-1979), or a negative status. */
int shield_mp_substeps(void* handle, double timestep);

/* state: the step's input state (its 13 state fields and land are read; its
 * tendency and precipitation pointers are ignored). A gradient pointer may
 * be NULL to skip that field. */
int shield_mp_step_vjp(void* handle, const ShieldMpFields* state, const ShieldMpCotangents* cot,
                       const ShieldMpGradients* grad, double timestep, void* stream);

/* Allocation-free step: one step of shield_mp_step with no handle and no
 * device allocation. It has no counterpart in the reference. It is meant for
 * hosts that may not call cudaMalloc: a model whose memory pool owns all of
 * the GPU's memory, or a caller whose physics interface forbids allocating.
 * The caller passes every input and output, as for shield_mp_step, plus
 * what shield_mp_create would have taken (cfg, nx, ny, nz, area); the
 * constants are recomputed on the host each call.
 *
 * The cloud-fraction accumulator that a handle would own lives instead in
 * one fixed device array of 16 MiB inside the library. Every GPU that loads
 * the library holds that array until the process exits.
 *  - Size limit: nx * ny * nz <= 2097152. Larger domains fail with
 *    SHIELD_ELAYOUT and should use shield_mp_step.
 *  - The first call on each device finds and clears the array, and
 *    synchronises that device. Make that first call before any stream
 *    capture: made while `stream` is capturing, it fails with SHIELD_EINVAL.
 *    After a cudaDeviceReset the next call repeats this set-up.
 *  - All calls on a device share the array. It keeps what the last call
 *    left. Pass first_step != 0 on the first step of a run, or when
 *    switching to another domain: this zeroes the accumulator and the error
 *    word, as a new handle starts at zero. Calls that overlap on the GPU
 *    (other streams, threads or domains) race on the array.
 *  - A column that produces a NaN or an infinity is recorded in a word of
 *    the same array; shield_mp_check_noalloc reads and clears it.
 *  - Errors are reported through shield_last_error. */
int shield_mp_step_noalloc(const ShieldMpConfig* cfg, int nx, int ny, int nz, ShieldField2D area,
                           const ShieldMpFields* fields, double timestep, int precision, int first_step,
                           void* stream);

/* The allocation-free step's failure check, like shield_mp_check for a
 * handle (no counterpart in the reference): waits for `stream`, then returns
 * SHIELD_OK with *bad_column = -1, or SHIELD_EDEVICE with the first column
 * (i + nx j) that produced a NaN or an infinity since the last check or
 * first_step call, and clears the record. nx is the calls' domain width,
 * used only for the message. Allocates nothing. */
int shield_mp_check_noalloc(int nx, int64_t* bad_column, void* stream);

/* ---------------------------------------------------------------------------
 * Ensembles: many independent domains (members of different sizes and
 * timesteps, one shared config and level count) advanced by ONE persistent
 * launch. pySHiELD has no batched call; this replaces a loop of
 * Microphysics.__call__ over members (microphysics.py:1981-2263), each member
 * with its own Microphysics instance.
 *
 * shield_mp_ensemble_create computes every member's constants, copies its
 * cell area and allocates its persistent accumulator (zero), and uploads the
 * member table once. shield_mp_ensemble_step then enqueues the zeroing of
 * the plan's work-item counter (an 8-byte memset) and a single kernel, with
 * no allocation and no copy, so it can be captured in a CUDA graph and
 * replayed. Supported level counts: 65..128. */
typedef struct {
  ShieldMpFields fields; /* the member's fields; its precipitation outputs may be NULL */
  int nx, ny;            /* the member's horizontal domain */
  double timestep;       /* the member's step */
  ShieldField2D area;    /* the member's cell area (grid_data.area) */
} ShieldMpMember;

int shield_mp_ensemble_create(const ShieldMpConfig* cfg, int nz, int nmembers, const ShieldMpMember* members,
                              int precision, void** plan);
/* cols_per_block in {2, 4, 6, 8} for 65..80 levels (two columns share each
 * group of 5 warps), in {1, 2, 4} for 81..128 levels; the launch has
 * blocks_per_sm x (number of SMs) persistent blocks. */
int shield_mp_ensemble_step(void* plan, int cols_per_block, int blocks_per_sm, void* stream);
/* copy member m's persistent accumulator (nz*nx*ny doubles, level-major)
 * into device memory at `out`, on `stream` */
int shield_mp_ensemble_qaz(void* plan, int m, double* out, void* stream);
int shield_mp_ensemble_destroy(void* plan);

/* Test hook: the scalars the step uses for `timestep` (physical constants,
 * setupm constants, sub-step values) in the order of the internal parameter
 * block; returns how many doubles were written (at most n). */
int shield_mp_constants(void* handle, double timestep, double* out, int n);

/* Test hook: copy the persistent cloud-fraction accumulator (nz*nx*ny
 * doubles, level-major) into / out of device memory at `qaz`. */
int shield_mp_get_qaz(void* handle, double* qaz, void* stream);
int shield_mp_set_qaz(void* handle, const double* qaz, void* stream);

/* update_physics_state_with_tendencies (physics.py:151-194):
 * out_X = X + X_dt * dt for the ten (X, X_dt) pairs in this order:
 * qvapor/qv_dt, qliquid/ql_dt, qrain/qr_dt, qice/qi_dt, qsnow/qs_dt,
 * qgraupel/qg_dt, qcld/qa_dt, pt/pt_dt, ua/udt, va/vdt.
 * The domain is nx x ny x nz, at most 2^31 - 1 points (SHIELD_ELAYOUT
 * otherwise). */
int shield_update_physics_state(int nx, int ny, int nz, const ShieldField3D* state10, const ShieldField3D* tend10,
                                const ShieldField3D* out10, double dt, void* stream);

/* The column part of UpdateAtmosphereState.__call__
 * (update_atmos_state.py:301-349, fv_update_phys.py:152-188), in the
 * reference's order and on the reference's domains:
 *   fill_gfs_delp(delp, q, 1e-9) on the full (halo) horizontal domain,
 *       nz+1 levels; q is physics_updated_specific_humidity, or the dycore
 *       qvapor with SHIELD_UAS_DYCORE_ONLY (then nothing else runs);
 *   prepare_tendencies_and_update_tracers on the compute domain, nz+1 levels
 *       (levels 0..nz-1 written), with rdt = 1 / dt_atmos;
 *   with SHIELD_UAS_APPLY: moist_cv and update_pressure_and_surface_winds on
 *       the compute domain, nz+1 levels, with the call's dt.
 * The horizontal halo exchange of u_dt/v_dt, AGrid2DGridPhysics and
 * CubedToLatLon are not part of this call.
 * Every field must provide nz+1 levels; fill_gfs_delp also reads and
 * writes `hx` halo points on each side of the compute domain.
 * Field order of `f` (ShieldField3D, origin at the compute-domain corner):
 *   0 u_dt 1 v_dt 2 pt_dt 3 u_t1 (physics_updated_ua) 4 v_t1
 *   5 physics_updated_pt 6 physics_updated_specific_humidity
 *   7 physics_updated_qliquid 8 physics_updated_qrain 9 physics_updated_qsnow
 *   10 physics_updated_qice 11 physics_updated_qgraupel 12 u_t0 (physics ua)
 *   13 v_t0 (physics va) 14 pt_t0 (physics pt) 15 dycore qvapor 16 qliquid
 *   17 qrain 18 qsnow 19 qice 20 qgraupel 21 prsi 22 dycore delp
 *   23 dycore pt 24 pe 25 peln 26 pk 27 dycore ua 28 dycore va
 * Outputs ps, u_srf, v_srf: 2-D fields (their sk is ignored).
 * At most nz = 128 levels (SHIELD_ELAYOUT otherwise). */
#define SHIELD_UAS_APPLY 1       /* apply_tendencies = True */
#define SHIELD_UAS_DYCORE_ONLY 2 /* dycore_only = True */
int shield_update_atmos_state(int nx, int ny, int nz, int hx, int mode, const ShieldField3D* f, ShieldField3D ps,
                              ShieldField3D u_srf, ShieldField3D v_srf, double rdt, double dt, double kappa,
                              double cp_air, void* stream);

/* Fields of shield_physics_prestep: the PhysicsState storages
 * (pySHiELD/physics_state.py:17-300) and Physics' own scratch
 * (physics.py:222-225), each with the origin at the compute-domain corner
 * and nz + 1 levels of storage. The member order is fixed. */
typedef struct {
  ShieldField3D phii, prsi, prsik; /* interface fields; prsik is Physics._prsik */
  ShieldField3D delz, delp;
  ShieldField3D qvapor, qliquid, qrain, qice, qsnow, qgraupel, qo3mr, qsgs_tke;
  ShieldField3D pt;
  ShieldField3D dm;      /* Physics._dm3d */
  ShieldField3D delprsi;
  ShieldField3D del_gz;  /* Physics._del_gz */
  ShieldField3D phil;
  ShieldField3D omga, dz, wmp; /* read / written by prepare_microphysics only */
  ShieldField3D pt_dt, qv_dt, ql_dt, qr_dt, qi_dt, qs_dt, qg_dt, qa_dt, udt, vdt; /* the microphysics
                                   tendencies that prepare_microphysics zeroes; a NULL ptr is skipped */
} ShieldPhysicsFields;

#define SHIELD_PHYS_PREPARE_MICROPHYSICS 1 /* run prepare_microphysics (GFS_microphysics in the schemes) */

/* The physics driver's steps before the microphysics, Physics.__call__
 * (physics.py:276-330), in the reference's order and on its domains:
 *   atmos_phys_driver_statein on the compute domain, nz + 1 levels
 *       (externals nwat, ptop, pk0inv = (1/p00)^kappa, pktop = (ptop/p00)^kappa,
 *       p00 = 1e5, computed here from ptop as Physics.__init__ does);
 *   get_prs_fv3 and get_phi_fv3 on the full domain (hx halo points on each
 *       side), nz + 1 levels;
 *   with SHIELD_PHYS_PREPARE_MICROPHYSICS: prepare_microphysics on the
 *       compute domain, nz levels.
 * One fused kernel; see pyshield_b200/csrc/physics.cu. */
int shield_physics_prestep(int nx, int ny, int nz, int hx, int nwat, double ptop, int flags,
                           const ShieldPhysicsFields* fields, void* stream);

/* DycoreToPhysics' copy (update_atmos_state.py:95-142, :160-167, :196-232):
 * for each of the 16 fields in the order qvapor, qliquid, qrain, qsnow,
 * qice, qgraupel, qo3mr, qsgs_tke, qcld, pt, delp, delz, ua, va, w, omga,
 * physics = dycore on i in [0, nx], j in [0, ny] (the compute domain plus
 * one interface point, which the storages must have) and k in [0, nz); at
 * most 2^31 - 1 points (SHIELD_ELAYOUT otherwise). */
int shield_copy_dycore_to_physics(int nx, int ny, int nz, const ShieldField3D* dycore16,
                                  const ShieldField3D* physics16, void* stream);

/* DycoreToPhysics' copy followed by shield_physics_prestep, as one launch:
 * the results, in every physics storage, are those of
 * shield_copy_dycore_to_physics then shield_physics_prestep (the copy of
 * update_atmos_state.py:196-232 followed by physics.py:276-330), but the
 * pre-step reads the dycore storages where the copy would have put them and
 * writes each copied field once, so the separate copy's pass over HBM goes.
 * dycore16 / physics16: the copy's 16 fields in the order of
 * shield_copy_dycore_to_physics; the physics ones are the storages of
 * `fields` where both name a field. Needs hx >= 1 (the copy's interface
 * points i = nx, j = ny lie in the pre-step's halo). */
int shield_physics_prestep_from_dycore(int nx, int ny, int nz, int hx, int nwat, double ptop, int flags,
                                       const ShieldPhysicsFields* fields, const ShieldField3D* dycore16,
                                       const ShieldField3D* physics16, void* stream);

/* AGrid2DGridPhysics (update_dwind_phys.py): the A-grid wind tendencies
 * turned into D-grid winds. Indices are relative to the compute-domain
 * origin. One region of a cube edge: the points [lo, hi) along the edge line
 * `line` (j for the south / north edges, i for west / east), corrected with
 * the neighbour at +1 (dir = 1, the part below the edge's midpoint) or -1. */
typedef struct {
  int line, lo, hi, dir;
} ShieldEdgeRegion;
typedef struct {
  int n[4];                  /* regions per edge: south, north, west, east */
  ShieldEdgeRegion r[4][2];  /* in the reference's order (lower, upper) */
} ShieldEdgePlan;
/* The grid vectors (DriverGridData): 2-D fields at the compute origin, and
 * the 1-D south / north edge weights along i (element stride edge_stride). */
typedef struct {
  ShieldField2D vlon1, vlon2, vlon3, vlat1, vlat2, vlat3;
  ShieldField2D es1_1, es1_2, es1_3, ew2_1, ew2_2, ew2_3;
  ShieldField2D edge_vect_w, edge_vect_e;
  const double* edge_vect_s;
  const double* edge_vect_n;
  int64_t edge_stride;
} ShieldDwindGeometry;

/* With grid_type <= 3: u += dt5 (ue . es1) on i in [0, nx), j in [0, ny],
 * v += dt5 (ve . ew2) on i in [0, nx], j in [0, ny), ue / ve from the
 * tendencies with the plan's edge corrections, then u_dt = v_dt = 0 on i, j
 * in [-1, n + 1); the tendencies need one halo point, filled by the caller's
 * halo exchange. With grid_type > 3: the doubly periodic update on the
 * compute domain (plan and geometry unused). dt5 = dt_atmos / 2.
 * (ny + 2) * nz must stay below 2^31 (SHIELD_ELAYOUT otherwise). */
int shield_agrid_to_dgrid(int nx, int ny, int nz, int grid_type, double dt5, const ShieldEdgePlan* plan,
                          const ShieldDwindGeometry* geometry, ShieldField3D u, ShieldField3D v, ShieldField3D u_dt,
                          ShieldField3D v_dt, void* stream);

/* The cube-sphere update of shield_agrid_to_dgrid on several tiles at once
 * (a GPU holding the subtiles of several ranks, up to all six cube tiles):
 * one launch updates u and v on every tile, a second zeroes every tile's
 * tendencies, where separate calls take two launches per tile. Each tile's
 * results are those of its own shield_agrid_to_dgrid call. 1 to 6 tiles,
 * grid_type <= 3 each. */
typedef struct {
  int nx, ny, nz, grid_type;
  double dt5;
  ShieldEdgePlan plan;
  ShieldDwindGeometry geometry;
  ShieldField3D u, v, u_dt, v_dt;
} ShieldDwindTile;
int shield_agrid_to_dgrid_tiles(int ntiles, const ShieldDwindTile* tiles, void* stream);

/* The handle's device error word: every step records the first column
 * whose outputs hold a NaN or an infinity (the kernel never traps). This
 * call waits for `stream`, then returns SHIELD_OK with *bad_column = -1, or
 * SHIELD_EDEVICE with the column (i + nx j) and a message, and clears the
 * word. */
int shield_mp_check(void* handle, int64_t* bad_column, void* stream);

/* Test hook: the scalars shield_mp_step uses for `timestep` (physical
 * constants, setupm constants, sub-step values), computed on the host
 * without touching the GPU; returns how many doubles were written. */
int shield_mp_setup_constants(const ShieldMpConfig* cfg, double timestep, double* out, int n);

/* Message of the last failing handle-free call on this host thread. */
int shield_last_error(char* buf, size_t n);

#ifdef __cplusplus
}
#endif

#endif /* SHIELD_MP_H */
