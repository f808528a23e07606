/*
 * aero_b200.h -- C ABI of the B200-native Navier-Stokes step (libaero_b200.so).
 *
 * Plain pointers, sizes and a cudaStream_t (passed as void*): no torch types.  Every
 * device buffer is owned by the caller; the library never allocates or frees device
 * memory and never synchronises the stream, so every call can be captured in a CUDA
 * graph.  Functions return AERO_OK (0) or a negative AERO_E* code; aero_last_error()
 * gives a thread-local message for the last failure on the calling thread.
 *
 * The entry points replace these parts of the reference (Aerolume, src/aerolume/solvers):
 *
 *   aero_ns3d_plan_create      ns3d/fused.py:226 load_kernels (builds the per-config constants)
 *   aero_ns3d_step             ns3d/fused.py:378 fast_step_phys (+ core.py:765 step3d_phys),
 *                              followed by the smoke update of ns3d/solver.py:646
 *                              _advance_tracers (ns3d/fused.py:553 fast_dye and
 *                              ns3d/dye.py:301 apply_solids_and_sources)
 *   aero_ns3d_smoke            ns3d/fused.py:553 fast_dye + ns3d/dye.py:301 apply_solids_and_sources
 *   aero_ns3d_project          ns3d/core.py:604 project3d
 *   aero_ns3d_poisson_solve    ns3d/poisson.py:152 PoissonSolver3D.solve
 *   aero_ns3d_workspace_bytes  (no counterpart: the reference allocates inside torch)
 *   aero_ns3d_fields           ns3d/fields.py:45 gradient_field, ns3d/solver.py:1374 _centred
 *   aero_ns3d_probe            ns3d/fields.py:78 trilinear (surface probes, slices, wake lines)
 *   aero_ns3d_build_masks      ns3d/geometry.py:385 build_geometry3d with its exact signed
 *                              distance (geometry.py:229 grid_signed_distance, use_shared=False)
 *   aero_mesh_signed_distance  ns3d/geometry.py:126 mesh_signed_distance
 *   aero_record_history        ns3d/solver.py:706 FlowSolver3D._record (history ring rows)
 *   aero_smoke_emitters        ns3d/emitters.py:200 apply_smoke_sources (smoke emitters)
 *   aero_welford               ns3d/solver.py:732 FlowSolver3D._welford (running means)
 *   aero_ns2d_plan_create      ns2d/core.py:182 make_operators (the per-config constants)
 *   aero_ns2d_step             ns2d/core.py:815 step_full (heat transfer its only placed
 *                              physics: physics.py:623-884, the report of core.py:974
 *                              _report), with the dye update of its lines 959-962
 *                              (core.py:703 advect_dye, core.py:779 _zero_dye_in_solids)
 *   aero_ns2d_poisson_solve    ns2d/poisson.py:126 PoissonSolver.solve
 *   aero_ns2d_sweep_*          (no counterpart: many 2D instances in one persistent launch; the
 *                              reference loops ns2d/solver.py:489 advance over them)
 *   aero_closure_*, aero_mlp_* (no counterpart: the learned subgrid closure, which stands in
 *                              for ns3d/core.py:448 eddy_viscosity3d (WALE) where it applies)
 */
#ifndef AERO_B200_H
#define AERO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AERO_ABI_VERSION 6

#define AERO_OK 0
#define AERO_EINVAL -1        /* invalid argument or inconsistent configuration     */
#define AERO_EUNSUPPORTED -2  /* a feature the library does not implement: no fallback */
#define AERO_ECUDA -3         /* a CUDA launch or runtime call failed                */

#define AERO_MAX_BODIES 8
#define AERO_MAX_FANS 4
#define AERO_MAX_PORTS 4
#define AERO_MAX_HEATERS 4

enum { AERO_F32 = 0, AERO_F64 = 1 };
enum { AERO_ADV_UPWIND3 = 0, AERO_ADV_CENTRAL = 1 };
enum { AERO_LES_NONE = 0, AERO_LES_SMAGORINSKY = 1, AERO_LES_WALE = 2, AERO_LES_VREMAN = 3 };
/* velocity ghost-cell rules of ns3d/core.py:147-181 */
enum {
  AERO_GHOST_EDGE = 0, AERO_GHOST_EVEN = 1, AERO_GHOST_ODD = 2, AERO_GHOST_AFFINE = 3,
  AERO_GHOST_FACE_ODD = 4, AERO_GHOST_PERIODIC_CELL = 5, AERO_GHOST_PERIODIC_FACE = 6
};
/* temperature side conditions of ns3d/physics.py:589-607 (left, right, front, back, bottom, top) */
enum {
  AERO_TH_PERIODIC = 0, AERO_TH_OUTFLOW = 1, AERO_TH_ADIABATIC = 2, AERO_TH_INFLOW = 3,
  AERO_TH_TEMPERATURE = 4, AERO_TH_HEAT_FLUX = 5
};

/* Everything static about one 3D solve: grid, rules, constants (ns3d/core.py:61-108,
 * ns3d/physics.py:494-560, ns3d/dye.py:140-151).  Scalars are doubles whatever the
 * field dtype; the kernels round them to the field type as the reference does. */
typedef struct AeroNs3dConfig {
  int32_t abi_version;          /* AERO_ABI_VERSION                                        */
  int32_t dtype;                /* AERO_F32 or AERO_F64                                    */
  int32_t nx, ny, nz;           /* cells                                                   */
  double h;
  int32_t periodic[3];          /* x, y, z                                                 */
  int32_t closed;               /* walls at x0 and x1 (domain = "closed")                  */
  int32_t symmetry;             /* y = y0 symmetry plane (forces doubled)                  */
  int32_t advection;            /* AERO_ADV_*                                              */
  int32_t les;                  /* AERO_LES_*                                              */
  double les_c;                 /* model constant                                          */
  double nu;                    /* 1 / Re                                                  */
  double eta;                   /* Brinkman permeability                                   */
  double cfl;
  int32_t has_dt_fixed;
  double dt_fixed;
  int32_t ghost_kind[3][3][2];  /* [u, v, w][x, y, z][lo, hi] : AERO_GHOST_*               */
  double ghost_val[3][3][2];    /* value of AFFINE rules (moving road)                     */
  double ref_area, length_ref, span_ref;
  double moment_ref[3];
  double y0;
  int32_t window[6];            /* body cell window k0, k1, j0, j1, i0, i1 (empty: none)   */
  int32_t nbody;
  /* heat transfer (thermal = 0: off) */
  int32_t thermal;
  double kappa, pe, ri, prt, eta_t;
  int32_t side_kind[6];         /* AERO_TH_*                                               */
  double side_val[6];
  int32_t has_heat_max;
  double heat_max;
  int32_t n_tbody;              /* "temperature" bodies                                    */
  int32_t t_index[AERO_MAX_BODIES];
  int32_t has_adia, has_skin;
  double flux_rate[AERO_MAX_BODIES];
  /* smoke (smoke = 0: off) */
  int32_t smoke;
  int32_t dye_window[6];        /* nozzle window (empty: no nozzles)                       */
  double pulse_on, pulse_period;
  /* step controls of the placed physics (ns3d/physics.py:1144-1181, 1230-1262) */
  double u_floor;               /* speed scale of the momentum sources (0: none)           */
  int32_t pid;                  /* PID control of dt towards pid_target x the limit         */
  double pid_target;
  int32_t paint;                /* painted solids (geom paint_*; physics.py:1074-1141)      */
  int32_t nfan;                 /* actuator discs (geom fans; physics.py:831-979)           */
  int32_t fan_swirl;            /* any fan with swirl                                       */
  int32_t nport;                /* jets and vents (geom ports; physics.py:981-1072)         */
  double port_source;           /* their net mass flux in outlet-face units (h sum m)       */
  double port_leak;             /* uniform scalar leak of an unbalanced closed box (Q / V)  */
  int32_t nheat;                /* volumetric heaters (geom heaters; physics.py:464-491)    */
  /* learned subgrid closure (geom closure): the eddy viscosity of an MLP's subgrid stress in
   * place of WALE where it applies, WALE elsewhere; les must be AERO_LES_WALE, dtype FP32 */
  int32_t closure;
  /* a uniform body force added to the tendencies (the verification cases' ops.forcing,
   * ns3d/core.py:565-566; forcing = 0: none) */
  int32_t forcing;
  double force[3];
} AeroNs3dConfig;

/* One actuator disc (ns3d/physics.py:831-979): its cell window, the force, swirl and
 * disc-average weights on the window's u, v, w faces (the shapes of the body window's
 * masks, over the fan's own window), the PI constants, and its state: 0-d scalars of the
 * plan's dtype that every step updates in place (thrust T, disc velocity ud, PI error
 * e_prev, swirl amplitude). */
typedef struct AeroNs3dFan {
  int32_t window[6];            /* k0, k1, j0, j1, i0, i1                                  */
  int32_t velocity_mode;        /* 1: PI on the thrust towards target; 0: fixed thrust     */
  double target, kp, ki, tmax, swirl;
  const void *f_u, *f_v, *f_w;  /* n_g phi_g / (sum phi h^3)                               */
  const void *s_u, *s_v, *s_w;  /* swirl weights                                           */
  const void *m_u, *m_v, *m_w;  /* disc-average weights                                    */
  void *thrust, *ud, *e_prev, *swirl_amp;
} AeroNs3dFan;

/* One jet or vent (ns3d/physics.py:981-1072): a mass source m = Q phi_c on the cells of its
 * window (taken out of the projection's right-hand side), momentum on the window's faces
 * (a jet: f = Q speed n_g phi_g; a vent: f = Q phi_g times the local velocity), and the
 * temperature it carries (a jet's theta; a vent takes the local value out). */
typedef struct AeroNs3dPort {
  int32_t window[6];            /* k0, k1, j0, j1, i0, i1                                  */
  int32_t vent;                 /* 1: vent, 0: jet                                         */
  double theta;                 /* a jet's temperature                                     */
  const void *f_u, *f_v, *f_w;  /* face weights over the window (body-mask shapes)         */
  const void *m;                /* cell weights over the window                            */
} AeroNs3dPort;

/* One volumetric heater (ns3d/physics.py:464-491 HeatSourceSet): its cell window and the
 * source density on the window's cells (wz, wy, wx; conduction units, times kappa in the heat
 * equation), device, of the plan's dtype. */
typedef struct AeroNs3dHeater {
  int32_t window[6];            /* k0, k1, j0, j1, i0, i1                                  */
  const void *q;
} AeroNs3dHeater;

/* Window masks and constant inputs (device pointers of the plan's dtype; NULL when absent).
 * Shapes are those of ns3d/geometry.py:275-303 and ns3d/physics.py:314-461. */
typedef struct AeroNs3dGeom {
  const void *chi_u, *chi_v, *chi_w, *chi_c;
  const void *a_u, *a_v, *a_w;
  const void *k_u, *k_v, *k_w;  /* (nbody, 3, ...) force / moment weights                */
  const void *chi_t, *a_t, *w_t;
  const void *adia_u, *adia_v, *adia_w;
  const void *vol_w, *skin;
  const void *dye_weight;
  const void *u_inlet;          /* (nz, ny)                                                */
  /* painted solid fractions on the whole grid (u, v, w faces and cells; read at every step,
   * so strokes between steps take effect) */
  const void *paint_u, *paint_v, *paint_w, *paint_c;
  const AeroNs3dFan *fans;      /* host array of cfg.nfan descriptors, read at every step  */
  const AeroNs3dPort *ports;    /* host array of cfg.nport descriptors                     */
  const AeroNs3dHeater *heaters; /* host array of cfg.nheat descriptors                  */
  const struct AeroClosureModel *closure; /* the trained closure when cfg.closure (host struct) */
} AeroNs3dGeom;

/* State in and out (device pointers of the plan's dtype).  u may alias u0, v v0, w w0 and
 * theta theta0; dye must not alias dye0.  t0, t, dt are 0-d scalars; coeffs is
 * (nbody, 6), heat_rate (nbody).  theta/dye pointers are ignored when the plan has no
 * heat transfer / smoke. */
typedef struct AeroNs3dFields {
  const void *u0, *v0, *w0, *theta0, *dye0, *t0;
  void *u, *v, *w, *p, *theta, *dye, *t, *dt;
  void *coeffs, *heat_rate;
  /* PID controller state (0-d scalars of the plan's dtype, read and updated in place by a
   * step whose dt comes from the rule; dt_prev <= 0 means "first step") */
  void *pid_dt_prev, *pid_e1, *pid_e2;
  /* diagnostics (NULL: not computed): a 0-d scalar of the plan's dtype that receives the sum
   * of squares of the last stage's projection right-hand side -- the divergence of the stage
   * value minus the jets' and vents' mass sources (physics.py:1303-1305 record_divergence,
   * called by fused.py:480-482 on the last stage when the solver records a diagnostics row) */
  void *div_sq;
} AeroNs3dFields;

typedef struct AeroNs3dPlan AeroNs3dPlan;

int aero_abi_version(void);
const char *aero_last_error(void);

/* Validate a configuration and build its host-side constants. */
int aero_ns3d_plan_create(const AeroNs3dConfig *cfg, AeroNs3dPlan **plan);
void aero_ns3d_plan_destroy(AeroNs3dPlan *plan);

/* Device workspace the plan needs (bytes, 256-byte aligned base required). */
size_t aero_ns3d_workspace_bytes(const AeroNs3dPlan *plan);

/* Fill the plan's tables (twiddles, eigenvalues) in a fresh workspace; once per workspace. */
int aero_ns3d_workspace_init(const AeroNs3dPlan *plan, void *workspace, void *stream);

/* One SSP-RK3 step with the configured physics, then the smoke update.
 * dt_in: NULL for the CFL / heat-equation rule evaluated on the device, else a device
 * 0-d scalar with the step to take. */
int aero_ns3d_step(const AeroNs3dPlan *plan, const AeroNs3dFields *f, const AeroNs3dGeom *g,
                   const void *dt_in, void *workspace, void *stream);

/* aero_ns3d_step that also records CUDA events (cudaEvent_t handles, created with timing
 * enabled) at the phase boundaries of the step, as external events so that they work inside a
 * captured CUDA graph.  Event i is recorded after phase i (up to nevents):
 *   0 start; 1 time step (maxima, eddy-viscosity pre-pass, dt);
 *   2 + 5 s .. 6 + 5 s for stage s = 0, 1, 2: outlet correction, stage kernel, divergence,
 *   Poisson solve (five transform passes and the psi accumulation), gradient correction;
 *   17 smoke; 18 end of step.  (No counterpart in the reference: a measurement hook.) */
#define AERO_NS3D_TRACE_EVENTS 19
int aero_ns3d_step_traced(const AeroNs3dPlan *plan, const AeroNs3dFields *f, const AeroNs3dGeom *g,
                          const void *dt_in, void *workspace, void *stream, void *const *events, int32_t nevents);

/* Smoke alone (the step's tracer update): dye <- MUSCL step of dye0 with (u, v, w) and dt,
 * then solids cleared and nozzles relaxed at time t.  Fields of f used: u, v, w, dye0, dye,
 * and dt and t as inputs (the step just taken and the new time).  dye must not alias dye0.
 * g->chi_c NULL skips the clearing inside solids and g->dye_weight NULL the nozzles, which
 * leaves the advection alone (ns3d/fused.py:553 fast_dye). */
int aero_ns3d_smoke(const AeroNs3dPlan *plan, const AeroNs3dFields *f, const AeroNs3dGeom *g, void *stream);

/* psi with L psi = f, zero mean (f and psi: (nz, ny, nx) device arrays; may alias). */
int aero_ns3d_poisson_solve(const AeroNs3dPlan *plan, const void *f, void *psi, void *workspace,
                            void *stream);

/* Allocation-free variant of aero_ns3d_poisson_solve.  No counterpart in the reference: it is
 * for callers that cannot allocate device memory (a host that reserves the GPU's memory in its
 * own arena, or a real-time loop in which cudaMalloc / cudaFree would synchronise the device).
 * The transform tables go to a static device array of AERO_STATIC_SCRATCH_BYTES that every GPU
 * which loads the library holds until exit; the caller passes no workspace.  The tables take
 * 7n values per axis of n cells plus n * n for an axis whose length has a prime factor above 3
 * (dense transform): FP64 fits three FFT axes of up to 2048 cells, or one dense axis of up to
 * about 330 beside two FFT axes of 256.  Larger grids are rejected with AERO_EINVAL and a
 * message naming the bytes they need.  The first call on a device looks up the array's device
 * address (with that device current); make that first call before any stream capture.  Calls
 * share the array: calls that overlap on the GPU race.  Allocates nothing (no cudaMalloc,
 * cudaFree or allocating library routine). */
#define AERO_STATIC_SCRATCH_BYTES (1u << 20)
int aero_ns3d_poisson_solve_static(const AeroNs3dPlan *plan, const void *f, void *psi, void *stream);

/* In place: (u, v, w) <- (u, v, w) - grad psi with lap psi = div(u, v, w); psi written. */
int aero_ns3d_project(const AeroNs3dPlan *plan, void *u, void *v, void *w, void *psi, void *workspace,
                      void *stream);

/* Cell-centred output fields of a state (u, v, w: the plan's staggered shapes), the B200 side of
 * ns3d/fields.py:24-75 gradient_field and ns3d/solver.py:1374-1416 FlowSolver3D._centred:
 * out[AERO_FIELD_U..AERO_FIELD_NUT] are (nz, ny, nx) device arrays, or NULL to skip one.  The
 * eddy viscosity is switched off inside solids with g->chi_c (g may be NULL: no bodies). */
enum {
  AERO_FIELD_U = 0, AERO_FIELD_V = 1, AERO_FIELD_W = 2, AERO_FIELD_SPEED = 3,
  AERO_FIELD_VORTICITY = 4, AERO_FIELD_Q = 5, AERO_FIELD_NUT = 6, AERO_FIELD_COUNT = 7
};
int aero_ns3d_fields(const AeroNs3dPlan *plan, const void *u, const void *v, const void *w, const AeroNs3dGeom *g,
                     void *const *out, void *stream);

/* Trilinear sampling (ns3d/fields.py:78 trilinear) of a (shape[0], shape[1], shape[2]) =
 * (nz, ny, nx) field whose entry (k, j, i) sits at origin + ((i, j, k) + off) h, at npts
 * points (x, y, z) (device, the plan's dtype); points outside are clamped to the edge. */
int aero_ns3d_probe(const AeroNs3dPlan *plan, const void *field, const int32_t shape[3], const double origin[3],
                    const double off[3], const void *pts, int64_t npts, void *out, void *stream);

/* ---- mask construction (ns3d/geometry.py:385-495) ---------------------------------- */

/* The operator fields build_geometry3d reads, and the body window the caller chose
 * (geometry.py:323 body_window3d, or a fixed one for live attitude edits). */
typedef struct {
  int32_t abi_version;          /* AERO_ABI_VERSION                                        */
  int32_t dtype;                /* AERO_F32 or AERO_F64 (masks and mesh coordinates)       */
  int32_t nx, ny, nz;
  double h, x0, y0, z0;
  int32_t periodic[3];          /* x, y, z: periodic axes keep their boundary faces        */
  int32_t window[6];            /* k0, k1, j0, j1, i0, i1 (non-empty, inside the domain)   */
  double mask_width, mask_shift;/* ramp half-width and wall shift, in cells                */
  double moment_ref[3];
  int32_t nbody;                /* 1 .. AERO_MAX_BODIES                                    */
} AeroMaskConfig;

/* One immersed mesh (ns3d/config.py:81 ImmersedMesh): device vertices (nvert, 3) in the
 * config dtype, device faces (nface, 3) of vertex indices in 0 .. nvert-1 (the caller checks
 * them: the kernels clamp an index out of range to vertex 0 instead of faulting), rigid spin. */
typedef struct {
  const void *vertices;
  int32_t nvert;
  const int32_t *faces;
  int32_t nface;
  double omega, center[3], axis[3];
} AeroMaskBody;

/* Outputs on the window (geometry.py:275-303 Geometry3D): chi_u (wz, wy, wx+1), chi_v
 * (wz, wy+1, wx), chi_w (wz+1, wy, wx), chi_c (wz, wy, wx), a_* like chi_*, k_u (nbody, 3,
 * wz, wy, wx+1) and likewise k_v, k_w. */
typedef struct {
  void *chi_u, *chi_v, *chi_w, *chi_c, *a_u, *a_v, *a_w, *k_u, *k_v, *k_w;
} AeroMaskOut;

size_t aero_ns3d_masks_workspace_bytes(const AeroMaskConfig *cfg, const AeroMaskBody *bodies);
int aero_ns3d_build_masks(const AeroMaskConfig *cfg, const AeroMaskBody *bodies, const AeroMaskOut *out,
                          void *workspace, void *stream);

/* Exact signed distance (negative inside) of npoints device points (x, y, z) to one mesh,
 * with the face plane distance within plane_zone of a face (geometry.py:126-196). */
size_t aero_mesh_sdf_workspace_bytes(int32_t dtype, int32_t nface, int64_t npoints);
int aero_mesh_signed_distance(int32_t dtype, const void *vertices, int32_t nvert, const int32_t *faces, int32_t nface,
                              const void *points, int64_t npoints, double plane_zone, void *out, void *workspace,
                              void *stream);

/* ---- smoke emitters (ns3d/emitters.py:57-87, 200-210) ------------------------------- */

/* One field emitter: its cell window, the smoke channel it feeds, the weights on the window
 * (wz, wy, wx) and its device parameters [rate, start, stop, period, t_on] (dtype). */
typedef struct {
  int32_t window[6];
  int32_t channel;
  const void *weight, *params;
} AeroSmokeEmitter;

/* In order, each emitter relaxes its channel towards its rate inside its window while its
 * release switch is on at the device time t: c += w on (rate - c).  channels is a host array
 * of nchannel device pointers to (nz, ny, nx) arrays of dtype. */
int aero_smoke_emitters(int32_t dtype, int32_t nz, int32_t ny, int32_t nx, void *const *channels, int32_t nchannel,
                        const AeroSmokeEmitter *emitters, int32_t nemit, const void *t, void *stream);

/* ---- per-step bookkeeping (ns3d/solver.py:706-744) --------------------------------- */

/* One history row: hist[slot] = [t, sum over bodies of coeffs (nbody, 6)] at slot = *hist_n
 * mod capacity, body_c = coeffs (when non-NULL), phist[slot] = [t, extra (n_extra)] (when
 * phist is non-NULL), *hist_n += 1, and *pending += dt (FP64, when pending is non-NULL).  t,
 * dt, coeffs, extra, hist, phist are device arrays of dtype; hist_n a device int64. */
int aero_record_history(int32_t dtype, const void *t, const void *dt, const void *coeffs, int32_t nbody,
                        void *body_c, void *hist, int64_t capacity, int64_t *hist_n, const void *extra,
                        int32_t n_extra, void *phist, double *pending, void *stream);

/* The time-weighted Welford update of nfield (<= 5) fields x[f] (count[f] elements) into
 * mean[f], m2[f] with weight w = *pending: r = w / (*time + w), mean += d r, m2 += d (x -
 * mean) w; then *time += w, *pending = 0.  The pointer arrays are host arrays of device
 * pointers; pending and time are device FP64 scalars. */
int aero_welford(int32_t dtype, int32_t nfield, const void *const *x, void *const *mean, void *const *m2,
                 const int64_t *count, double *pending, double *time, void *stream);

/* ---- learned subgrid closure ---------------------------------------------------------
 * No counterpart in the reference: a per-cell MLP (10 inputs -> 3 x 128 SiLU -> 6 outputs)
 * from the filtered velocity gradient to the subgrid stress, trained on pairs that the plain
 * step makes by box-filtering its own fine periodic runs, run on the tensor cores in BF16 with
 * FP32 accumulation.  In the step it replaces the WALE eddy viscosity of ns3d/core.py:448-482
 * (ns3d/fused.py:102-132 ns3d_nut_wale) by the eddy viscosity with the learned stress's
 * dissipation, nu_t = -tau:S / (2 S:S); WALE stays wherever that dissipation is not positive
 * or an input lies outside its training range.
 *
 * Inputs of a gradient g (g33 = -(g11 + g22)): g11, g12, g13, g21, g22, g23, g31, g32 over |g|,
 * (|W|^2 - |S|^2) / |g|^2 and sqrt(6) tr(S^3) / |S|^3 (S, W the symmetric and antisymmetric
 * parts); outputs tau_xx, tau_yy, tau_zz, tau_xy, tau_xz, tau_yz over Delta^2 |g|^2, Delta the
 * filter width (the grid spacing of the step).  Inputs and outputs are standardised with the
 * model's means and standard deviations. */
#define AERO_CLOSURE_IN 10
#define AERO_CLOSURE_OUT 6
#define AERO_CLOSURE_HIDDEN 128
/* FP32 master parameters of the MLP, one flat array in this order: W1 (128, 10), b1 (128),
 * W2 (128, 128), b2 (128), W3 (128, 128), b3 (128), W4 (6, 128), b4 (6); weights row-major
 * [out][in].  The kernels read the BF16 copy of the weights (same offsets) and the FP32 biases. */
#define AERO_CLOSURE_NPARAM 35206
typedef struct AeroClosureModel {
  const float *params;          /* device, AERO_CLOSURE_NPARAM FP32                         */
  const void *params_bf16;      /* device, AERO_CLOSURE_NPARAM BF16 (the weights' copy)      */
  float in_mean[AERO_CLOSURE_IN], in_std[AERO_CLOSURE_IN];
  float in_lo[AERO_CLOSURE_IN], in_hi[AERO_CLOSURE_IN];     /* training range of the raw inputs */
  float out_mean[AERO_CLOSURE_OUT], out_std[AERO_CLOSURE_OUT];
} AeroClosureModel;

/* Training pairs of an n^3 periodic FP32 state (u (n, n, n+1), v (n, n+1, n), w (n+1, n, n),
 * cell size h) filtered by factor^3 boxes onto m^3 = (n / factor)^3 cells: g8 (8, m^3) the
 * gradient of the filtered velocity by the step's own stencil (core.py:400-445) at spacing
 * Delta = factor h, tau (6, m^3) the subgrid stress mean(u_a u_b) - mean(u_a) mean(u_b) of the
 * cell-centred velocities.  work: 3 m^3 floats.  n % factor == 0. */
int aero_closure_pairs(int32_t n, int32_t factor, const float *u, const float *v, const float *w, double h, float *g8,
                       float *tau, float *work, void *stream);
/* Raw inputs feat (n, 10), the output scale Delta^2 |g|^2 and validity (uint8) of n gradients
 * g8 (8, n); with tau (6, n) non-NULL also the scaled targets (n, 6). */
int aero_closure_features(int64_t n, const float *g8, double delta, const float *tau, float *feat, float *scale,
                          uint8_t *valid, float *target, void *stream);
/* Standardised BF16 inputs x (n, 16; columns 10..15 zero) and, with target non-NULL, FP32
 * targets t (n, 6) with the model's means and standard deviations. */
int aero_closure_normalise(int64_t n, const float *feat, const float *target, const AeroClosureModel *m, void *x,
                           float *t, void *stream);
/* The MLP on n standardised BF16 inputs x (n, 16): standardised outputs y (n, 6), FP32.
 * status: device int, bit 2 set when a tensor-core wait ran out. */
int aero_mlp_forward(const AeroClosureModel *m, const void *x, int64_t n, float *y, int32_t *status, void *stream);
/* Device bytes of the training workspace for a batch (a multiple of 128). */
size_t aero_mlp_train_workspace_bytes(int32_t batch);
/* Gradient of the batch's mean squared error (over the batch rows idx and the 6 outputs) with
 * respect to the parameters, added to grad (FP32, AERO_CLOSURE_NPARAM), by the tensor-core
 * forward and backward passes; loss (device double) += the batch's sum of squared errors. */
int aero_mlp_gradients(const float *params, const void *params_bf16, float *grad, const void *x, const float *t,
                       const int32_t *idx, int32_t batch, double *loss, void *workspace, int32_t *status, void *stream);
/* One Adam step (lr, beta1 0.9, beta2 0.999, eps 1e-8, step count `step` >= 1) on the batch
 * rows idx (batch) of the standardised pairs (x, t): forward, mean squared error, backward,
 * all on the tensor cores; params (FP32) and params_bf16 updated in place, adam_m / adam_v the
 * moments (FP32, AERO_CLOSURE_NPARAM each), grad (FP32, zero on entry and on return); loss
 * (device double) += the batch's sum of squared errors.  workspace: 256-byte aligned. */
int aero_mlp_train_step(float *params, void *params_bf16, float *adam_m, float *adam_v, float *grad, const void *x,
                        const float *t, const int32_t *idx, int32_t batch, int32_t step, float lr, double *loss,
                        void *workspace, int32_t *status, void *stream);
/* The closure's eddy-viscosity pass on n cells: grad9 (9, n) holds each cell's gradient (g11,
 * g12, g13, g21, g22, g23, g31, g32) and window factor (1 - chi_c); nu (n) holds the WALE nu_t on
 * entry and the closure's nu_t where it applies on return.  nut_max (device, NULL to skip)
 * receives the maximum as the ordered bits of a double; counts (device, 2 x uint64, NULL to skip) adds
 * the cells evaluated and the cells that kept WALE.  delta: the grid spacing. */
int aero_closure_eddy_viscosity(const AeroClosureModel *m, const float *grad9, int64_t n, double delta, float *nu,
                                unsigned long long *nut_max, uint64_t *counts, int32_t *status, void *stream);
/* Cells the last closure step evaluated and cells that kept WALE, summed over its eddy-viscosity
 * passes since the workspace was initialised (reads through a host copy: synchronises). */
int aero_ns3d_closure_counts(const AeroNs3dPlan *plan, const void *workspace, uint64_t out[2], void *stream);

/* Device-side status word of the last step on this workspace (0 = fine; bit 0: a
 * non-finite value reached a reduction; bit 1: a plane load timed out; bit 2: a tensor-core
 * wait of the closure timed out).  Reads through a host copy: synchronises. */
int aero_ns3d_read_status(const AeroNs3dPlan *plan, const void *workspace, int32_t *status, void *stream);
/* Bound of the plane waits of the eddy-viscosity and stage kernels: polls of a plane's barrier
 * before a CTA gives up, sets bit 1 of the status word, lets the copies it issued land and
 * returns with the rest of its chunk unwritten (0: the default, 2^24 polls).
 * test_extra_bytes > 0 is for tests of that bound only: every plane then waits for that many
 * bytes more than its copies bring, so every wait runs out (0 in use; at most 4096).
 * (No counterpart in the reference, which has no bounded waits.) */
int aero_ns3d_set_wait_bound(AeroNs3dPlan *plan, int32_t spin_limit, int32_t test_extra_bytes);

/* The checked build (libaero_b200_checked.so, compiled with AERO_BOUNDS_CHECK) records the
 * first out-of-range shared- or global-memory index a kernel would have used -- (code, index,
 * bound, block << 32 | thread) -- and skips that access.  Synchronising read that also clears
 * the record; in the release library it returns AERO_EUNSUPPORTED.  (No counterpart in the reference: a debugging hook.) */
int aero_debug_check(int64_t *out4);

/* ---- 2D step ----------------------------------------------------------------------- */

typedef struct AeroNs2dPlan AeroNs2dPlan;

/* Everything a 2D step needs besides the fields (ns2d/core.py:67-108 Ops).  Arrays are
 * C-contiguous (ny, nx) with the staggered shapes of ns2d/core.py:9-12: u (ny, nx+1),
 * v (ny+1, nx), p / dye (ny, nx). */
typedef struct {
  int32_t abi_version;          /* AERO_ABI_VERSION                                        */
  int32_t dtype;                /* AERO_F32 or AERO_F64                                    */
  int32_t nx, ny;               /* cells, >= 4 each                                        */
  double h;                     /* cell size                                               */
  int32_t periodic;             /* both axes periodic (core.py:80)                         */
  int32_t closed;               /* walls on all four sides (core.py:102)                   */
  int32_t advection;            /* AERO_ADV_*                                              */
  int32_t les;                  /* AERO_LES_*                                              */
  double les_c;                 /* model constant                                          */
  double nu;                    /* 1 / Re                                                  */
  double eta;                   /* Brinkman permeability                                   */
  double cfl;
  int32_t has_dt_fixed;
  double dt_fixed;
  int32_t ghost_kind[2][2][2];  /* [u, v][x, y][lo, hi] : AERO_GHOST_* (core.py:284-325)    */
  double ghost_val[2][2][2];    /* wall speed of AERO_GHOST_AFFINE                         */
  double force_ref;             /* coefficients = F / (0.5 force_ref)                      */
  int32_t window[4];            /* body cell window j0, j1, i0, i1 (empty: no bodies)      */
  int32_t nbody;                /* <= AERO_MAX_BODIES                                      */
  int32_t dye;                  /* advect the dye after the step                           */
  /* heat transfer (ns2d/physics.py:305-322, 623-923; thermal = 0: off) */
  int32_t thermal;
  double kappa, ri, prt;        /* 1 / Pe, Richardson number, turbulent Prandtl number    */
  double gravity[2];            /* unit gravity direction (x, y)                           */
  double eta_t, theta_in;       /* thermal permeability, inlet temperature                 */
  int32_t wall_mode[4];         /* AERO_TH2_* of the left, right, bottom, top sides        */
  double wall_value[4];         /* wall temperature (TEMPERATURE / INLET) or gradient G    */
  double diff_coef;             /* largest diffusion coefficient (physics.py:833-848)      */
  int32_t n_temp, n_flux;       /* temperature bodies, heat-flux bodies                    */
  int32_t has_ins, has_vol;     /* insulation factors / area fractions present             */
  /* placed physics besides heat transfer (ns2d/physics.py:70-140): actuator-strip fans with
   * their PI controllers (<= AERO_MAX_FANS), heaters (thermal plans), a paint layer of drawn
   * obstacles, the PID-controlled step (diagnostics.py:104-124); their fields are in
   * AeroNs2dGeom, the controller memory in AeroNs2dFields */
  int32_t nfan, heaters, paint, pid;
  int32_t ports;                /* jets and vents (physics.py:362-433)                      */
  /* smoke channels with emitter groups and smoking jets (physics.py:497-540, 805-830; 0: the
   * single comb channel of `dye`): channels (<= AERO_MAX_DYE_CHANNELS; channel 0 is dye, the
   * others dye_extra), emitter groups (<= AERO_MAX_DYE_GROUPS) and the channel of each */
  int32_t dye_channels, n_groups;
  int32_t group_channel[8];
  /* the Werner-Wengle shear on the no-slip domain walls (core.py:505-564): bit 0 bottom, 1 top,
   * 2 left, 3 right (0: off); the floor's speed when the bottom moves */
  int32_t wall_model;
  double wall_ground_speed;
  /* a uniform body force added to the tendencies (the verification cases' ops.forcing,
   * core.py:597-599; forcing = 0: none) */
  int32_t forcing;
  double force[2];
} AeroNs2dConfig;

#define AERO_MAX_DYE_CHANNELS 4
#define AERO_MAX_DYE_GROUPS 8

/* temperature boundary modes of a 2D side (ns2d/scalar.py:96-146) */
enum { AERO_TH2_ADIABATIC = 0, AERO_TH2_TEMPERATURE = 1, AERO_TH2_HEAT_FLUX = 2, AERO_TH2_INLET = 3,
       AERO_TH2_OUTLET = 4, AERO_TH2_PERIODIC = 5 };

/* Window masks (geometry.py:160-178) and boundary profiles, device pointers. */
typedef struct {
  const void *chi_u, *chi_v, *chi_c;  /* (wy, wx+1), (wy+1, wx), (wy, wx)                  */
  const void *a_u, *a_v;              /* solid velocity times chi                           */
  const void *k_u, *k_v;              /* (nbody, 2, ...): [force weight, moment weight]     */
  const void *u_inlet;                /* (ny) inlet u (tunnel)                              */
  const void *dye_inlet;              /* (ny) inlet dye comb, or NULL for zeros             */
  /* heat transfer on the same window (ns2d/geometry.py:120-158): temperature bodies'
   * chi_t, a_t (wy, wx) and shares w_t (n_temp, wy, wx); insulation ins_u (wy, wx+1),
   * ins_v (wy+1, wx); heat-flux skins q_skin (wy, wx) and weights w_f (n_flux, wy, wx);
   * area fractions vol_u, vol_v for the buoyancy share */
  const void *chi_t, *a_t, *w_t, *ins_u, *ins_v, *q_skin, *w_f, *vol_u, *vol_v;
  /* the reference's live 0-d device scalars ops.nu, ops.eta, phys.kappa, phys.eta_t
   * (ns2d/core.py:167-176 set_reynolds fills them in place while a captured graph stays
   * valid), read by every launch; NULL: the config's nu, eta, kappa, eta_t */
  const void *nu, *eta, *kappa, *eta_t;
  /* placed physics (the reference's Physics tensors, read at every launch, plan dtype):
   * fans: force per unit thrust fan_gu (nfan, ny, nx+1), fan_gv (nfan, ny+1, nx), averaging
   * weight fan_phi (nfan, ny, nx), direction fan_dir (nfan, 2), and per fan value, width,
   * kp, ki, dpmax, isvel, isthrust (nfan); the sources' speed floor u_floor (0-d);
   * heaters: density heat (ny, nx) and its maximum heat_max (0-d); paint: paint_c (ny, nx),
   * paint_u (ny, nx+1), paint_v (ny+1, nx) and their force weights paint_wu, paint_wv */
  const void *fan_gu, *fan_gv, *fan_phi, *fan_dir, *fan_value, *fan_width, *fan_kp, *fan_ki, *fan_dpmax,
      *fan_isvel, *fan_isthrust, *u_floor;
  const void *heat, *heat_max;
  const void *paint_c, *paint_u, *paint_v, *paint_wu, *paint_wv;
  /* jets and vents, with paint the combined penalisation: xchi_u, xa_u (ny, nx+1), xchi_v,
   * xa_v (ny+1, nx) (paint alone: xchi = paint, xa NULL); the ports' mass source src and the
   * vents' sinks src_neg (ny, nx), their net volume flow q_net (0-d), the jets' temperature
   * penalisation pt_chi, pt_a (ny, nx; NULL without heat transfer or jets) */
  const void *xchi_u, *xa_u, *xchi_v, *xa_v, *src, *src_neg, *q_net, *pt_chi, *pt_a;
  /* smoke channels: inlet values (dye_channels, ny) (NULL: zeros); per emitter group its
   * weight and target (ny, nx) and timing [start, stop, period, duty]; per channel the smoking
   * jets' weight (ny, nx) or NULL */
  const void *dye_inflow;
  const void *group_w[8], *group_target[8], *group_timing[8];
  const void *port_dye[4];
} AeroNs2dGeom;

/* Step inputs (u0, v0, t0, dye0) and outputs; u / v may alias u0 / v0. */
typedef struct {
  const void *u0, *v0, *t0, *dye0;
  void *u, *v, *p, *t, *dt, *dye;
  void *coeffs;                       /* (nbody, 3): Cd, Cl, Cm                             */
  /* heat transfer: theta in / out (ny, nx; may alias) and the step's heat report
   * (ns2d/core.py:974-995), all double: heat of each temperature body (n_temp), wall
   * temperature of each heat-flux body (n_flux), wall heat of the left, right, bottom and
   * top sides (4), heat storage (1), flow heat in at the inlet / out at the outlet (2) */
  const void *theta0;
  void *theta, *heat, *theta_wall, *wall_heat, *heat_storage, *flow_heat;
  /* placed physics (plan dtype): the previous step's dt (0-d; <= 0: first step) and the
   * controller memory in / out (2 + 2 nfan: the PID's last two errors, then per fan its
   * integral and pressure jump; core.py State.ctrl); out: the fans' thrust and disc velocity
   * (nfan each) and the painted obstacles' force coefficients [Cd, Cl] (2) */
  const void *dt_prev, *ctrl0;
  void *ctrl, *fan_thrust, *fan_ud, *paint_force;
  /* jets and vents with heat transfer (double, 1 each): the heat the jets add and the heat
   * leaving with the vents' fluid (core.py:990-993) */
  void *jet_heat, *vent_heat;
  /* smoke channels 1 .. dye_channels - 1 in and out ((dye_channels - 1, ny, nx); channel 0 is
   * dye0 / dye) */
  const void *dye_extra0;
  void *dye_extra;
} AeroNs2dFields;

int aero_ns2d_plan_create(const AeroNs2dConfig *cfg, AeroNs2dPlan **plan);
void aero_ns2d_plan_destroy(AeroNs2dPlan *plan);
size_t aero_ns2d_workspace_bytes(const AeroNs2dPlan *plan);
int aero_ns2d_workspace_init(const AeroNs2dPlan *plan, void *workspace, void *stream);

/* One SSP-RK3 step (dt_in NULL: the CFL / viscous rule on the device, else a device scalar),
 * then the dye update when the plan has dye. */
int aero_ns2d_step(const AeroNs2dPlan *plan, const AeroNs2dFields *f, const AeroNs2dGeom *g, const void *dt_in,
                   void *workspace, void *stream);

/* psi with L psi = f, zero mean ((ny, nx) device arrays; may alias). */
int aero_ns2d_poisson_solve(const AeroNs2dPlan *plan, const void *f, void *psi, void *workspace, void *stream);

/* ---- the batched sweep: many 2D instances in one persistent launch ---------------------
 * No counterpart in the reference, which steps its solver once per instance (ns2d/solver.py:489
 * advance, core.py:815 step_full each).  A sweep records the step of each instance (plan,
 * fields, geometry, workspace: the arguments of aero_ns2d_step, bound at creation, like a
 * captured graph) as its sequence of operations, and aero_ns2d_sweep_step runs all of them in
 * one persistent cooperative kernel: the CTAs (co-resident, as many per SM as the tuning asks
 * and the kernel allows) take the work items of all instances' operations, numbered phase by
 * phase (phase p: operation p of every instance).  Every instance's result is bit-identical to
 * its own aero_ns2d_step.  FP32 plans without LES, heat transfer or dye, with the CFL time step,
 * transform lengths of at least 64.  Tuning: lcap the log2 of the widest compile-time transform
 * tile in lines (2..3), ctas_per_sm (1..4; 3 and 4 compile the kernel for fewer registers per thread),
 * order 0 (the instances' order) or 1 (largest first), schedule 0 (a grid barrier between
 * phases), 1 (no barriers: an item waits until its own instance has finished its earlier
 * operations, items dealt round robin to the CTAs) or 2 (as 1, the CTAs taking items from a
 * queue), tiles (1..16) the stage or transform tiles one work item runs. */
typedef struct AeroNs2dSweep AeroNs2dSweep;
typedef struct {
  int32_t lcap, ctas_per_sm, order, schedule, tiles;
} AeroSweepTuning;
int aero_ns2d_sweep_create(int32_t n, const AeroNs2dPlan *const *plans, const AeroNs2dFields *fields,
                           const AeroNs2dGeom *geoms, void *const *workspaces, const AeroSweepTuning *tuning,
                           AeroNs2dSweep **sweep);
void aero_ns2d_sweep_destroy(AeroNs2dSweep *sweep);
/* Device bytes of the sweep's operation tables (256-byte aligned workspace). */
size_t aero_ns2d_sweep_workspace_bytes(const AeroNs2dSweep *sweep);
/* Upload the tables into the workspace (synchronises the stream once). */
int aero_ns2d_sweep_init(const AeroNs2dSweep *sweep, void *workspace, void *stream);
/* One step of every instance: one persistent launch (capturable in a CUDA graph). */
int aero_ns2d_sweep_step(const AeroNs2dSweep *sweep, void *workspace, void *stream);
/* Status word since the last read (bit 0: a grid barrier or an instance wait ran out; the
 * launch then stopped); synchronises, then clears it. */
int aero_ns2d_sweep_read_status(const AeroNs2dSweep *sweep, void *workspace, int32_t *status, void *stream);
/* The bound of the waits (polls before giving up) and, for tests of that bound, extra arrivals
 * (barrier) or finished items (instance waits) to wait for that never come (0 in use). */
int aero_ns2d_sweep_set_barrier(AeroNs2dSweep *sweep, int32_t spin_limit, int32_t extra);
/* [phases, operations, work items per step, CTAs, dynamic shared bytes, lcap] */
int aero_ns2d_sweep_info(const AeroNs2dSweep *sweep, int64_t out[6]);

#ifdef __cplusplus
}
#endif
#endif /* AERO_B200_H */
