/*
 * apollo_dg.h — C ABI of the B200 nodal-DG right-hand side and SSP Runge–Kutta
 * stepper.  Plain pointers and sizes only; the library owns every device buffer
 * it allocates and the caller frees nothing of it.
 *
 * State layout at this boundary is Apollo's: per element, node-major then field,
 * U[k][node][field] in float64 (src/subsolvers/wxnodaldg2dmethod.cc:199,330-332).
 *
 * Reference interfaces each entry point stands in for (paths inside Apollo):
 *   apollo_dg_create / set_equation / add_bc / set_mesh
 *        WxNodalDG2dMethod<REAL>::setup(wxc, DM)  src/subsolvers/wxnodaldg2dmethod.cc:50-152
 *        with WxHyperbolicEqnSet::setup            src/hyper/wxhyperboliceqnset.cc:43-89
 *        and the geometry/cubature constructors    src/lib/wxnodaldggeometry2d.cc:10-107,
 *                                                   src/lib/wxcubature2d.cc:10-169
 *   apollo_dg_init_dt
 *        WxNodalDG2dMethod<REAL>::init(dt, Vec)     src/subsolvers/wxnodaldg2dmethod.cc:154-233
 *   apollo_dg_rhs
 *        WxNodalDG2dMethod<REAL>::step(t, dt, in, out) -> WxStepperStatus{status, suggestedDt}
 *                                                   src/subsolvers/wxnodaldg2dmethod.cc:235-542
 *   apollo_dg_step
 *        WxPetscTimeSteppingSolver::solve (TSSSP)  src/subsolvers/wxpetsctimestepping.h:69-101
 *        with ApSolver::ComputeRHSforTS/MonitorVTK src/solvers/apsolver.cc:421-480
 *   apollo_dg_destroy
 *        WxNodalDG2dMethod<REAL>::~WxNodalDG2dMethod src/subsolvers/wxnodaldg2dmethod.cc:18-45
 */
#ifndef APOLLO_DG_H
#define APOLLO_DG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct apollo_dg apollo_dg;

/* Return codes.  The reference calls exit(1) where these are returned. */
typedef enum {
  APOLLO_OK = 0,
  APOLLO_ERR_CONFIG = 1,      /* unknown kind, bad parameter, unsupported order */
  APOLLO_ERR_MESH = 2,        /* non-positive Jacobian or edge length, bad connectivity */
  APOLLO_ERR_NONPHYSICAL = 3, /* rho <= 0 or p <= 0 in the Euler flux with no floor set */
  APOLLO_ERR_NAN = 4,         /* NaN in a right-hand side */
  APOLLO_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
  APOLLO_ERR_CUDA = 6,        /* a CUDA runtime call failed */
  APOLLO_ERR_STATE = 7,       /* call out of order (no mesh, no equation, no state) */
  APOLLO_ERR_ARG = 8,         /* null pointer or size out of range */
  APOLLO_ERR_ALLOC = 9        /* device allocation failed */
} apollo_status;

/* Arithmetic of the right-hand side.  The state, the stage accumulation, the
 * dt reduction and the conserved sums stay float64 in every form. */
typedef enum {
  APOLLO_PREC_FP64 = 0,  /* plain float64 path */
  APOLLO_PREC_MIXED = 1  /* tensor-core contractions with split operands, fp32 accumulation */
} apollo_precision;

/* Pointer location flags for apollo_dg_rhs / set_state / get_state. */
#define APOLLO_HOST_PTR 0
#define APOLLO_DEVICE_PTR 1

typedef struct {
  int polynomial_order; /* N; kernels exist for N = 2..5 ("polynomialOrder") */
  double cfl;           /* "cfl" */
  int device;           /* CUDA device ordinal */
  void* stream;         /* cudaStream_t to run on; NULL = a stream owned by the handle */
} apollo_dg_config;

/* Setup -------------------------------------------------------------------- */
apollo_status apollo_dg_create(const apollo_dg_config* cfg, apollo_dg** out);

/* Equation plugin by Apollo kind name, parameters in the order listed:
 *   "advectionEqn"  ux, uy, uz                     (1 field)
 *   "eulerEqn"      gas_gamma, minPressure, minDensity   (5 fields: rho, rhou, rhov, rhow, E)
 *   "phMaxwellEqn"  c0, gamma, chi                 (8 fields: Ex, Ey, Ez, Bx, By, Bz, phi, psi)
 * and two planar forms of the same equations (an extension; identical
 * arithmetic when the dropped fields are zero):
 *   "eulerEqn2d"    gas_gamma, minPressure, minDensity   (4 fields: rho, rhou, rhov, E)
 *   "maxwellTM"     c0                             (3 fields: Ez, Bx, By)
 * Numerical flux: Lax-Friedrichs unless apollo_dg_set_numerical_flux says otherwise. */
apollo_status apollo_dg_set_equation(apollo_dg* h, const char* kind, const double* params, int nparams);

/* ---- Apollo input-deck text.  Apollo configures this sub-solver from the
 * cryptset blocks of its .pin input deck (WxNodalDG2dMethod::setup,
 * src/subsolvers/wxnodaldg2dmethod.cc:50-152, and WxHyperbolicEqnSet::setup,
 * src/hyper/wxhyperboliceqnset.cc:43-89): the nodalDG2d block's
 * polynomialOrder and cfl, and the lists Equations, boundaryConditions and
 * Limiter naming blocks whose Kind and keys configure each plugin.  These
 * calls take that text (a whole deck, or one block) with Apollo's key names
 * and defaults; the deck's Python preamble of "NAME = expression" lines may be
 * included, and values may be arithmetic over those names.  As in Apollo's
 * reader, a key written after a sub-block of its block is not read, and of a
 * key written twice the first counts.  With kind NULL
 * the block is found through the list (or is the text's only block); with a
 * kind, the text's keys are that plugin's.  Errors: APOLLO_ERR_CONFIG with the
 * reason in err (host-only calls) or apollo_dg_last_error. */
/* Host only: polynomial_order and cfl of the nodalDG2d block into *cfg (the
 * device and stream fields are left as they are). */
apollo_status apollo_dg_deck_config(const char* text, apollo_dg_config* cfg, char* err, int err_len);
/* Host only: the equation block as apollo_dg_set_equation's kind and
 * params[nparams] (at most 8), and its Numerical_Flux ("LF" if absent). */
apollo_status apollo_dg_deck_equation(const char* kind, const char* text, char* kind_out, int kind_len,
                                      double* params, int* nparams, char* flux_out, int flux_len, char* err,
                                      int err_len);
/* Host only: *count receives the number of boundary conditions the deck
 * lists (the boundaryConditions of the block holding Equations; a text
 * without Equations is one condition's block); entry `index` (if below
 * *count) as apollo_dg_add_bc's kind and params. */
apollo_status apollo_dg_deck_bc(const char* kind, const char* text, int index, int* count, char* kind_out,
                                int kind_len, double* params, int* nparams, char* err, int err_len);
/* Host only: *count receives the number of sources the deck lists (the
 * Sources of the block holding Equations; a text without Equations is one
 * source's block); entry `index` as apollo_dg_add_source's kind, out_range[nout]
 * (at most 8) and params. */
apollo_status apollo_dg_deck_source(const char* kind, const char* text, int index, int* count, char* kind_out,
                                    int kind_len, int* out_range, int* nout, double* params, int* nparams, char* err,
                                    int err_len);
/* Host only: the first block of the deck's Limiter list as
 * apollo_dg_set_limiter's kind and params (kind_out "" when there is none). */
apollo_status apollo_dg_deck_limiter(const char* kind, const char* text, char* kind_out, int kind_len,
                                     double* params, int* nparams, char* err, int err_len);
/* The same, applied to a handle: apollo_dg_set_equation (+ the numerical
 * flux), apollo_dg_add_bc for every listed condition in order,
 * apollo_dg_add_source for every listed source, and apollo_dg_set_limiter
 * (removed when the deck lists none). */
apollo_status apollo_dg_set_equation_text(apollo_dg* h, const char* kind, const char* text);
apollo_status apollo_dg_add_bc_text(apollo_dg* h, const char* kind, const char* text);
apollo_status apollo_dg_add_source_text(apollo_dg* h, const char* kind, const char* text);
apollo_status apollo_dg_set_limiter_text(apollo_dg* h, const char* kind, const char* text);

/* Euler numerical flux by Apollo's "Numerical_Flux" name (WxEulerEqn::setup,
 * src/hyperapps/euler/wxeulereqn.cc:45-87): "LF" (default), "HLL", "Roe",
 * "Wave"; any other name selects LF, as Apollo does (the call succeeds and
 * apollo_dg_last_error says so).  The fluxes reproduce Apollo's arithmetic,
 * including its HLL bound |S_R| truncated to an integer, its Roe flux's
 * y-momentum component of 0 and x-momentum component set from the rotated
 * y-momentum flux, and Wave's fall-through to LF on rotated traces.
 * "advectionEqn" takes "LF" (Apollo's, dissipation max(|ux|, |uy|)) or the
 * extension "upwind" (dissipation |n.u|, the exact upwind flux; the dt
 * policy keeps Apollo's speed).  "maxwellTM" takes "LF" (Apollo's,
 * dissipation c0 on every field) or the extension "upwind" (the exact upwind
 * flux: no dissipation on the normal magnetic field, whose wave speed is 0).
 * "phMaxwellEqn" has only LF (the name is ignored).
 * Mixed precision and the derivatives (tangent and adjoint) take every one
 * of them. */
apollo_status apollo_dg_set_numerical_flux(apollo_dg* h, const char* name);

/* Limiter applied to every stage input before its right-hand side, as
 * WxNodalDG2dMethod::step does (src/subsolvers/wxnodaldg2dmethod.cc:243-247,
 * "Limiter = [...]").  kind "eulerLimiterHW" (WxHestavenWarburtonEulerLimiter,
 * src/hyperapps/euler/wxhesthavenwarburtoneulerlimiter.cc) with params
 * gas_gamma, min_pressure, min_density, Euler kinds only; or kind
 * "tuAliabadiLimiter" (WxTuAliabadiLimiter,
 * src/hyperapps/multifluid/aptualiabadilimiter.cc) with no params: Euler kinds
 * with the equation's own gas_gamma, minPressure, minDensity and its
 * primitive-variable floors, and the Maxwell kinds, whose nodes it sets to the
 * element averages (advection has no such hook in Apollo).  NULL or "" removes
 * the limiter.  Call after apollo_dg_set_mesh and the boundary conditions.
 * Orders 2..4 (at order 5 Apollo reads past its face-average array); for the
 * Euler kinds, boundary conditions that read no time or position (wall, zero
 * gradient, inflow, Dirichlet, fixed), since Apollo's limiters hand them
 * none.  apollo_dg_step
 * limits each stage's work state (the step's solution is combined unlimited,
 * as in PETSc's SSP stepper); apollo_dg_rhs limits a copy of its input.
 * In mixed precision the stepper also rebuilds the fp32 face traces of each
 * limited stage input.  Partitioned meshes and the derivatives refuse it
 * (APOLLO_ERR_CONFIG). */
apollo_status apollo_dg_set_limiter(apollo_dg* h, const char* kind, const double* params, int nparams);

/* Launch and tile shape of this handle's kernels, as the batch autotuner
 * picks them (apollo_dg_batch_autotune): the persistent grids use
 * SMs / grid_share CTAs; tile_shape selects the mixed stage kernel:
 *   0  the fused kernel (whole flux-deviation operand of a tile in shared
 *      memory, tensor-core face traces) where it applies: "eulerEqn2d" with
 *      the Lax-Friedrichs flux at orders 2..4; elsewhere as 2
 *   1  the chunked kernel with 16-column operand chunks in three buffers
 *   2  the chunked kernel with 24-column chunks (16 at order 5) in two buffers
 * 1 and 2 compute the same result bit for bit (the same MMAs in the same K
 * order); 0 agrees with them within the mixed form's error.  No counterpart
 * in Apollo. */
apollo_status apollo_dg_set_launch_shape(apollo_dg* h, int grid_share, int tile_shape);

/* Float64 stage kernels of this handle.  0 (the default): the volume, face
 * and LIFT kernels.  1: the fused stage kernel (the volume and surface terms
 * and the stage update of a tile of elements in one pass, each element
 * evaluating its own faces as Apollo does, DRAM traffic near the compulsory
 * bytes) wherever it applies: a whole mesh, no source plugins, and a stage
 * whose output does not overlap its input.  2: the fused kernel where the
 * mesh's tiles fit about one wave of resident blocks (small meshes, where
 * three launches cost more than the work), the three kernels elsewhere (the
 * face kernel evaluates each face once, which a per-element pass cannot).
 * The forms agree within float64 round-off, not bit for bit, so the default
 * keeps every handle (whole, partitioned, batched) on the same arithmetic. */
apollo_status apollo_dg_set_fp64_kernels(apollo_dg* h, int fused);

/* The element average of a nodal field is sum_n w[n] u[n]: w[Np] receives the
 * weights (half the column sums of the reference mass matrix, Apollo's
 * LimiterElementAVE, src/lib/wxnodaldggeometry2d.h:84-98). */
apollo_status apollo_dg_averaging_weights(const apollo_dg* h, double* w);

/* Source plugin, appended to the equation's source set (WxHyperbolicSrcSet,
 * src/hyper/wxhyperbolicsrcset.cc:16-71; "Sources = [...]"), for the kinds
 * whose value depends on time and position only:
 *   "tranverseMagneticSrc"   (no params; Apollo's spelling)
 *        s = exp(t) (x (1-x) y (1-y) + 2 x (1-x) + 2 y (1-y))
 *        (src/hyperapps/maxwell/wxtransversemagneticsrc.h:37-44)
 *   "pointCurrentSrc"        xLocation, yLocation, radius, currentDensity,
 *        frequency, phase, charge, mass, epsilon0: s = j0 q/(m eps0)
 *        sin(omega t + phase) within radius of (x, y), 0 elsewhere
 *        (src/hyperapps/maxwell/wxpointcurrent.h)
 * out_range[nout]: the plugin's OutRange; its first entry is the field (in
 * Apollo's numbering of the full equation: Ez of phMaxwellEqn is 2, also for
 * "maxwellTM") that the source adds into.  As in Apollo the source is
 * evaluated at the cubature points at the stage time and enters the volume
 * term as V^T (w J S); every form (float64, mixed precision, partitioned,
 * derivatives, the no-allocation right-hand side) includes it.  Up to 4
 * sources; apollo_dg_set_equation clears them. */
apollo_status apollo_dg_add_source(apollo_dg* h, const char* kind, const int* out_range, int nout,
                                   const double* params, int nparams);

/* Boundary-condition plugin, appended to the list; a face tagged t uses the
 * t-th condition added (Apollo's boundaryConditions[t-1]).  Kinds and params:
 *   "gridFixedBC"                   value
 *   "isentropicVortexBC"            u0, v0, x0, y0, gas_gamma, beta
 *   "maxwellTransverseMagneticBC"   (none)
 *   "phmConductingWallBC"           (none)
 *   "eulerWallBC"                   (none)      normal momentum reflected
 *   "eulerZeroGradientBC"           (none)      interior state
 *   "eulerInflowBC"                 Mach_number, Flow_angle (degrees), gas_gamma, Pressure, density
 *   "eulerDirichletBC"              density, xvelocity, yvelocity, zvelocity, gas_gamma, pressure  */
apollo_status apollo_dg_add_bc(apollo_dg* h, const char* kind, const double* params, int nparams);

/* Mesh: vertices (vx, vy), counter-clockwise triangles etov[K][3] (vertex 0 ->
 * reference (-1,-1), 1 -> (1,-1), 2 -> (-1,1)); face_tag[K][3]: 0 = pair with
 * the face sharing both vertices (or, if none, boundary condition 1), t > 0 =
 * boundary condition t; vert_canon[nverts]: canonical vertex id used for
 * pairing (periodic identification), may be NULL.  Builds geometry, face map
 * and operators on the device. */
apollo_status apollo_dg_set_mesh(apollo_dg* h, int nverts, const double* vx, const double* vy, int K,
                                 const int* etov, const int* face_tag, const int* vert_canon);

/* Sizes: fields per node, nodes per element, elements, cubature points, Gauss
 * points per face. */
int apollo_dg_num_fields(const apollo_dg* h);
int apollo_dg_num_nodes(const apollo_dg* h);
int apollo_dg_num_elements(const apollo_dg* h);
int apollo_dg_num_cubature(const apollo_dg* h);
int apollo_dg_num_gauss(const apollo_dg* h);

/* Physical node coordinates x, y [K][Np] into host memory. */
apollo_status apollo_dg_node_coords(apollo_dg* h, double* x, double* y);

/* Resident state U [K][Np][m]: copy in / out (host or device pointer). */
apollo_status apollo_dg_set_state(apollo_dg* h, const double* U, int where);
apollo_status apollo_dg_get_state(apollo_dg* h, double* U, int where);

/* The same copies queued on the handle's stream, returning at once (no
 * counterpart in Apollo, whose state is a host-side PETSc Vec).  The caller
 * orders them against its own streams (a handle created on the caller's
 * stream, or apollo_dg_synchronize) and keeps U untouched until the stream
 * has passed the copy; a host U must be page-locked for the copy to be
 * asynchronous.  Together with apollo_dg_step_async they let independent
 * states stream through one handle without a host wait per step. */
apollo_status apollo_dg_set_state_async(apollo_dg* h, const double* U, int where);
apollo_status apollo_dg_get_state_async(apollo_dg* h, double* U, int where);

/* Initial dt from the resident state: 2/3 cfl dtscale rmin / max wave speed,
 * wave speeds from the Riemann solver at every node. */
apollo_status apollo_dg_init_dt(apollo_dg* h, double* dt);

/* One right-hand-side evaluation out = L(in) at time t (dt is passed to the
 * boundary hooks as Apollo does).  in/out are [K][Np][m], host or device
 * pointers per `where`; suggested_dt (may be NULL) receives
 * 2/3 cfl dtscale rmin / max numerical-flux speed. */
apollo_status apollo_dg_rhs(apollo_dg* h, double t, double dt, const double* in, double* out,
                            double* suggested_dt, int where, apollo_precision prec);

/* Advance the resident state by up to nsteps SSPRK(5,2) steps (PETSc TSSSP
 * default), starting at *t with step *dt.  After each step the next dt is
 * min(dt, suggestion of the last stage), clipped so t does not pass tend
 * (tend <= 0: no end time).  On return *t and *dt hold the time reached and
 * the dt for the next step.  With tend <= 0 the steps are queued without host
 * synchronisation (one CUDA graph per step); the call returns after the last
 * step completes. */
apollo_status apollo_dg_step(apollo_dg* h, int nsteps, double* t, double* dt, double tend, apollo_precision prec);

/* Same as apollo_dg_step but returns as soon as the work is queued on the
 * handle's stream; *t and *dt are not updated (read them with
 * apollo_dg_get_time after apollo_dg_synchronize). */
apollo_status apollo_dg_step_async(apollo_dg* h, int nsteps, double t, double dt, apollo_precision prec);
apollo_status apollo_dg_get_time(apollo_dg* h, double* t, double* dt);
apollo_status apollo_dg_synchronize(apollo_dg* h);

/* Per-field sums of the element integrals of U (M J U summed), float64. */
apollo_status apollo_dg_integrals(apollo_dg* h, const double* U, int where, double* sums);

/* Per-field sums of the element integrals of U^2 (J u^T Mref u summed, with
 * Mref = (V V^T)^-1 the reference mass matrix whose inverse Apollo keeps as VVT,
 * src/lib/wxnodaldggeometry2d.cc:71-75), float64: the electromagnetic energy
 * of the Maxwell TM fields is half the sum over Ez, Bx, By.  U as in
 * apollo_dg_integrals (NULL: the resident state).  Apollo has no such sum; it
 * serves the energy-drift check of the cavity mode. */
apollo_status apollo_dg_energy(apollo_dg* h, const double* U, int where, double* sums);

/* Diagnostics: average device time in milliseconds of each kernel of one
 * right-hand side, over `iters` evaluations of the resident state (CUDA events
 * on the handle's stream).  ms[0..2] = volume, face, LIFT + update.  *nk
 * receives the number of kernels timed. */
apollo_status apollo_dg_kernel_times(apollo_dg* h, apollo_precision prec, int iters, double* ms, int* nk);

/* The float64 right-hand side for callers that cannot allocate device memory
 * when they evaluate it (a host framework that owns all device memory through
 * its own allocator and forbids allocations behind its back, or a loop that
 * must not take the device-wide synchronisation of cudaMalloc).  No counterpart
 * in Apollo.  Same result as apollo_dg_rhs with APOLLO_PREC_FP64 on device
 * pointers; the kernels' scratch (volume term, face traces, face fluxes) lives
 * in a 64 MiB static device array that every GPU loading this library holds
 * until the process exits, so this call allocates nothing.  The handle itself
 * was built (and allocated) by apollo_dg_create / apollo_dg_set_mesh.
 *   in, out       device pointers [K][Np][m], distinct
 *   suggested_dt  may be NULL; when given, the call waits for the stream and
 *                 reports non-physical states and NaN like apollo_dg_rhs.
 *                 With NULL the call does not wait and reports no such
 *                 status: a NaN or non-physical state goes unreported, and
 *                 the next call clears the evidence
 *   stream        cudaStream_t to run on (NULL: the legacy default stream)
 * Meshes whose scratch exceeds 64 MiB ((Np + 6 (N + 1) * 2) * m * 8 bytes per
 * element, about 28,000 elements at N = 4 with 4 fields) are rejected with
 * APOLLO_ERR_ARG.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture.  All calls share the one array: calls that overlap on the GPU, on
 * any handle or stream of the same device, race.  Handles with a limiter
 * (apollo_dg_set_limiter) or a partitioned mesh with peers are refused
 * (APOLLO_ERR_STATE). */
apollo_status apollo_dg_rhs_noalloc(apollo_dg* h, double t, double dt, const double* in, double* out,
                                    double* suggested_dt, void* stream);

/* ---- Derivatives (float64).  No counterpart in Apollo, which has no adjoint.
 * A trajectory here is nsteps SSPRK(5,2) steps of FIXED size dt (the adaptive
 * dt policy of apollo_dg_step is not differentiated); stage times are
 * t0 + n dt + dt {0, 1/4, 1/2, 3/4, 1}, as in apollo_dg_step. */

/* Advance the resident state by nsteps fixed steps, keeping every
 * checkpoint_every-th state on the device (ceil(nsteps / checkpoint_every)
 * states) for apollo_dg_backward. */
apollo_status apollo_dg_forward_fixed(apollo_dg* h, int nsteps, double t0, double dt, int checkpoint_every);

/* The same trajectory with binomial checkpointing (Griewank's revolve):
 * `snapshots` state slots, the initial state's included, of which the forward
 * pass fills those of the schedule's first descent; apollo_dg_backward then
 * re-runs the steps it needs from them, splitting each interval where the
 * total of re-run steps is least (dynamic programming while nsteps^2
 * snapshots / 2 stays under 1.5e8, the binomial rule beyond: beta(c, t) =
 * C(c + t, c) steps need t passes with c free slots).  More snapshots than
 * steps are not allocated.  A second apollo_dg_backward of the same trajectory first
 * re-runs the first descent, whose slots the first sweep reused.  Derivative memory: `snapshots` states and the 5 stage states
 * of one step (the two-level schedule of apollo_dg_forward_fixed holds
 * nsteps / checkpoint_every states and 5 checkpoint_every stage states). */
apollo_status apollo_dg_forward_revolve(apollo_dg* h, int nsteps, double t0, double dt, int snapshots);

/* Host only: the forward steps the backward sweep after
 * apollo_dg_forward_revolve(nsteps, snapshots) runs (each reversed step's
 * own recording included), and how many states the forward pass stores
 * (NULL: not wanted).  APOLLO_ERR_STATE if the schedule failed its own check
 * (every slot holds the step it is used for, steps reversed last to first). */
apollo_status apollo_dg_revolve_schedule(int nsteps, int snapshots, long long* recomputed_steps, int* spine_states);

/* Steps the last apollo_dg_backward re-ran forward (with revolve: its
 * schedule's count; with checkpoints every C steps: nsteps). */
apollo_status apollo_dg_adjoint_stats(const apollo_dg* h, long long* recomputed_steps);

/* Discrete adjoint of the last apollo_dg_forward_fixed trajectory: given
 * ubar_T = dJ/dU(T) (any terminal functional J), writes ubar_0 = dJ/dU(0).
 * Each checkpoint segment is re-run once, keeping its 5 x checkpoint_every
 * stage states; then every stage is reversed with the exact transpose of the
 * float64 right-hand side's linearisation.  [K][Np][m] arrays, host or device. */
apollo_status apollo_dg_backward(apollo_dg* h, const double* ubar_T, double* ubar_0, int where);

/* Forward-mode derivative: advances the resident state by nsteps fixed steps
 * and writes duT = (dU(T)/dU(0)) du0. */
apollo_status apollo_dg_tangent(apollo_dg* h, int nsteps, double t0, double dt, const double* du0, double* duT,
                                int where);

/* One right-hand side's derivatives at the state x (time t):
 * out = L'(x) v (jvp), out = L'(x)^T w (vjp; out distinct from x and w). */
apollo_status apollo_dg_rhs_jvp(apollo_dg* h, double t, const double* x, const double* v, double* out, int where);
apollo_status apollo_dg_rhs_vjp(apollo_dg* h, double t, const double* x, const double* w, double* out, int where);

/* Device bytes held for derivatives (scratch, checkpoints, segment states). */
apollo_status apollo_dg_adjoint_memory(const apollo_dg* h, size_t* bytes);

/* ---- Batched ensembles.  No counterpart in Apollo (one mesh per run there).
 * Many independent meshes of one equation, of any sizes and orders 2..5,
 * advance together: the instances of one order share one discretisation
 * (their elements concatenated, each with its own dt, time, dt policy and
 * wave-speed reduction), each stage is one persistent launch over all of them,
 * and one CUDA graph per step runs the order groups concurrently. */
typedef struct apollo_dg_batch apollo_dg_batch;

apollo_status apollo_dg_batch_create(const apollo_dg_config* cfg, const char* eq_kind, const double* eq_params,
                                     int n_params, apollo_dg_batch** out);
apollo_status apollo_dg_batch_add_bc(apollo_dg_batch* b, const char* kind, const double* params, int n_params);
/* Every instance's Euler numerical flux (apollo_dg_set_numerical_flux's
 * names); before apollo_dg_batch_finalize. */
apollo_status apollo_dg_batch_set_numerical_flux(apollo_dg_batch* b, const char* name);
/* Adds one mesh (the arguments of apollo_dg_set_mesh) of order N; *instance
 * receives its index. */
apollo_status apollo_dg_batch_add_mesh(apollo_dg_batch* b, int N, int nverts, const double* vx, const double* vy,
                                       int K, const int* etov, const int* face_tag, const int* vert_canon,
                                       int* instance);
/* Builds the discretisations; no meshes can be added afterwards. */
apollo_status apollo_dg_batch_finalize(apollo_dg_batch* b);
int apollo_dg_batch_size(const apollo_dg_batch* b);
apollo_status apollo_dg_batch_instance_info(const apollo_dg_batch* b, int inst, int* N, int* K, int* Np, int* fields);
apollo_status apollo_dg_batch_node_coords(const apollo_dg_batch* b, int inst, double* x, double* y);
apollo_status apollo_dg_batch_set_state(apollo_dg_batch* b, int inst, const double* U, int where);
apollo_status apollo_dg_batch_get_state(apollo_dg_batch* b, int inst, double* U, int where);
/* Initial dt of every instance (Apollo's init policy), dt[instances]. */
apollo_status apollo_dg_batch_init_dt(apollo_dg_batch* b, double* dt);
/* nsteps steps of every instance from its own (t[i], dt[i]); both arrays are
 * updated in place (dt policy of apollo_dg_step, no end time). */
apollo_status apollo_dg_batch_step(apollo_dg_batch* b, int nsteps, double* t, double* dt, apollo_precision prec);
/* Times the candidate launch and tile shapes of each order group for this
 * precision and keeps the fastest: the persistent grid's share of the SMs
 * (all, half, a quarter) and, in mixed precision, the stage kernel's operand
 * chunking (0: 24-column chunks, 16 at order 5, in a two-buffer ring; 1:
 * 16-column chunks in a three-buffer ring; the same arithmetic either way).
 * share[4] and shape[4] (either may be NULL) receive the picks per order
 * 2..5 (share 0 and shape -1: order absent). */
apollo_status apollo_dg_batch_autotune(apollo_dg_batch* b, apollo_precision prec, int* share, int* shape);
const char* apollo_dg_batch_last_error(const apollo_dg_batch* b);
apollo_status apollo_dg_batch_destroy(apollo_dg_batch* b);

/* ---- Gmsh 2.2 ASCII meshes (host only).  Replaces PETSc's DMPlexCreateGmsh
 * (src/solvers/apsolver.cc:318-327) and the "Face Sets" labels of
 * wxNodalDGgeometry2D::FacePair2d (src/lib/wxnodaldggeometry2d.cc:334-356).
 * Triangles become cells, oriented counter-clockwise; lines carry the physical
 * tag (their first tag) of a boundary.  An element with a labelled face applies
 * its label to all its unpaired faces, as Apollo does; unpaired faces of
 * unlabelled elements get tag 1 (Apollo's default -1, boundary condition 1);
 * where one element's faces carry different labels, each labelled face keeps
 * its own.  The arrays are apollo_dg_set_mesh's (no periodic map). */
typedef struct apollo_dg_mesh apollo_dg_mesh;
/* err (optional, err_len bytes) receives the reason on failure. */
apollo_status apollo_dg_mesh_read_gmsh(const char* path, apollo_dg_mesh** out, char* err, int err_len);
apollo_status apollo_dg_mesh_info(const apollo_dg_mesh* m, int* nverts, int* K);
/* vx, vy [nverts], etov [K][3], face_tag [K][3]; NULL arrays are skipped. */
apollo_status apollo_dg_mesh_arrays(const apollo_dg_mesh* m, double* vx, double* vy, int* etov, int* face_tag);
apollo_status apollo_dg_mesh_destroy(apollo_dg_mesh* m);

/* ---- Partitioned meshes (one handle per rank, one rank per GPU).  Replaces
 * Apollo's PETSc DMPlex distribution with an overlap-1 halo refreshed by
 * DMGlobalToLocal before every right-hand side (src/solvers/apsolver.cc:318-392)
 * and its MPI_Allreduce of the dt estimate (apsolver.cc:431-433): here only the
 * face traces of cut faces cross between ranks, once per stage, and the
 * caller's communicator (NCCL, MPI, ...) moves them.
 *
 * Host-only calls (no device needed): */
/* Recursive coordinate bisection of the element centroids: part[K] receives
 * a rank in 0..nparts-1 per element, parts within one element of K/nparts. */
apollo_status apollo_dg_partition(int nverts, const double* vx, const double* vy, int K, const int* etov,
                                  int nparts, int* part);

typedef struct {
  int n_local;  /* elements owned by the rank */
  int n_ghost;  /* remote elements sharing a face with a local one */
  int n_peers;  /* ranks exchanged with */
  int n_send;   /* trace blocks sent per stage (one per cut face) */
  int n_recv;   /* trace blocks received per stage */
} apollo_dg_halo_sizes;

/* The halo plan of one rank of the global mesh (apollo_dg_set_mesh's mesh
 * arguments) under the partition part[K].  Fills *sizes; each array that is
 * not NULL receives: local_elems[n_local] and ghost_elems[n_ghost] (global
 * element ids), peers[n_peers] (ascending), send_count / recv_count[n_peers]
 * (blocks per peer), send_faces[n_send] (global face id 3k+f of the local side
 * of each block sent, peer-major) and recv_faces[n_recv] (global face id of the
 * remote side of each block received).  Within one peer, blocks go in
 * ascending order of the sending side's face id, on both ranks. */
apollo_status apollo_dg_halo_plan(int nverts, int K, const int* etov, const int* face_tag, const int* vert_canon,
                                  const int* part, int rank, apollo_dg_halo_sizes* sizes, int* local_elems,
                                  int* ghost_elems, int* peers, int* send_count, int* recv_count, int* send_faces,
                                  int* recv_faces);

/* Device calls: */
/* Like apollo_dg_set_mesh with the GLOBAL mesh, keeping the elements with
 * part[k] == rank (in global order; node coordinates, states and
 * apollo_dg_num_elements refer to them) plus ghost slots for the traces of
 * their remote neighbours.  Every face keeps the orientation it has in the
 * global mesh and dt uses the global inscribed radius, so the ranks together
 * compute bit for bit what one handle on the whole mesh computes.  With
 * peers, apollo_dg_rhs, apollo_dg_step(_async) and the derivative calls are
 * refused (APOLLO_ERR_STATE): step with the staged calls below. */
apollo_status apollo_dg_set_mesh_partition(apollo_dg* h, int nverts, const double* vx, const double* vy, int K,
                                           const int* etov, const int* face_tag, const int* vert_canon,
                                           const int* part, int rank);
/* Peers (ascending), blocks per peer and the bytes of one trace block in this
 * precision (float64 or float32 traces); any pointer may be NULL. */
apollo_status apollo_dg_halo_info(const apollo_dg* h, apollo_precision prec, int* n_peers, int* peers,
                                  int* send_count, int* recv_count, int* block_bytes);
/* Caller-owned device buffers, 16-byte aligned: send and recv hold the blocks
 * of all peers back to back in peer order (the largest block size of the two
 * precisions times n_send / n_recv bytes), lam one 8-byte word that the caller
 * reduces with MAX across ranks as a signed 64-bit integer (the bits of a
 * non-negative double). */
apollo_status apollo_dg_halo_bind(apollo_dg* h, void* send, size_t send_bytes, void* recv, size_t recv_bytes,
                                  void* lam);
/* Staged stepping, all on the handle's stream (nothing waits on the host):
 *   apollo_dg_dist_start(t, dt)          once, before the first step
 *   per step, for stage = 0..4:
 *     apollo_dg_stage_begin(stage)       traces of the stage input, packed into send
 *     <caller: send -> peers, peers -> recv>
 *     apollo_dg_stage_end(stage)         recv unpacked into the ghost slots, the stage
 *   <caller: MAX all-reduce of the lam word> (stage 4 wrote it)
 *   apollo_dg_step_end()                 the dt policy of apollo_dg_step
 * then apollo_dg_get_time as after apollo_dg_step_async.  The caller orders
 * its transfers after the begin call's work and before the end call's on the
 * handle's stream (or synchronises it). */
apollo_status apollo_dg_dist_start(apollo_dg* h, double t, double dt, apollo_precision prec);
apollo_status apollo_dg_stage_begin(apollo_dg* h, int stage, apollo_precision prec);
apollo_status apollo_dg_stage_end(apollo_dg* h, int stage, apollo_precision prec);
apollo_status apollo_dg_step_end(apollo_dg* h);

/* Test hook for the failure path of the mixed-precision stage kernel (no
 * counterpart in Apollo).  polls: how many polls a bounded device wait makes
 * before it gives up (0 restores the default, about 2 s); stall_first_wait != 0
 * points the kernel's first wait at a barrier that nothing completes, so the
 * wait runs out, the kernel drains its tensor-core work and copies, frees its
 * tensor memory and returns, and the call reports APOLLO_ERR_TIMEOUT.  No GPU
 * fault is involved; the handle stays usable once the switch is cleared. */
apollo_status apollo_dg_debug_set_waits(apollo_dg* h, unsigned polls, int stall_first_wait);

/* Test hook for allocation failures (no counterpart in Apollo): the n-th
 * device allocation the library makes from now on, counting from 0 and over
 * all handles of the process, fails as if the device were out of memory (the
 * call reports APOLLO_ERR_ALLOC; a mesh that fails leaves its handle with no
 * mesh).  n < 0 switches the hook off. */
void apollo_dg_debug_fail_alloc(int n);

/* Error text of the last failing call on this handle. */
const char* apollo_dg_last_error(const apollo_dg* h);

apollo_status apollo_dg_destroy(apollo_dg* h);

#ifdef __cplusplus
}
#endif
#endif /* APOLLO_DG_H */
