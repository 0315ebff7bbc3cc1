/* dgb200: B200-native explicit DG residual and Runge-Kutta time step for the
 * 3D compressible Navier-Stokes / Euler equations on structured hex meshes.
 *
 * C ABI of the drop-in replacement for the reference's single-GPU path
 * (solver/solve_cuda.cu + solver/time_cuda.cu, driven by solver/cudg.cu).
 * Plain C types only: host pointers and sizes, optional device pointers and a
 * CUDA stream passed as void*.  Every entry point returns a DGB_* status code;
 * nothing calls exit() (the reference aborts through errout, error.cpp:34-52).
 *
 * Data layouts are the reference's:
 *   state   U[e][r][b]   element-major, 5 conserved variables, (p+1)^3 nodal
 *                        coefficients ordered [z[y[x]]]  (geometry_common.cpp:467-470)
 *   nodes   X[e][n][3]   (q+1)^3 geometry nodes per element, [z[y[x]]] order
 *                        (geometry_common.cpp:44-48)
 *   element e = i + nx*(j + ny*k)                         (geometry_shared.cpp:171)
 *   bounds  six btype codes for -x +x -y +y -z +z         (boundaries.cpp:26-35)
 */
#ifndef DGB200_H
#define DGB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum {
  DGB_OK = 0,
  DGB_ERR_ARG = 1,          /* bad argument, size or layout */
  DGB_ERR_UNSUPPORTED = 2,  /* valid input outside what this library implements */
  DGB_ERR_CUDA = 3,         /* a CUDA runtime call failed */
  DGB_ERR_GEOMETRY = 4,     /* singular Jacobian / mass matrix, mismatched periodic bounds */
  DGB_ERR_NONFINITE = 5,    /* a residual or state value became NaN/Inf */
  DGB_ERR_IO = 6,           /* .dg file could not be read or written */
  DGB_ERR_BOUNDARY = 7      /* subsonic inflow with no non-negative boundary Mach root */
};

/* boundary types, same codes as the reference's btype enum (boundaries.cpp:26-35) */
enum {
  DGB_BT_INTERIOR = -1,
  DGB_BT_PERIODIC = -2,
  DGB_BT_FREESTREAM = -3,
  DGB_BT_INVISCID_WALL = -4,
  DGB_BT_SUBSONIC_INFLOW = -5,
  DGB_BT_SUBSONIC_OUTFLOW = -6,
  DGB_BT_NO_SLIP_WALL = -7,
  /* An extension the reference lacks (its no-slip wall keeps the interior
   * energy, bound_states.cpp:42-49): a no-slip wall at the temperature set by
   * dgb_set_wall_temperature (default: the reference temperature T).  Ghost
   * state: interior density, zero velocity, E = rho R Tw / (gamma - 1). */
  DGB_BT_ISOTHERMAL_WALL = -8
};

/* time schemes, same order as the reference's time_scheme enum (time.cpp:23-27) */
enum { DGB_RK4 = 0, DGB_TVDRK3 = 1 };

/* arithmetic of the residual path */
enum {
  DGB_FP64 = 0,        /* everything in FP64 */
  DGB_MIXED_FP32 = 1   /* FP32 contractions and fluxes, FP64 geometry / inverse mass / RK */
};

typedef struct dgb_handle dgb_handle;

/* mesh: the fields of the reference's core_geometry that define a mesh
 * (geometry_common.cpp:25-83) */
typedef struct {
  int nx, ny, nz;          /* elements per direction */
  int p, q;                /* solution and geometry order */
  const double* nodes;     /* [nx*ny*nz][(q+1)^3][3] */
  long long bounds[6];     /* btype code per domain side */
} dgb_mesh_desc;

/* physical and reference parameters: the reference's `parameters` struct
 * (solver_params.cpp:22-36) */
typedef struct {
  double gamma;      /* ratio of specific heats */
  double R;          /* specific gas constant */
  double mu;         /* dynamic viscosity */
  double c;          /* reference speed of sound */
  double T;          /* reference static temperature */
  double P;          /* reference static pressure */
  double Ufr[5];     /* freestream conserved state */
  double source[5];  /* constant volume source per conserved variable */
  double eta;        /* BR2 stabilisation constant */
} dgb_params;

/* Human-readable text for a status code. */
const char* dgb_error_string(int status);

/* Detail of the last failure on the calling thread (empty if none). */
const char* dgb_last_error_message(void);

/* Builds the device-resident geometry and workspaces for one mesh.
 * Replaces cuda_device_geometry::cuda_device_geometry (solve_cuda.cu:171) and
 * cuda_residual_workspace (solve_cuda.cu:303), plus the host precompute they
 * consume (core_geometry::precompute, geometry_common.cpp:292;
 * shared_geometry::precompute_face_geometry, geometry_shared.cpp:156).
 * Meshes of affine elements keep one Jacobian per element; a mesh with any
 * curved (non-affine, q >= 2) element gets per-point geometry.  Uses the
 * current CUDA device. */
int dgb_create(const dgb_mesh_desc* mesh, const dgb_params* params, int precision,
               dgb_handle** out);

/* Element geometry as dgb_create built it on the device, copied to out
 * (count doubles, which must equal the part's size):
 *   DGB_GEO_ELEMENT  [E][36]          per element: inverse Jacobian [9]
 *                                     (row-major d xi_i / d x_c), detJ, the
 *                                     six outward unit normals [6][3], the
 *                                     six surface Jacobians, 2 zeros; taken
 *                                     at the element centre
 *   DGB_GEO_VOLUME   [E][10][P^3]     curved meshes: inverse Jacobian [9] and
 *                                     detJ at each volume Gauss point
 *   DGB_GEO_FACE     [E][6][14][P^2]  curved meshes: inverse Jacobian [9],
 *                                     outward unit normal [3], surface
 *                                     Jacobian and BR2 lifting scale at each
 *                                     face Gauss point
 * (P = p + 1; Gauss points x-fastest, face points in the face's axis order:
 * x faces (y,z), y faces (x,z), z faces (x,y)).  The per-point parts of an
 * affine mesh return DGB_ERR_ARG.  The reference keeps the same quantities
 * in core_geometry (geometry_common.cpp:292-454) and shared_geometry
 * (geometry_shared.cpp:156-267). */
enum { DGB_GEO_ELEMENT = 0, DGB_GEO_VOLUME = 1, DGB_GEO_FACE = 2 };
int dgb_get_geometry(dgb_handle* h, int part, double* out, size_t count);

/* Whether the mesh got per-point geometry, and the host wall time dgb_create
 * spent building the element geometry on the device (node upload, kernels
 * and checks; the handle's other allocations excluded).  Either output may
 * be NULL. */
int dgb_geometry_stats(const dgb_handle* h, int* curved, double* build_seconds);

/* Frees everything dgb_create allocated.  Replaces free_cuda_device_geometry
 * (solve_cuda.cu:267) and free_cuda_residual_workspace (solve_cuda.cu:323). */
int dgb_destroy(dgb_handle* h);

/* Orders the handle's work after / on this CUDA stream (cudaStream_t as void*;
 * NULL = legacy default stream, the reference's only stream). */
int dgb_set_stream(dgb_handle* h, void* stream);

/* Waits for the work the handle has queued: its stream and the host copies
 * of dgb_step_host_async; returns the status of the asynchronous host steps
 * since the last synchronization. */
int dgb_synchronize(dgb_handle* h);

/* Optional heat conduction, an extension the reference does not have (its
 * viscous flux carries no heat flux, flux.cpp:185-201): the energy flux gains
 * kappa grad T with kappa = mu c_p / Pr, in the volume, trace, dual-consistency
 * and lifting terms and in their adjoint.  Pr = 0 (the default) or +inf turns
 * it off, which is the reference's physics bit for bit; Pr < 0 or NaN is an
 * argument error.  Discards captured step graphs and any recorded forward run
 * (dgb_forward_record), which used the old physics. */
int dgb_set_prandtl(dgb_handle* h, double prandtl);

/* Replaces the physical parameters given to dgb_create (gamma, R, mu, the
 * reference state, source, eta) on an existing handle; the mesh, geometry,
 * state and Prandtl number stay.  Lets a caller vary viscosity or forcing
 * (e.g. with dgb_backward_params) without rebuilding the geometry.  Discards
 * captured step graphs and any recorded forward run. */
int dgb_set_params(dgb_handle* h, const dgb_params* params);

/* Temperature of the isothermal walls (DGB_BT_ISOTHERMAL_WALL), > 0; until
 * set it is the parameters' reference temperature T.  Discards captured
 * graphs and any recorded forward run. */
int dgb_set_wall_temperature(dgb_handle* h, double Tw);

/* Number of doubles in one state array: nx*ny*nz * 5 * (p+1)^3. */
long long dgb_state_size(const dgb_handle* h);

/* Host <-> device state copies in the reference layout U[e][r][b].
 * Replace shuffle_state + cudaMemcpy (cudg.cu:97-106) and the reverse
 * (cudg.cu:117-122). */
int dgb_set_state(dgb_handle* h, const double* U_host);
int dgb_get_state(dgb_handle* h, double* U_host);

/* Device -> device variants (caller-owned device arrays); synchronise. */
int dgb_set_state_device(dgb_handle* h, const double* U_dev);
int dgb_get_state_device(dgb_handle* h, double* U_dev);

/* Running mean of the resident state, the reference's "mean" output
 * (update_mean, output.cpp:39-49, called after every step from -mean_start,
 * dg.cpp:123-131): after step `tstep` >= mean_start,
 *   mean = (mean * (tstep - mean_start) + U) / (tstep + 1 - mean_start),
 * starting from zero at tstep == mean_start.  Queued on the handle's stream.
 * dgb_set_mean / dgb_get_mean copy it from / to the host (e.g. to continue
 * averaging after reading a .dg file that holds a "mean" output). */
int dgb_mean_update(dgb_handle* h, unsigned long long tstep, unsigned long long mean_start);
int dgb_set_mean(dgb_handle* h, const double* mean_host);
int dgb_get_mean(dgb_handle* h, double* mean_host);

/* Device pointer of the handle's resident state (for callers that keep data
 * on the GPU).  Writes through it count from the next dgb_step on: the
 * handle drops its Gauss-point copy of the state when it hands it out. */
int dgb_state_device_ptr(dgb_handle* h, double** U_dev);

/* The form dgb_step computes in.  DGB_STEP_GAUSS (the default) keeps the
 * state at the (p+1)^3 Gauss points of each element while it steps, V = (B x
 * B x B) U, where the mass matrix is diagonal and the interpolations to and
 * from the Gauss points drop out; it converts U -> V before its first step
 * and V -> U after its last (and continues from V across calls while the
 * state is not set otherwise, so a run split into calls is the same run).
 * DGB_STEP_NODAL steps the nodal coefficients.  Both are the reference's
 * discretisation; they agree to rounding.  The recorded runs of the adjoint
 * (dgb_forward_record*) step in the same form as dgb_step, and the backward
 * sweep reverses that form; its adjoint vectors enter and leave in the nodal
 * layout.  DGB_STEP_GAUSS_TC is the Gauss-point form whose mixed-precision
 * stage does its volume contractions on the tensor cores (three TF32
 * products per term, FP32 accumulation); it takes mixed-precision handles
 * with p = 3 or 4, affine elements and no heat flux (else
 * DGB_ERR_UNSUPPORTED), and is slower than the default FP32x2 stage: it is
 * kept as the measured alternative. */
enum { DGB_STEP_GAUSS = 0, DGB_STEP_NODAL = 1, DGB_STEP_GAUSS_TC = 2 };
int dgb_set_step_form(dgb_handle* h, int form);

/* One residual evaluation of U: R = un-inverted residual (may be NULL) and
 * f = dU/dt = -Minv R.  Host pointers; copies in and out.
 * Replaces cuda_residual (solve_cuda.cu:1235) / residual (solve.cpp:150). */
int dgb_residual(dgb_handle* h, const double* U_host, double* R_host, double* f_host);

/* Same on device pointers, on the handle's stream, no host synchronisation. */
int dgb_residual_device(dgb_handle* h, const double* U_dev, double* R_dev, double* f_dev);

/* Advances the resident state nsteps steps of size dt with RK4 or TVD-RK3.
 * norms_host (may be NULL) receives, per step, sqrt(sum R^2 / size) of the
 * first stage's residual, the number the reference prints each step
 * (time_cuda.cu:36-47, time_distributed.cpp:23-44).
 * Replaces RK4_cuda / tvdRK3_cuda (time_cuda.cu:126-185) and
 * RK4_distributed / tvdRK3_distributed (time_distributed.cpp:46-102).
 * Returns DGB_ERR_NONFINITE if a residual norm became NaN/Inf (the reference
 * aborts on a NaN norm, time_distributed.cpp:41-42). */
int dgb_step(dgb_handle* h, int scheme, double dt, unsigned long long nsteps,
             double* norms_host);

/* dgb_step for a state kept in host memory: U_in (host, layout U[e][r][b])
 * is copied in, nsteps RK steps are taken, and the state after them is
 * written to U_out (host; may equal U_in), with the printed norm of every
 * step in norms_host (may be NULL).  The same kernels and results as
 * dgb_set_state + dgb_step + dgb_get_state, bit for bit, with the copies
 * overlapped with the work: the state comes in in pieces of elements on a
 * second stream while the pieces already in are changed to Gauss-point
 * values and their face traces computed, the first stage runs on a piece as
 * soon as the pieces its neighbours lie in are in, and the last two stages
 * of the last step run piece by piece, each last-stage piece copied out
 * while the others compute.  Overlap needs page-locked
 * (pinned) host buffers; pageable ones give the same results.  The nodal
 * step form (dgb_set_step_form) takes the plain calls.  No counterpart in
 * the reference, whose driver copies the state in once and out at each
 * checkpoint (cudg.cu:96-126). */
int dgb_step_host(dgb_handle* h, int scheme, double dt, unsigned long long nsteps, const double* U_in,
                  double* U_out, double* norms_host);

/* dgb_step_host without waiting: the copies and the steps are queued and the
 * call returns.  U_in is read and U_out and norms_host written as the queued
 * copies run, so none of them may be touched before dgb_synchronize(h),
 * which also reports the status of the steps (a non-finite norm, a boundary
 * without a Mach root).  Consecutive calls on a handle pipeline: a call's
 * copy in of a piece waits for the handle's earlier work and for the
 * previous call's copy out of that piece (U_in may be the previous U_out),
 * not for the rest of the previous copies out, so stepping a host state in
 * place call after call overlaps each call's copies out with the next one's
 * copies in.  Other calls on the handle may follow without synchronizing
 * (they are ordered after the queued steps); a dgb_step in between resets
 * the status the synchronization reports.  No counterpart
 * in the reference. */
int dgb_step_host_async(dgb_handle* h, int scheme, double dt, unsigned long long nsteps, const double* U_in,
                        double* U_out, double* norms_host);

/* Kernel launches issued by the last dgb_step / dgb_residual call. */
long long dgb_last_launch_count(const dgb_handle* h);

/* Measurement hook: runs `reps` RK steps of the resident state launch by
 * launch (no graph) with a CUDA event between consecutive launches on the
 * handle's stream; ms_out[k] is the mean duration of launch k of one step.
 * *nk: capacity of ms_out in, launches per step out.  Advances the state like
 * dgb_step. */
int dgb_profile_step(dgb_handle* h, int scheme, double dt, int reps, double* ms_out, int* nk);

/* One FP64 residual f = -Minv R of a device-resident state U_dev into f_dev
 * (both caller-owned device arrays, layout U[e][r][b]), for callers that may
 * not allocate GPU memory -- e.g. a host application that owns the device
 * memory pool, or a solver that has claimed all of HBM for its own state.
 * It calls no cudaMalloc / cudaFree: every intermediate (operator tables,
 * element geometry, neighbour table, face traces, status word) lives in one
 * file-scope device array of 32 MiB built into the library, which every GPU
 * that loads the library holds until the process exits.  Meshes needing more
 * scratch than that (about 4,000 affine or 1,500 curved elements at p = 3) are rejected with
 * DGB_ERR_ARG and a message giving the size needed.
 * Each call looks up the array's device address on the current device (no
 * allocation); `stream` (cudaStream_t as void*, NULL = legacy default) must
 * belong to the current device.  All calls share the array and it keeps the
 * last call's contents: calls whose GPU work could overlap (different
 * streams or host threads) race -- order them.  The call copies from
 * pageable host memory and synchronises `stream` before returning, so it
 * cannot be made while `stream` is being captured.
 * This entry point has no counterpart in the reference. */
int dgb_residual_noalloc(const dgb_mesh_desc* mesh, const dgb_params* params, const double* U_dev,
                         double* f_dev, void* stream);

/* ------------------------------------------------------------------ adjoint
 * Discrete adjoint of the FP64 residual and of the RK steps, hand-written
 * (reverse mode of every kernel).  The reference has no adjoint: these entry
 * points have no counterpart there.  They cover every mesh and boundary
 * type the forward path does.  A mixed-precision handle recomputes states in
 * its own precision and applies the FP64 adjoint at them. */

/* Ubar = (df/dU)^T lam at U, f = -Minv R(U) as dgb_residual computes it.
 * Host arrays in the state layout; synchronises. */
int dgb_residual_vjp(dgb_handle* h, const double* U_host, const double* lam_host, double* Ubar_host);

/* Same on device arrays (Ubar must not alias U or lam), on the handle's
 * stream, no host synchronisation. */
int dgb_residual_vjp_device(dgb_handle* h, const double* U_dev, const double* lam_dev, double* Ubar_dev);

/* Reverse of one RK step U -> U' of `scheme`, as dgb_step takes it (in its
 * form, dgb_set_step_form): lam_dev holds the adjoint of U' on entry and the
 * adjoint of U on return (in place).  U_dev is unchanged.  Synchronises. */
int dgb_step_vjp_device(dgb_handle* h, int scheme, double dt, const double* U_dev, double* lam_dev);

/* Recorded forward run: advances the resident state by nsteps like dgb_step
 * (norms_host as there, may be NULL) and keeps up to `slots` device copies of
 * intermediate states (one of them the initial state) for dgb_backward,
 * placed by binomial checkpointing so that the backward sweep recomputes the
 * fewest steps: slots >= nsteps stores every state, slots = 1 recomputes
 * every step from the initial state.  Holds slots * dgb_state_size doubles
 * of device memory until the handle is destroyed. */
int dgb_forward_record(dgb_handle* h, int scheme, double dt, unsigned long long nsteps, int slots,
                       double* norms_host);

/* Recorded forward run that keeps every state and every intermediate RK
 * stage state (nsteps * 4 states for RK4, * 3 for TVD-RK3, on the device), so
 * that dgb_backward recomputes nothing: each reverse step is the residual
 * VJPs of its stages only.  Same states and norms as dgb_step. */
int dgb_forward_record_stages(dgb_handle* h, int scheme, double dt, unsigned long long nsteps,
                              double* norms_host);

/* Backward sweep through the last recorded run: given dJ/dU_N (the adjoint
 * of the final state) returns dJ/dU_0.  The resident state is left at U_N.
 * May be called repeatedly for different dJ/dU_N; when a sweep has
 * overwritten checkpoints the next one first recomputes them from U_0. */
int dgb_backward(dgb_handle* h, const double* dJdUN_host, double* dJdU0_host);
int dgb_backward_device(dgb_handle* h, const double* dJdUN_dev, double* dJdU0_dev);

/* Parameters the backward sweep can differentiate: dJdparams[DGB_DPARAM_MU]
 * = dJ/dmu (dynamic viscosity, at a fixed Prandtl number: the heat flux
 * scales with mu), dJdparams[DGB_DPARAM_SOURCE + r] = dJ/dsource[r] and
 * dJdparams[DGB_DPARAM_TWALL] = dJ/dTw, the isothermal walls' temperature
 * (0 on a mesh without them). */
enum { DGB_DPARAM_MU = 0, DGB_DPARAM_SOURCE = 1, DGB_DPARAM_TWALL = 6, DGB_NDPARAMS = 7 };

/* dgb_backward plus the gradient of J with respect to the parameters above
 * over the recorded run, into dJdparams[DGB_NDPARAMS] (host).  Each residual
 * is affine in mu, so df/dmu = (f(mu1) - f(0)) / mu1 (mu1 = mu, or 1 for an
 * inviscid handle), two FP64 residuals per stage; df/dsource[r] = 1 at every
 * node of variable r (the source is tested with the mass matrix's
 * quadrature).  About twice the cost of dgb_backward.  The reference has no
 * counterpart (it has no adjoint). */
int dgb_backward_params(dgb_handle* h, const double* dJdUN_host, double* dJdU0_host, double* dJdparams_host);
/* Same on device arrays; dJdparams_dev (DGB_NDPARAMS doubles) is overwritten. */
int dgb_backward_params_device(dgb_handle* h, const double* dJdUN_dev, double* dJdU0_dev,
                               double* dJdparams_dev);

/* Steps recomputed and reversed by the last backward sweep, and the forward
 * steps of the whole checkpoint plan (recorded run included). */
int dgb_adjoint_stats(const dgb_handle* h, long long* forward_steps, long long* reverse_steps,
                      long long* planned_forward_steps);

/* The binomial checkpoint plan itself (host only): 2 * *nops entries
 * (kind, argument) into ops_out (capacity cap), kind 0 = advance `argument`
 * steps, 1 = store the work state in buffer `argument`, 2 = restore it from
 * buffer `argument`, 3 = reverse step `argument`.  ops_out may be NULL to
 * query the size. */
int dgb_checkpoint_plan(long long nsteps, int slots, long long* ops_out, long long cap, long long* nops,
                        long long* forward_steps, int* peak_slots);

/* ---------------------------------------------------------------- host side
 * Host-only helpers (no GPU needed) that mirror the reference's setup
 * functions, for drivers and for checks. */

/* n-point Gauss-Legendre rule on [a,b] (quadrature.cpp:84-205). */
int dgb_gauss_legendre(int n, double a, double b, double* x, double* w);

/* Equispaced Lagrange basis on [0,1] and its derivative (basis.cpp:91-148). */
double dgb_lagrange1d(int i, int p, double x);
double dgb_lagrange1d_deriv(int i, int p, double x);

/* The element geometry of dgb_get_geometry computed on the host's threads
 * instead (the builder dgb_residual_noalloc uses), with the same checks and
 * messages as dgb_create; dgb_create's device builder gives the same bits.
 * *curved (may be NULL) is set when some element is not affine.  geo gets
 * the DGB_GEO_ELEMENT part (ngeo doubles); gv and gf the DGB_GEO_VOLUME and
 * DGB_GEO_FACE parts of a curved mesh (ngv, ngf doubles; untouched for an
 * affine mesh).  Any of the three may be NULL; a non-NULL one of the wrong
 * size is DGB_ERR_ARG. */
int dgb_geometry_host(const dgb_mesh_desc* mesh, int* curved, double* geo, size_t ngeo, double* gv, size_t ngv,
                      double* gf, size_t ngf);

/* Geometry nodes of the reference's bump / stretched channel generator
 * (generate_bump_nodes, geometry_common.cpp:494-576, as called by
 * bump_shared, geometry_shared.cpp:275-292).  nodes: [nx*ny*nz][(q+1)^3][3]. */
int dgb_bump_nodes(int nx, int ny, int nz, int q, double lx, double ly, double lz,
                   double a, double bmp_height, double bmp_center, double bmp_variance,
                   double* nodes);

/* make_reference_state (solver_params.cpp:40-70). */
int dgb_make_reference_state(double gamma, double gcnst, double mu, double c, double rho,
                             double u, double v, double w, double eta,
                             const double* source, dgb_params* out);

/* Writes a .dg file byte-compatible with the reference's write_state
 * (io.cpp:33-90): outputs appear in the reference's hash-map order
 * (djb2 mod 256, data_structures.cpp:538-583). */
int dgb_write_state(const char* fname, unsigned long long tstep, const dgb_mesh_desc* mesh,
                    int noutput, const char* const* keys, const double* const* data);

/* Reads a .dg header (io.cpp:92-124): sizes and bounds; nodes and the state
 * named `key` are copied when their pointers are non-NULL.  Returns
 * DGB_ERR_IO on a short or malformed file, or when `key` is given and the
 * file holds no output of that name (whether or not data is NULL). */
int dgb_read_state(const char* fname, unsigned long long* tstep, int* nx, int* ny, int* nz,
                   int* p, int* q, long long* bounds, double* nodes, const char* key,
                   double* data);

#ifdef __cplusplus
}
#endif

#endif /* DGB200_H */
