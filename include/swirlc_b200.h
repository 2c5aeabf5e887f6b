/*
 * swirlc_b200 C-ABI: B200 (sm_100a) kernels for Swirl-C's compressible
 * finite-volume right-hand side, its halo fill, the SSP-RK3/RK2 stage update
 * and the CFL time-step reduction.
 *
 * Conventions shared by every entry point
 *  - Fields are device arrays in the reference layout [nz+2h][nx+2h][ny+2h]
 *    (y fastest), halos included; `SwcGrid.sx` / `.sz` give the element
 *    strides of x and z (the y stride is 1).
 *  - Conserved fields come in the order rho, rho_u, rho_v, rho_w, rho_e,
 *    followed by `SwcScheme.nscalars` transported scalars rho_phi.
 *  - A face value stored at index i belongs to face i-1/2, as in the
 *    reference (compressible_navier_stokes.py:442-453).
 *  - `stream` is a cudaStream_t passed as void*; every call is asynchronous
 *    on that stream and allocates nothing.
 *  - Every call returns SWC_OK (0) or a negative status; swc_last_error()
 *    gives the message of the last failing call on the calling thread. No
 *    C++ exception crosses this boundary.
 */
#ifndef SWIRLC_B200_H_
#define SWIRLC_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWC_ABI_VERSION 1
#define SWC_MAX_FIELDS 8 /* 5 conserved + up to 3 transported scalars */

/* Status codes. */
enum {
  SWC_OK = 0,
  SWC_ERR_ARG = -1,         /* bad pointer, size or enum (ValueError)      */
  SWC_ERR_UNSUPPORTED = -2, /* configuration not implemented (NotImplementedError) */
  SWC_ERR_LAUNCH = -3,      /* CUDA launch or runtime failure              */
  SWC_ERR_TIMEOUT = -4,     /* a bounded device wait gave up               */
  SWC_ERR_NONFINITE = -5    /* non-finite value detected                   */
};

enum { SWC_F32 = 0, SWC_F64 = 1 };
/* interpolation_scheme (compressible_navier_stokes.py:39-43); SWC_NODE is
 * the identity face value used by the reference tests' WENO mock. */
enum { SWC_WENO5 = 0, SWC_WENO3 = 1, SWC_MUSCL = 2, SWC_NODE = 3 };
enum { SWC_LIM_VAN_LEER = 0, SWC_LIM_MC = 1, SWC_LIM_MINMOD = 2,
       SWC_LIM_MINMOD3 = 3 /* the prototype's three-slope minmod */ };
/* numeric_flux_scheme (riemann_solver.py:24-27). */
enum { SWC_HLL = 0, SWC_HLLC = 1 };
/* BoundaryCondition (bc_types.py:22-27) plus NONE = leave the halo as is. */
enum { SWC_BC_PERIODIC = 0, SWC_BC_DIRICHLET = 1, SWC_BC_NEUMANN = 2,
       SWC_BC_NONE = 4 };
/* Stage output modes: RHS: out = L(uk); EULER: out = uk + L*dt;
 * CONVEX: out = u0*c0 + (uk + L*dt)*c1 (rk3.py:69-83);
 * AVERAGE: out = c0*(u0 + (uk + dt*L)) (rk2.py:67-86). */
enum { SWC_OUT_RHS = 0, SWC_OUT_EULER = 1, SWC_OUT_CONVEX = 2,
       SWC_OUT_AVERAGE = 3 };

typedef struct SwcGrid {
  int32_t nx, ny, nz; /* interior cells along x, y, z                    */
  int32_t halo;       /* halo layers stored on each side (cfg.halo_width) */
  int64_t sx, sz;     /* element strides of x and z                      */
  double dx, dy, dz;  /* cfg.dx, cfg.dy, cfg.dz                          */
} SwcGrid;

typedef struct SwcScheme {
  int32_t dtype;     /* SWC_F32 / SWC_F64                                   */
  int32_t interp;    /* SWC_WENO5 ...                                       */
  int32_t limiter;   /* MUSCL limiter, SWC_LIM_*                             */
  int32_t riemann;   /* SWC_HLL / SWC_HLLC                                   */
  int32_t diffusion; /* cfg.include_diffusion                               */
  int32_t nscalars;  /* transported scalars after rho_e (0..3)              */
  int32_t gravity_mask; /* bit d set: rho_u_d gets rho*G*g[d] (gravity.py:51-102) */
  int32_t zseg;      /* z planes per CTA in the stage kernel; 0 = automatic */
  int32_t tile;      /* unused by the single-grid stage (16x16 y x x cells)  */
  int32_t reserved;
  double nu, pr;     /* transport_parameters (simple.py:44-45)              */
  double g[3];       /* cfg.g, the gravity unit vector                      */
  /* Per-axis gravitational terms a_d[i] = G*g_d*coord_d[i] on the local
   * cell-centre mesh with halos (generic.py:282-319, utils.py:43-89); the
   * potential energy is (-a_x - a_y) - a_z. NULL means zero. Arrays are in
   * `dtype` with n_d + 2*halo entries. */
  const void* pe_axis[3];
} SwcScheme;

typedef struct SwcBC {
  int32_t kind;      /* SWC_BC_*                                            */
  int32_t per_layer; /* 0: `value` in every layer; 1: `planes` per layer    */
  double value;      /* Dirichlet value or Neumann increment per layer      */
  /* Dirichlet planes [halo][A][B] in `dtype`; (A, B) are the two other axes
   * in storage order (z, x, y) with halos: x-faces (z, y), y-faces (z, x),
   * z-faces (x, y). Layer 0 is the outermost layer on the low side and the
   * innermost on the high side (boundary_test.py:175-298). */
  const void* planes;
} SwcBC;

typedef struct SwcFieldBC {
  int32_t via_primitive; /* BC given on field/rho (boundary.py:516-531)     */
  int32_t reserved;
  SwcBC side[3][2];      /* [x, y, z][low, high]                            */
} SwcFieldBC;

/* Device-resident time control used by the step loop without host syncs. */
typedef struct SwcClock {
  double t;       /* simulated time                                      */
  double dt;      /* step size used by the current step                  */
  double dtmin;   /* min over cells/dims of delta/(|u|+c) for the next step */
  double cfl;     /* > 0: dt = min(cfl*dtmin, t_end - t); else dt fixed  */
  double t_end;   /* > 0: clamp the last step to end at t_end            */
  int64_t step;   /* completed steps                                     */
} SwcClock;

/* Library and error reporting. */
int swc_abi_version(void);
int swc_last_error(char* buf, size_t len);
/* Number of this library's kernel launches issued by the calling thread. */
int64_t swc_launch_count(void);

/* Halo fill of `nfields` fields, dims in order x, y, z, for a single
 * replica (boundary.py:34-86, 464-539; boundary.update_boundary :606-629).
 * Fields with via_primitive are filled after rho (index rho_index) is
 * complete. Replaces swirl_lm halo_exchange.inplace_halo_exchange as called
 * from boundary.py:77-86. */
int swc_halo_fill(const SwcGrid* grid, int32_t dtype, int32_t nfields,
                  void* const* fields, const SwcFieldBC* bcs,
                  int32_t rho_index, void* stream);

/* One fused pass: RHS of the conserved state `uk` (halos already filled)
 * followed by the stage combination selected by `mode`. `u0` may be NULL
 * for SWC_OUT_RHS / SWC_OUT_EULER; `uout` may alias `u0` (pointwise) but
 * never `uk`. `dt` is a device double; `dtmin_out`, when not NULL, is a
 * device double min-reduced (atomically) with the CFL limit of `uout`.
 * Interior cells of `uout` are written; its halos are left untouched.
 * Replaces the rhs of get_rhs_fn (compressible_navier_stokes.py:68-268)
 * and one stage of rk3.integrate / rk2.integrate (rk3.py:87-120,
 * rk2.py:69-86). */
int swc_rk_stage(const SwcGrid* grid, const SwcScheme* scheme,
                 const void* const* uk, const void* const* u0,
                 void* const* uout, int32_t mode, double c0, double c1,
                 const double* dt, double* dtmin_out, void* stream);

/* Extensions of the fused stage: transported scalars, hydrostatic helper
 * states and face / flux boundary conditions. */
#define SWC_MAX_OVERRIDES 8
/* Face BC (boundary.py:186-461): a primitive (u, v, w, e, phi) or its
 * conservative (rho_u, ..., rho_phi) set on both face states. */
enum { SWC_FACE_PRIMITIVE = 0, SWC_FACE_CONSERVATIVE = 1 };
/* Flux BC type (bc_types.BoundaryFluxType; boundary.py:89-183). */
enum { SWC_FLUX_CONVECTIVE = 0, SWC_FLUX_DIFFUSIVE = 1, SWC_FLUX_TOTAL = 2 };

typedef struct SwcOverride {
  int32_t var;        /* 1..3 velocity / momentum x, y, z; 4 e / rho_e;
                         5 + k scalar k (flux BCs: 0 is rho as well)     */
  int32_t mode;       /* face: SWC_FACE_*; flux: SWC_FLUX_*              */
  double value;       /* used when `plane` is NULL                       */
  const void* plane;  /* one face plane [A][B] in dtype, axes as in
                         SwcBC.planes (halos included), or NULL          */
} SwcOverride;

typedef struct SwcStageExt {
  /* Hydrostatic reference states (fields with halos), both or neither:
   * the momentum flux and HLLC use p_dyn = p - p_ref, reconstructed like
   * the primitives with p_dyn = 0 in the halos of outer sides, and gravity
   * acts on rho - rho_ref (compressible_navier_stokes.py:299-335,
   * hllc.py:105-120). HLLC takes its sound speeds from p_dyn, as the
   * reference does, so p_dyn must stay >= 0 on the faces. */
  const void* p_ref;
  const void* rho_ref;
  int32_t boundary[3][2]; /* 1: side [dim][low/high] is on the boundary of
                             the whole grid (all sides for one grid)     */
  int32_t nface[3][2];    /* face overrides per side                     */
  int32_t nflux[3][2];    /* flux overrides per side                     */
  int32_t reserved;
  SwcOverride face[3][2][SWC_MAX_OVERRIDES];
  SwcOverride flux[3][2][SWC_MAX_OVERRIDES];
} SwcStageExt;

/* swc_rk_stage with the extensions above. Fields: 5 + scheme->nscalars
 * (rho_phi_k after rho_e). `ext` may be NULL (no helper states, no face or
 * flux BCs). Face overrides act on the faces between the halo and the
 * interior on sides marked `boundary`; a density face BC is not supported
 * (in the reference it drops p and h from the face primitives). Face BCs
 * with diffusion are rejected, as in the reference
 * (compressible_navier_stokes.py:185-196). */
int swc_rk_stage_ext(const SwcGrid* grid, const SwcScheme* scheme,
                     const SwcStageExt* ext, const void* const* uk,
                     const void* const* u0, void* const* uout, int32_t mode,
                     double c0, double c1, const double* dt,
                     double* dtmin_out, void* stream);

/* One time step in place on `u` (5 fields): [clock begin] -> halo fill ->
 * fused stages -> [clock end]. order 3: SSP-RK3 (rk3.py:87-120); order 2:
 * RK2 (rk2.py:69-86). `work` holds 10 field buffers (two states of the
 * shape of u) used as scratch. `clock_dev` is a device SwcClock: the step
 * uses clock->dt; with clock->cfl > 0 the step starts with
 * dt = min(cfl*dtmin, t_end-t) and its last stage min-reduces the CFL limit
 * of the new state into clock->dtmin for the next step (so before the first
 * step clock->dtmin must hold the limit of the initial state, e.g. from
 * swc_cfl_reduce). Replaces Simulation.step (simulation.py:68-105) for one
 * replica. */
int swc_rk_step(const SwcGrid* grid, const SwcScheme* scheme,
                const SwcFieldBC* bcs, int32_t order, void* const* u,
                void* const* work, SwcClock* clock_dev, void* stream);

/* Size of the built-in work space of swc_rk_step_noalloc (64 MiB). */
#define SWC_NOALLOC_MAX_BYTES (64ll << 20)

/* swc_rk_step without the `work` argument; it has no counterpart in the
 * reference. It is for callers that cannot provide the ten work buffers:
 * hosts that must not allocate device memory while running (a plugin whose
 * host owns and budgets all device memory, a real-time loop where an
 * allocation could block or fail) and bindings with no CUDA allocator. The
 * work states live in one array of SWC_NOALLOC_MAX_BYTES inside this library,
 * held on every GPU that loads it until the process exits; the call itself
 * allocates nothing. Grids whose ten padded fields (10 * sz * (nz + 2*halo)
 * elements, each field rounded up to 256 bytes) exceed it are rejected with
 * SWC_ERR_ARG before anything is launched (e.g. 96^3 f32 with halo 3 fits,
 * 128^3 does not). The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress with that device current); make that call
 * before any stream capture. The address is cached for the process: after a
 * cudaDeviceReset it is stale and the entry point must not be called again
 * in that process. All calls share the array, which keeps the last
 * call's contents, so calls that overlap on the GPU race: serialise them
 * (one stream, or events between streams and threads). Nothing in the array
 * needs to be zero; halo sides set to SWC_BC_NONE keep whatever the array
 * held there. */
int swc_rk_step_noalloc(const SwcGrid* grid, const SwcScheme* scheme,
                        const SwcFieldBC* bcs, int32_t order, void* const* u,
                        SwcClock* clock_dev, void* stream);

/* One member of a batch: an independent grid with its own state, work
 * buffers, halo BCs, potential energy and clock. */
typedef struct SwcBatchMember {
  SwcGrid grid;
  void* u[5];             /* conserved state (device), updated in place     */
  void* work[10];         /* two work states of the shape of u (device)     */
  const void* pe_axis[3]; /* as SwcScheme.pe_axis, for this member's mesh   */
  SwcFieldBC bcs[5];      /* halo BCs of rho..rho_e (read during the call)  */
  SwcClock* clock;        /* this member's device clock (own CFL dt)        */
  int32_t tile;           /* cells per CTA (y x x): 0 or 1 16x16, 2 8x32    */
  int32_t zseg;           /* z planes per CTA; 0 auto                       */
} SwcBatchMember;

/* One time step of every member (order 3: SSP-RK3, order 2: RK2), each with
 * the dt of its own clock, as swc_rk_step does for one grid. All members
 * share `scheme` (its pe_axis, tile and zseg are replaced by the members').
 * Each RK stage is one batched halo fill (one pass for members whose dims
 * are all periodic or zero-gradient, else one pass per dim) and one batched
 * stage launch per tile shape over all members, instead of a launch
 * sequence per member. With 16x16 tiles each member's result equals swc_rk_step's bit for
 * bit; 8x32 tiles (for members at most 8 cells wide in y; not available for
 * f64 WENO5) can differ from it in the last bit. Members must not share
 * buffers. No counterpart in the reference, which advances
 * one grid per program: replaces calling Simulation.step
 * (simulation.py:68-105) on each member in turn. */
int swc_batch_step(const SwcScheme* scheme, int32_t order, int32_t nmembers,
                   const SwcBatchMember* members, void* stream);

/* Reverse mode of one fused stage for WENO5 or MUSCL (any SWC_LIM_*
 * limiter) with HLL or HLLC (+ viscous), no transported scalars, on the
 * halo-filled state `uk` of that stage (halo width >= 3). On the
 * interior cells
 *   vout = alpha*lam + c1*x1 + c2*x2 + beta * H^T J_L(H uk)^T lam,
 * (x1, x2 may be NULL; H: halo fill with `bcs`), halos of vout set to 0,
 * and nu_bar (device double; may be NULL) += beta * lam . dL/dnu, where L
 * is the right-hand side a stage adds (compressible_navier_stokes.py:
 * 68-268) and lam the cotangent of the stage output (its halos are not
 * read). A stage out = A*u0 + B*(uk + dt*L(uk)) (rk3.py:87-120) has the uk
 * cotangent B*lam + B*dt*H^T J^T lam (alpha = B, beta = B*dt) and the u0
 * cotangent A*lam, which x1 / x2 let the caller fold in. vout must not alias
 * uk, lam, x1 or x2. `scratch` is SWC_VJP_SCRATCH caller buffers of the
 * shape of uk, each holding at least (nx+2h)(ny+2h)(nz+2h) elements and
 * 8-byte aligned (primitives and their cotangents, copies transposed to
 * [z][y][x] for the y faces, the per-segment and tangential parts that
 * are summed in a fixed order, the per-warp nu partials). Every sum has a
 * fixed order (no floating-point atomics whose order depends on
 * scheduling), so the same inputs give the same bits on every run. The
 * first call in a process sets the kernels' shared-memory limit for its
 * dtype: make it outside stream capture. The reference differentiates
 * this path with TF's GradientTape; this is its discrete adjoint. */
#define SWC_VJP_SCRATCH 79
int swc_rk_stage_vjp(const SwcGrid* grid, const SwcScheme* scheme,
                     const SwcFieldBC* bcs, const void* const* uk,
                     const void* const* lam, double alpha, double beta,
                     const void* const* x1, double c1, const void* const* x2,
                     double c2, void* const* vout, double* nu_bar,
                     void* const* scratch, void* stream);

/* Reverse of one whole time step, SSP-RK3 (order 3, rk3.py:87-120) or RK2
 * (order 2, rk2.py:69-86), in one call: the two or three stage adjoints of
 * swc_rk_stage_vjp with the step's coefficients. `stages` holds order x 5
 * pointers, the halo-filled stage states (u, u1[, u2]) the forward step
 * advanced; g is the cotangent of the step's output, gn receives that of
 * its input (interior; halos 0), nu_bar (may be NULL) accumulates the nu
 * cotangent. `work` is 10 caller fields of the grid's shape (the stage
 * cotangents g1, then g2; RK2 uses only g1). gn must not alias g, work or a
 * stage (SWC_ERR_ARG, checked before any launch). Replaces the
 * per-step loop a caller of the reference would run under GradientTape
 * (no counterpart call in the reference). */
int swc_rk_step_vjp(const SwcGrid* grid, const SwcScheme* scheme,
                    const SwcFieldBC* bcs, int32_t order,
                    const void* const* stages, double dt, const void* const* g,
                    void* const* gn, void* const* work, double* nu_bar,
                    void* const* scratch, void* stream);

/* dtmin_out <- min(dtmin_out, min over interior cells and dims of
 * delta_d / (|u_d| + c)), c = sqrt(gamma p / rho) (CFL rule of the
 * reference's prototype, demo/swirl_c_prototype.ipynb `solve`). */
int swc_cfl_reduce(const SwcGrid* grid, const SwcScheme* scheme,
                   const void* const* u, double* dtmin_out, void* stream);

/* Start of a step: clock->dt = cfl>0 ? min(cfl*dtmin, t_end-t) : dt;
 * resets clock->dtmin to +inf for the coming reduction. */
int swc_clock_begin_step(SwcClock* clock_dev, void* stream);
/* End of a step: t += dt, step += 1. */
int swc_clock_end_step(SwcClock* clock_dev, void* stream);

/* Non-finite detector (no reference counterpart: the reference's TF graph
 * propagates NaN silently). The CFL reductions (swc_cfl_reduce and the one
 * fused into the last stage of swc_rk_step / swc_batch_step) visit every
 * new cell; a cell whose rho, p or rho_e is not finite, or whose CFL limit
 * is NaN (p/rho < 0), contributes a limit of 0, which no finite state has.
 * This call waits for `stream`, reads the clock and returns
 * SWC_ERR_NONFINITE when clock->dtmin is 0 (the state after the last
 * completed step is bad), else SWC_OK. It synchronises, so it is not for
 * use inside stream capture; the step calls themselves stay asynchronous. */
int swc_clock_status(const SwcClock* clock_dev, void* stream);

/* Component kernels behind the reference's unit-level API. */

/* Face reconstruction of one 3-D field along `dim` (0=x,1=y,2=z):
 * neg/pos at face i-1/2 (swirl_lm interpolation.weno(v, dim, k) and
 * flux_limiter(v, dim, MUSCL) as called at
 * compressible_navier_stokes.py:581-589). */
int swc_reconstruct(const SwcGrid* grid, int32_t dtype, int32_t interp,
                    int32_t limiter, int32_t dim, const void* v, void* neg,
                    void* pos, void* stream);

/* Pointwise intercell convective flux for `n` face points from reconstructed
 * primitive states. prim_neg/prim_pos hold 7 + nscalars arrays each:
 * rho, u, v, w, e, p, h, then the transported scalars phi (0..3). p_dyn_neg/pos may be NULL (helper p_dyn,
 * hllc.py:105-120). `pe` (n entries, may be NULL) is the potential energy
 * at the face index. flux holds 5 + nscalars outputs.
 * Replaces hll_convective_flux (hll.py:36-175) and hllc_convective_flux
 * (hllc.py:33-257) with the physical flux of
 * compressible_navier_stokes.py:338-427. */
int swc_riemann_flux(int64_t n, int32_t dtype, int32_t riemann, int32_t dim,
                     int32_t nscalars, const void* const* prim_neg,
                     const void* const* prim_pos, const void* p_dyn_neg,
                     const void* p_dyn_pos, const void* pe,
                     void* const* flux, void* stream);

/* Wave-speed estimates for `n` face points: s_l, s_r (hll.py:178-283) and,
 * when s_m is not NULL, the HLLC contact speed (hllc.py:260-347). */
int swc_wave_speeds(int64_t n, int32_t dtype, int32_t dim,
                    const void* const* prim_neg, const void* const* prim_pos,
                    const void* pe, void* s_l, void* s_m, void* s_r,
                    void* stream);

/* Stencils on a full 3-D array along `dim`: op 0 forward_1, 1 backward_1,
 * 2 central_2 (gradient.py:21-94), 3 linear_interpolation
 * (interpolation.py:21-53). Points whose stencil leaves the array get 0. */
int swc_stencil(const SwcGrid* grid, int32_t dtype, int32_t op, int32_t dim,
                double h, const void* f, void* out, void* stream);

/* Viscous terms on every face i-1/2 of a whole 3-D array (halo 0 grid, the
 * spacings from grid->dx/dy/dz), from cell values q = {rho, u, v, w, p},
 * computed with the fused stage's own face routine (so the values are bit
 * for bit the viscous part of the stage's fluxes). Faces whose stencil
 * leaves the array get 0. `what`:
 *  SWC_VISC_FLUX   out[15]: diffusive flux of rho, rho_u, rho_v, rho_w,
 *                  rho_e across x, y, z faces (out[d*5+k]);
 *                  compressible_navier_stokes.py:618-707
 *                  (_intercell_diffusive_flux); kappa = cp nu rho / pr.
 *  SWC_VISC_STRAIN out[9]: strain rate S_ij on the j faces (out[i*3+j]),
 *                  fluid.py:31-111 (reads u, v, w only).
 *  SWC_VISC_STRESS out[9]: tau_ij = 2 rho_f nu S_ij with the face
 *                  densities rho_face[j] given, diffusion.py:33-67.
 *  SWC_VISC_HEAT   out[3]: heat flux -kappa_f dT/dx_j, T = p/(rho R),
 *                  diffusion.py:76-109 (reads rho, p only). */
enum { SWC_VISC_FLUX = 0, SWC_VISC_STRAIN = 1, SWC_VISC_STRESS = 2,
       SWC_VISC_HEAT = 3 };
int swc_viscous_terms(const SwcGrid* grid, int32_t dtype, int32_t what,
                      const void* const* q, const void* const* rho_face,
                      double nu, double pr, void* const* out, void* stream);

/* Stage algebra for a user-supplied rhs function, elementwise over `n`
 * entries with the modes of swc_rk_stage (rk3.py:69-83, rk2.py:67-86):
 * EULER: out = uk + l*dt; CONVEX: out = u0*c0 + (uk + l*dt)*c1;
 * AVERAGE: out = c0*(u0 + (uk + dt*l)). `dt` is a device double. */
int swc_rk_combine(int64_t n, int32_t dtype, int32_t mode, double c0,
                   double c1, const double* dt, const void* u0,
                   const void* uk, const void* l, void* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SWIRLC_B200_H_ */
