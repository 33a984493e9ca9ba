/*
 * dgsem_b200 -- B200-native (sm_100a) FP64 DGSEM right-hand side and fused
 * SSPRK3 stage update behind a plain C ABI.
 *
 * This ABI replaces the reference's compile-time plugin surface for the hot
 * path (RetrO598/DGSEM):
 *   StructuredSolver<Equations, Basis, VolumeFlux, SurfaceFlux, Mesh, BCs>
 *     ::calc_rhs(Solution&, T time)      src/solver/structured_solver.hpp:466-480
 *     ::set_indicator_parameters(...)    src/solver/structured_solver.hpp:118-123
 *     ::get_ndofs()                      src/solver/structured_solver.hpp:125
 *   SSPRK3<T, Solver, Mesh, Solution>::step(solver, sol, dt)
 *                                        src/time_integrator/SSPRK3.hpp:159-181
 *   HGIndicator<Basis, Eq>::operator()   src/subcell_limiting/indicator.hpp:337-418
 *   InitialFunctor::apply                src/boundary_condition/initial_functor.hpp:33-59
 * The template parameters become descriptor enums: equation
 * (compressible_euler2D/3D, compressible_navier_stokes2D), two-point volume
 * flux (ChandrashekarFlux + Ranocha, Kennedy-Gruber), surface flux
 * (LaxFriedrichsFlux + 2D HLLC), volume integral (VolumeIntegralSplitForm /
 * VolumeIntegralShockCapturingHG) and one boundary condition per mesh face
 * (BoundarySet of PeriodicBC, DirichletBC, OutflowBC,
 * MixedDirichletSlipWallBC; src/boundary_condition/ headers).
 *
 * Data layout on the device (all FP64, caller-owned):
 *   state u[e][var][node], e = ie + nx*(je + ny*ke), node = in + n*(jn + n*kn)
 * (node numbering = reference local_dof, src/utils/local_dof.hpp:9-19).
 * dgsem_to_reference_layout / dgsem_from_reference_layout convert to and from
 * the reference's logical u(i, j[, k], dof, var).
 *
 * All pointers passed to compute entry points are DEVICE pointers unless the
 * name says host.  Every call is asynchronous on the context's stream unless
 * documented otherwise; no entry point allocates or synchronises during a
 * step, so steps can be captured into CUDA graphs.  Errors are returned as
 * dgsem_status, never by aborting.
 */
#ifndef DGSEM_B200_H_
#define DGSEM_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum dgsem_status {
  DGSEM_OK = 0,
  DGSEM_ERR_INVALID_ARG = 1,
  DGSEM_ERR_UNSUPPORTED = 2,
  DGSEM_ERR_CUDA = 3,
  DGSEM_ERR_NONFINITE = 4,
  DGSEM_ERR_TIMEOUT = 5,
  DGSEM_ERR_ALLOC = 6,
  DGSEM_ERR_SCRATCH_LIMIT = 7  /* state larger than the static scratch */
} dgsem_status;

typedef enum dgsem_equation {
  DGSEM_EULER_2D = 0,          /* equations/compressible_euler2D.hpp */
  DGSEM_EULER_3D = 1,          /* equations/compressible_euler3D.hpp */
  DGSEM_NAVIER_STOKES_2D = 2,  /* equations/compressible_navier_stokes2D.hpp */
  DGSEM_NAVIER_STOKES_3D = 3   /* equations/compressible_navier_stokes3D.hpp (periodic boxes) */
} dgsem_equation;

typedef enum dgsem_volume_flux {
  DGSEM_VF_CHANDRASHEKAR = 0,  /* base/numerical_flux.hpp:436-594 */
  DGSEM_VF_RANOCHA = 1,        /* not in the reference: Ranocha (2018/2020) */
  DGSEM_VF_KENNEDY_GRUBER = 2  /* not in the reference: Kennedy-Gruber (2008) */
} dgsem_volume_flux;

typedef enum dgsem_surface_flux {
  DGSEM_SF_LAX_FRIEDRICHS = 0, /* base/numerical_flux.hpp:39-228 */
  DGSEM_SF_HLLC = 1            /* 2D normal-rotated form of numerical_flux.hpp:283-378 */
} dgsem_surface_flux;

typedef enum dgsem_volume_integral {
  DGSEM_VI_SPLIT_FORM = 0,         /* space_integral/volume_flux.hpp:686-739 */
  DGSEM_VI_SHOCK_CAPTURING_HG = 1  /* space_integral/volume_flux.hpp:741-879 */
} dgsem_volume_integral;

typedef enum dgsem_bc_kind {
  DGSEM_BC_PERIODIC = 0,          /* periodic_boundary.hpp:9-22 */
  DGSEM_BC_DIRICHLET_DMR = 1,     /* DirichletBC(double-Mach state f(x,t)) */
  DGSEM_BC_OUTFLOW = 2,           /* outflow_boundary.hpp:57-110 */
  DGSEM_BC_MIXED_DMR_WALL = 3,    /* MixedDirichletSlipWallBC, Dirichlet for x < 1/6 */
  DGSEM_BC_DIRICHLET_CONST = 4,   /* DirichletBC with a constant state */
  DGSEM_BC_SLIP_WALL = 5,         /* reflecting wall (MixedDirichletSlipWallBC wall branch) */
  /* Navier-Stokes adiabatic walls (navier_stokes_wall_boundary.hpp): the
   * reflected state for the inviscid flux, the wall value of the gradient
   * variables (no-slip: zero velocity; slip: no normal velocity) for BR1, the
   * inner viscous flux on the momentum (no-slip) or no viscous flux (slip) */
  DGSEM_BC_NS_NOSLIP_ADIABATIC_WALL = 6,
  DGSEM_BC_NS_SLIP_ADIABATIC_WALL = 7
} dgsem_bc_kind;

typedef enum dgsem_initial_kind {
  DGSEM_IC_KELVIN_HELMHOLTZ = 0,  /* examples/Euler2D/kelvin_helmholtz_hg */
  DGSEM_IC_DOUBLE_MACH = 1,       /* examples/Euler2D/double_mach_reflection:9-32 */
  DGSEM_IC_TAYLOR_GREEN_3D = 2,   /* examples/Euler3D/inviscid_tgv:18-35 */
  DGSEM_IC_TAYLOR_GREEN_2D = 3,   /* params[0] = p0 */
  DGSEM_IC_ISENTROPIC_VORTEX = 4  /* params = {beta, x0, y0} */
} dgsem_initial_kind;

typedef struct dgsem_mesh_desc {
  int ndims;                 /* 2 or 3 */
  int polydeg;               /* N; nodes per direction n = N + 1 (1 <= N <= 7) */
  int64_t n_cells[3];        /* elements per direction (unused entries ignored) */
  double domain_left[3];     /* StructuredMesh domain_left */
  double domain_right[3];    /* StructuredMesh domain_right */
} dgsem_mesh_desc;

typedef struct dgsem_scheme_desc {
  int equation;              /* dgsem_equation */
  int volume_flux;           /* dgsem_volume_flux (two-point flux of the split form) */
  int surface_flux;          /* dgsem_surface_flux */
  int volume_integral;       /* dgsem_volume_integral */
  int bc[6];                 /* dgsem_bc_kind per face: left, right, bottom, top, back, front */
  double bc_state[4];        /* conserved state for DGSEM_BC_DIRICHLET_CONST */
  double gamma;              /* ratio of specific heats */
  double mu;                 /* dynamic viscosity (Navier-Stokes) */
  double prandtl;            /* Prandtl number (Navier-Stokes) */
  double alpha_max;          /* set_indicator_parameters: alpha_max (default 0.5) */
  double alpha_min;          /* alpha_min (default 0.001) */
  int alpha_smooth;          /* stored, unused (as in the reference) */
} dgsem_scheme_desc;

typedef struct dgsem_ctx dgsem_ctx;

/* Human-readable name of a status code (static string). */
const char* dgsem_status_string(dgsem_status s);

/* Creates a solver context: basis and metric tables, stage temporaries and
 * the alpha buffer live in the context (replaces the StructuredSolver
 * constructors, structured_solver.hpp:36-58, and StructuredElementInitializer,
 * data_container.hpp:729-772).  `stream` is a cudaStream_t (NULL = legacy
 * default stream).  Synchronous; allocates device memory. */
dgsem_status dgsem_ctx_create(const dgsem_mesh_desc* mesh,
                              const dgsem_scheme_desc* scheme, void* stream,
                              dgsem_ctx** out);
dgsem_status dgsem_ctx_destroy(dgsem_ctx* ctx);
dgsem_status dgsem_ctx_set_stream(dgsem_ctx* ctx, void* stream);

/* Sizes: number of elements, nodes per element (n^d), variables, and the
 * total number of doubles of one state array (elements * nodes * nvars).
 * get_ndofs() of the reference is nodes_per_element. */
dgsem_status dgsem_get_sizes(const dgsem_ctx* ctx, int64_t* n_elements,
                             int* nodes_per_element, int* nvars,
                             int64_t* state_len);

/* set_indicator_parameters(alpha_max, alpha_min, alpha_smooth). */
dgsem_status dgsem_set_indicator_parameters(dgsem_ctx* ctx, double alpha_max,
                                            double alpha_min, int alpha_smooth);

/* du = RHS(u, t): calc_rhs (structured_solver.hpp:466-480). */
dgsem_status dgsem_rhs(dgsem_ctx* ctx, const double* u, double* du, double t);

/* One fused SSPRK3 stage: u_out = a*u_n + b*u_in + c*dt*RHS(u_in, t_stage),
 * stage 1: (0, 1, 1) at t, stage 2: (3/4, 1/4, 1/4) at t+dt,
 * stage 3: (1/3, 2/3, 2/3) at t+dt/2 (SSPRK3.hpp:159-181).  u_out may alias
 * u_n (stage 3 writes in place like the reference) but not u_in. */
dgsem_status dgsem_ssprk3_stage(dgsem_ctx* ctx, int stage, const double* u_n,
                                const double* u_in, double* u_out, double t,
                                double dt);

/* One SSPRK3 step in place (three fused stage launches; temporaries owned by
 * the context). */
dgsem_status dgsem_ssprk3_step(dgsem_ctx* ctx, double* u, double t, double dt);

/* nsteps SSPRK3 steps in place, t_k = t0 + k*dt. */
dgsem_status dgsem_ssprk3_steps(dgsem_ctx* ctx, double* u, double t0,
                                double dt, int nsteps);

/* One SSPRK3 step in place that allocates nothing (no counterpart in the
 * reference, whose integrator owns its stage Views).  Same kernels and the
 * same result as dgsem_ssprk3_step, but the two stage states live in one
 * static device array of this library instead of the context's temporaries.
 * For callers that must not allocate or free device memory while stepping:
 * a host code whose memory manager holds the GPU's memory in its own pool
 * (a cudaMalloc could fail or fragment it) or that cannot take the
 * device-wide synchronisation a cudaFree may bring; and for many small
 * contexts on one device that step one after another through one scratch.
 *  - Limit: the state may hold at most DGSEM_STATIC_SCRATCH_MAX_STATE doubles
 *    (2^21, 16 MiB; the scratch is 2 x 16 MiB per device); larger states
 *    return DGSEM_ERR_SCRATCH_LIMIT and launch nothing.
 *  - u must be device memory of the CURRENT device and the context must
 *    have been created with that device current; otherwise (a host pointer,
 *    another device's memory or context) DGSEM_ERR_INVALID_ARG.
 *  - The first call on a device is its set-up: it looks up the scratch's
 *    address (cudaGetSymbolAddress, which may load the module that holds
 *    the scratch).  Make that first call before any stream capture.  A
 *    failed set-up returns DGSEM_ERR_CUDA, clears the CUDA error state and
 *    is tried again by the next call.
 *  - Nothing has to start at zero: each stage state is fully written before
 *    it is read.
 *  - There is ONE scratch per device, shared by every context: two calls
 *    whose launches overlap (different streams, threads or contexts without
 *    ordering between them) race on it and give wrong results.  Order them
 *    on one stream or synchronise between them. */
#define DGSEM_STATIC_SCRATCH_MAX_STATE 2097152
dgsem_status dgsem_ssprk3_step_static_scratch(dgsem_ctx* ctx, double* u,
                                              double t, double dt);

/* Device address of stage state k (0: u^(1), 1: u^(2)) of the static scratch
 * on the current device, for inspection: after a
 * dgsem_ssprk3_step_static_scratch call has completed it holds that step's
 * stage state in its first state_len doubles.  Read-only for the caller. */
dgsem_status dgsem_static_scratch_state(int k, const double** out);

/* nsteps SSPRK3 steps on a HOST array (the reference's host-side view of
 * the state): copies u_host to the device, steps, copies back and
 * synchronises.  u_host should be pinned for full copy bandwidth. */
dgsem_status dgsem_ssprk3_steps_host(dgsem_ctx* ctx, double* u_host, double t0,
                                     double dt, int nsteps);

/* CUDA graph of nsteps SSPRK3 steps on the device state u (3*nsteps fused
 * stage kernels).  dgsem_graph_launch(g, t0) replays it on the context's
 * stream starting at time t0 (stage times read from a device clock, so
 * time-dependent boundary states stay correct).  The graph keeps pointers to
 * u and to the context's temporaries. */
typedef struct dgsem_graph dgsem_graph;
dgsem_status dgsem_graph_create(dgsem_ctx* ctx, double* u, double dt,
                                int nsteps, dgsem_graph** out);
dgsem_status dgsem_graph_launch(dgsem_graph* g, double t0);
dgsem_status dgsem_graph_destroy(dgsem_graph* g);

/* ---------------------------------------------------------------------
 * Batched mode (no counterpart in the reference, which advances one mesh per
 * solver instance): n_meshes independent periodic meshes sharing one scheme
 * (Euler, split form), each with its own degree, element counts and domain.
 * The states of all meshes live in one device array; mesh m occupies
 * [offsets[m], offsets[m+1]) in the single-mesh layout.  Per stage one fused
 * launch per distinct degree, the degrees running concurrently.
 * --------------------------------------------------------------------- */
typedef struct dgsem_batch dgsem_batch;
typedef struct dgsem_batch_graph dgsem_batch_graph;
dgsem_status dgsem_batch_create(const dgsem_mesh_desc* meshes, int n_meshes,
                                const dgsem_scheme_desc* scheme, void* stream,
                                dgsem_batch** out);
dgsem_status dgsem_batch_destroy(dgsem_batch* b);
/* offsets: n_meshes + 1 entries (doubles). */
dgsem_status dgsem_batch_offsets(const dgsem_batch* b, int64_t* offsets);
/* params: 3 doubles per mesh (see dgsem_initial_kind) or NULL. */
dgsem_status dgsem_batch_initial_condition(dgsem_batch* b, int kind,
                                           const double* params, double* u);
/* One SSPRK3 step of every mesh; dt_host[m] is mesh m's time step. */
dgsem_status dgsem_batch_ssprk3_step(dgsem_batch* b, double* u, double t,
                                     const double* dt_host);
/* CUDA graph of nsteps batched steps (3 * nsteps * n_degrees launches, the
 * degrees as parallel branches); replay on the batch's stream. */
dgsem_status dgsem_batch_graph_create(dgsem_batch* b, double* u,
                                      const double* dt_host, int nsteps,
                                      dgsem_batch_graph** out);
dgsem_status dgsem_batch_graph_launch(dgsem_batch_graph* g);
dgsem_status dgsem_batch_graph_destroy(dgsem_batch_graph* g);
dgsem_status dgsem_batch_check_finite(dgsem_batch* b);
/* Autotunes the launch shape of every degree group on the batch's meshes
 * (stage-1 launches into a batch temporary; u is not modified); chosen
 * receives one variant per distinct degree (ascending), may be NULL. */
dgsem_status dgsem_batch_autotune(dgsem_batch* b, double* u, const double* dt_host,
                                  int* chosen);
dgsem_status dgsem_batch_launch_count(const dgsem_batch* b, int64_t* count);
/* Persistent mode (2D batches, LLF surface flux): every stage is ONE launch
 * over the meshes of all degrees; each block of 256 threads walks a work list
 * of (degree, element tile) items, higher degrees first, and runs that
 * degree's node-parallel stage body.  Results agree with the per-degree
 * launches to rounding (the same stage body; bit for bit where the
 * compiler emits the same arithmetic).  DGSEM_ERR_UNSUPPORTED for other
 * batches.  Graphs record the mode they were captured in. */
/* Selects one launch shape (dgsem_set_launch_variant's numbering) for every
 * degree group of the batch, as dgsem_batch_autotune would after timing;
 * DGSEM_ERR_INVALID_ARG if a group's scheme lacks it. */
dgsem_status dgsem_batch_set_launch_variant(dgsem_batch* b, int variant);
dgsem_status dgsem_batch_set_persistent(dgsem_batch* b, int enable);

/* Hennemann-Gassner blending factor per element and troubled-cell flag
 * (alpha > max(100 eps, eps^0.75), volume_flux.hpp:772-773).  Either output
 * may be NULL. */
dgsem_status dgsem_indicator(dgsem_ctx* ctx, const double* u, double* alpha,
                             uint8_t* flags);

/* Nodal initial condition (InitialFunctor at the reference node
 * coordinates).  params may be NULL when the kind takes none. */
dgsem_status dgsem_initial_condition(dgsem_ctx* ctx, int kind,
                                     const double* params, double* u);

/* Layout conversions between the device layout and the reference's logical
 * LayoutRight u(i, j[, k], dof, var). */
dgsem_status dgsem_to_reference_layout(dgsem_ctx* ctx, const double* u,
                                       double* u_ref);
dgsem_status dgsem_from_reference_layout(dgsem_ctx* ctx, const double* u_ref,
                                         double* u);

/* Non-finite detection: every stage kernel ORs a device flag when it writes a
 * NaN/Inf.  This call synchronises the stream, returns DGSEM_ERR_NONFINITE if
 * the flag is set (DGSEM_ERR_TIMEOUT if a pipelined stage kernel gave up
 * waiting for a tile copy), and clears it. */
dgsem_status dgsem_check_finite(dgsem_ctx* ctx);

/* Launch-shape autotuner (no reference counterpart; the reference has one
 * fixed Kokkos launch shape).  The fused stage kernel has up to 7 launch
 * shapes: 0-2 line-parallel (elements per block, register cap), 3-4
 * node-parallel with and without a register cap, 5 persistent node-parallel
 * streaming element tiles through shared memory with bulk copies (no shock
 * capturing or viscous terms; 2D or even n in 3D), 6 node-parallel with two
 * nodes per thread (3D, n = 2 or 4, no shock capturing or viscous terms).  The shapes of each group run the same source: their
 * results agree bit for bit where the compiler emits the same arithmetic and
 * to rounding where a register cap changes which multiply-adds it fuses
 * (seen between 3 and 4 at n = 7 with the Ranocha flux); 3-5 agree with 0-2
 * to rounding (same fluxes and the same alpha and troubled-cell flags,
 * different summation order).  Every shape is deterministic.  dgsem_autotune times
 * one SSPRK3 step from state u (into the context temporaries; u is not
 * modified) with each available shape, 7 times in rounds that visit the
 * shapes in rotated order, keeps the one with the smallest median and returns
 * it in *chosen (may be NULL); times_ms (7 doubles, may be NULL; 0 for an
 * unavailable shape) receives the median step times and forces re-timing.
 * Every timed step is preceded by an L2 eviction (a 256 MiB temporary
 * buffer, freed before returning), i.e. states stream from HBM as in large
 * runs; with the environment variable DGSEM_AUTOTUNE_WARM set, steps are
 * timed back to back instead (L2-resident small meshes).  Choices are cached
 * per (scheme, degree, element count, timing mode) for the process and, when
 * the environment variable DGSEM_TUNING_FILE names a file, persisted there.
 * Synchronous. */
dgsem_status dgsem_autotune(dgsem_ctx* ctx, const double* u, int* chosen,
                            double* times_ms);
/* Selects a launch shape; DGSEM_ERR_INVALID_ARG if the scheme lacks it. */
dgsem_status dgsem_set_launch_variant(dgsem_ctx* ctx, int variant);

/* Fused per-step diagnostics (replaces the reference's AnalysisObserver with
 * VolumeAverageEuler, observer/analysis_observer.hpp:56-110,
 * analyzer/volume_average_euler.hpp:9-69, which re-read the state in a
 * separate reduction every analysed step): while enabled, the stage-3 launch
 * of every step (dgsem_ssprk3_stage 3, dgsem_ssprk3_step, graphs captured
 * while enabled) also integrates the state it writes over the mesh, block by
 * block: volume sum w, kinetic energy sum w |m|^2/(2 rho), entropy sum
 * w (-rho (ln p - gamma ln rho) / (gamma - 1)), w = quadrature weight / |1/J|
 * (volume_weighted_analyzer_functor.hpp:80,104).  Enabling allocates the
 * partial buffer once (3 doubles per element; call it outside stream
 * capture).  dgsem_diagnostics sums the partials of the last such launch in a
 * fixed order (deterministic), returns the volume and the volume means of
 * kinetic energy and entropy, and synchronises the stream.  The non-finite
 * check of every stage is dgsem_check_finite. */
dgsem_status dgsem_set_diagnostics(dgsem_ctx* ctx, int enable);
dgsem_status dgsem_diagnostics(dgsem_ctx* ctx, double* volume,
                               double* mean_kinetic_energy, double* mean_entropy);

/* Number of kernel launches issued by this context so far (diagnostics). */
dgsem_status dgsem_launch_count(const dgsem_ctx* ctx, int64_t* count);

/* ---------------------------------------------------------------------------
 * Discrete adjoint (no reference counterpart): transposed linearisation of
 * the forward kernels' arithmetic and of SSPRK3, for 2D periodic meshes with
 * the Chandrashekar split form, LLF surface flux, Euler or Navier-Stokes
 * (BR1).  Other schemes return DGSEM_ERR_UNSUPPORTED.
 * ------------------------------------------------------------------------- */
typedef struct dgsem_adjoint dgsem_adjoint;

/* Workspace for nsteps SSPRK3 steps with a checkpoint every checkpoint_every
 * steps: ceil(nsteps / every) saved states plus 3 * every stage states of
 * one segment, all in device memory. */
dgsem_status dgsem_adjoint_create(dgsem_ctx* ctx, int nsteps, int checkpoint_every,
                                  dgsem_adjoint** out);
dgsem_status dgsem_adjoint_destroy(dgsem_adjoint* adj);

/* out = (dR/du(u))^T w, with R the right-hand side of dgsem_rhs.  out must
 * not alias w. */
dgsem_status dgsem_adjoint_rhs_vjp(dgsem_adjoint* adj, const double* u,
                                   const double* w, double* out);

/* Volume-weighted mean kinetic energy J(u) = sum w |m|^2/(2 rho) / sum w
 * with w = w_i w_j / |1/J| (analyzer/volume_average_euler.hpp:9-69) to the
 * host (value, may be NULL; synchronises when given) and dJ/du to the device
 * array grad (may be NULL). */
dgsem_status dgsem_kinetic_energy(dgsem_adjoint* adj, const double* u,
                                  double* value, double* grad);

/* Gradient of J(u(t0 + nsteps dt)) with respect to the initial state u0:
 * forward SSPRK3 with checkpoints, then the reverse sweep (each segment's
 * stage states recomputed from its checkpoint, the last one recorded during
 * the forward pass).  u0 is not modified; *value receives J (may be NULL);
 * grad_u0 (device, state layout) receives dJ/du0 for every variable.
 * Synchronous. */
dgsem_status dgsem_adjoint_gradient(dgsem_adjoint* adj, const double* u0,
                                    double t0, double dt, double* value,
                                    double* grad_u0);

/* FP64 fused-multiply-add throughput of the current device (no reference
 * counterpart: the reference has no timers): one warm-up and one timed
 * launch of `iters` x 128 independent FMAs per thread on every SM, timed
 * with CUDA events on `stream` (a cudaStream_t).  *flops_per_s receives
 * 2 x FMAs / s (the FP64-pipe bound of the roofline), *ms the launch time
 * (may be NULL).  Synchronous; changes no clock or power setting. */
dgsem_status dgsem_fp64_fma_peak(void* stream, int iters, double* flops_per_s,
                                 double* ms);

/* ---------------------------------------------------------------------------
 * On-disk output without VTK.
 * VTU: replaces VTUOutputObserver::write_vtu (observer/vtu_output_observer.hpp:
 * 65-235) and write_vtu_lagrange_quad/hex (vtu_output_observer_impl.cpp:
 * 15-117): VTK XML UnstructuredGrid, one Lagrange quadrilateral (2D, cell type
 * 70) or hexahedron (3D, 72) of order N per element with its nodes in VTK's
 * Lagrange point order, point data rho, rhou, rhov[, rhow], rhoE, pressure
 * (pressure with the given / the context's gamma), appended raw binary data.
 * The device variant copies u (device layout) to the host and synchronises.
 * The host variant needs no GPU.
 * ------------------------------------------------------------------------- */
dgsem_status dgsem_write_vtu(dgsem_ctx* ctx, const double* u, const char* path);
dgsem_status dgsem_write_vtu_host(const dgsem_mesh_desc* mesh, double gamma,
                                  const double* u_host, const char* path);

/* Binary checkpoint / restart (no reference counterpart: the reference has no
 * restart): header (magic "DGSEMCKP", version, mesh and scheme descriptors,
 * time, step, state length) + the state in the device layout.  Reading
 * requires the same mesh (degree, cells, domain) and returns
 * DGSEM_ERR_INVALID_ARG otherwise.  Device variants copy through the host and
 * synchronise; host variants need no GPU. */
dgsem_status dgsem_checkpoint_write(dgsem_ctx* ctx, const double* u, double time,
                                    int64_t step, const char* path);
dgsem_status dgsem_checkpoint_read(dgsem_ctx* ctx, double* u, double* time,
                                   int64_t* step, const char* path);
dgsem_status dgsem_checkpoint_write_host(const dgsem_mesh_desc* mesh,
                                         const dgsem_scheme_desc* scheme,
                                         const double* u_host, double time,
                                         int64_t step, const char* path);
dgsem_status dgsem_checkpoint_read_host(const dgsem_mesh_desc* mesh, double* u_host,
                                        double* time, int64_t* step, const char* path);

/* Per-node geometry of an arbitrary structured mesh (curvilinear included),
 * computed on the device from its node coordinates with the reference's
 * formulas and operation order, bit for bit: Jacobian matrix, contravariant
 * vectors (2D adjugate, 3D conservative curl form) and inverse Jacobian
 * (StructuredContainerInitializer::calc_jacobian_matrix /
 * calc_contravariant_vectors / calc_inverse_jacobian,
 * containers/data_container.hpp:230-312, 420-692; the reference runs them on
 * the host inside StructuredElementInitializer::init_elements, :729-772).
 * Device arrays, element e = ie + nx*(je + ny*ke), node = i + n*(j + n*k):
 *   x[(e*d + c)*n^d + node]           node coordinates (input)
 *   ja[((e*d + a)*d + c)*n^d + node]  contravariant vector Ja^a_c (output)
 *   inv_j[e*n^d + node]               1/J (output)
 * n <= 8 in 2D, n <= 5 in 3D.  Asynchronous on `stream` (a cudaStream_t). */
dgsem_status dgsem_geometry_from_coordinates(int ndims, int polydeg,
                                             const int64_t* n_cells, const double* x,
                                             double* ja, double* inv_j, void* stream);

/* Host-side copies of the basis tables (nodes, weights, inv_weights,
 * lhat(-1), lhat(+1), D, Dsplit, Dhat, inverse Legendre Vandermonde; the
 * n x n tables row-major) for polydeg N; out needs 5n + 4n^2 doubles.
 * No GPU needed. */
dgsem_status dgsem_basis_tables_host(int polydeg, double* out);

/* Host-side reconstruction of the per-node metrics the kernels use
 * (contravariant vectors Ja^a_c and 1/J) in the reference's logical layout
 * ja(cells..., dof, a, c), inv_j(cells..., dof).  No GPU needed. */
dgsem_status dgsem_metrics_host(const dgsem_mesh_desc* mesh, double* ja,
                                double* inv_j);

/* Host-side node coordinates of the mesh's LinearMapping (the reference's
 * container.node_coordinates, data_container.hpp:729-772) in the logical
 * layout coords(cells..., dof, dim).  No GPU needed. */
dgsem_status dgsem_coordinates_host(const dgsem_mesh_desc* mesh, double* coords);

#ifdef __cplusplus
}
#endif

#endif /* DGSEM_B200_H_ */
