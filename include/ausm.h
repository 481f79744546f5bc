/*
 * libausm — B200 (sm_100a) CUDA library for the explicit TVD-RK3 time step of the
 * AUSM-family 2-D Euler solver on body-fitted O-grids (huj31415/ausm-webgpu).
 *
 * C ABI: plain pointers and sizes, every call returns an int status (AUSM_OK = 0,
 * negative = error; ausm_last_error() gives the message).  A solver handle owns its
 * device memory and one CUDA stream; calls on one handle must be serialised by the
 * caller, distinct handles may be driven from different host threads.
 *
 * Each entry point names the reference interface it replaces (file:line inside the
 * reference project).  The reference exposes its operator surface as browser globals
 * and hooks (src/main.js, src/util.js, src/grid.js); the mapping is:
 *   prepareGrid()            main.js:658-705   -> ausm_generate_grid
 *   prepareState()           main.js:631-655   -> ausm_init_state
 *   updateSolver(name)       main.js:629       -> ausm_set_scheme
 *   uni.values.*.set(...)    util.js:162-190   -> ausm_set_params
 *   frame loop (n steps)     main.js:744-791   -> ausm_step
 *   forceCalc/Integration    main.js:808-810   -> ausm_forces
 *   gridVtxData writes       grid.js:267-296   -> ausm_set_body_* / ausm_set_outer / ausm_set_vertices
 *   state textures           main.js:117-119   -> ausm_get_state / ausm_set_state
 */
#ifndef AUSM_H
#define AUSM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define AUSM_OK 0
#define AUSM_ERR_INVALID (-1)  /* bad argument or size */
#define AUSM_ERR_CUDA (-2)     /* CUDA runtime error */
#define AUSM_ERR_OOM (-3)      /* device allocation failed */
#define AUSM_ERR_DIVERGED (-4) /* max wave speed or residual norm is NaN/Inf */
#define AUSM_ERR_STATE (-5)    /* call out of order (no grid or no state yet) */
#define AUSM_ERR_BUDGET (-6)   /* serving: request does not fit the HBM budget */
#define AUSM_ERR_TIMEOUT (-7)  /* a bounded device-side wait gave up */
#define AUSM_ERR_NOT_FOUND (-8) /* serving: unknown request id */

/* flux schemes, in the reference's selector order (util.js:114-118) */
#define AUSM_SLAU2 0
#define AUSM_SLAU 1
#define AUSM_AUSMUP 2

/* initial state: the reference's fluid at rest (ausm.js:1-17) or uniform freestream */
#define AUSM_INIT_REST 0
#define AUSM_INIT_FREESTREAM 1

/* outer boundary: the reference's rectangle (grid.js:238-255) or a circle (grid.js:232) */
#define AUSM_OUTER_RECT 0
#define AUSM_OUTER_CIRCLE 1

/* elliptic grid iteration: the reference's Jacobi ping-pong in FP32 (shaders/grid.js:33-110,
 * main.js:691-694), or multicolour Gauss-Seidel in FP64 with a converged-move stop (the
 * FP64 vertices it produces give the FP64 face metrics and force integration) */
#define AUSM_GRID_JACOBI 0
#define AUSM_GRID_MULTICOLOR 1

/* step engines: one fused kernel per RK stage (default), or the reference's five
 * dispatches per stage (boundary, j-flux, i-flux, residual, RK combine) */
#define AUSM_ENGINE_FUSED 0
#define AUSM_ENGINE_REFERENCE 1
#define AUSM_ENGINE_F64 2 /* the reference-shaped engine in FP64 (precision study) */

/* headless field outputs (ausm.js:617-707 without colour mapping) */
#define AUSM_FIELD_DENSITY 0
#define AUSM_FIELD_PRESSURE 1
#define AUSM_FIELD_TEMPERATURE 2
#define AUSM_FIELD_MACH 3
#define AUSM_FIELD_ENTROPY 4
#define AUSM_FIELD_WAVE_SPEED 5

/* Physical and numerical parameters: the reference's uniform fields on the path
 * (util.js:1-29, defaults util.js:78-96, main.js:874-887).  The inflow velocity is
 * mach * sqrt(gamma * in_pressure / in_rho) rotated by aoa_deg (util.js:180-185); the
 * inflow state is (rho, rho u, rho v, p/(gamma-1) + rho |V|^2 / 2) (main.js:780-784). */
typedef struct AusmParams {
  double gamma;       /* ratio of specific heats (util.js:92) */
  double in_rho;      /* freestream density (util.js:94) */
  double in_pressure; /* freestream pressure (util.js:93) */
  double mach;        /* freestream Mach number */
  double aoa_deg;     /* angle of attack, degrees (util.js:90) */
  double K_p;         /* AUSM+-up pressure diffusion (util.js:95) */
  double K_u;         /* AUSM+-up velocity diffusion (util.js:96) */
  double cfl;         /* CFL factor (util.js:82) */
  double maxdt;       /* dt cap; +inf = none (util.js:78) */
  int muscl;          /* 1 = MUSCL/van Albada reconstruction (main.js:885) */
  int scheme;         /* AUSM_SLAU2 / AUSM_SLAU / AUSM_AUSMUP */
  double ramp;        /* inflow ramp strength (util.js:89, main.js:779); 0 = off */
} AusmParams;

typedef struct ausm_solver ausm_solver;

/* Fills the reference's defaults (util.js:78-96, main.js:877-885). */
int ausm_default_params(AusmParams* p);

/* Selects the CUDA device that later ausm_create calls on this host thread use
 * (the library links its own CUDA runtime, so a host's device choice must be passed
 * here; the reference runs on the browser's one adapter, main.js:9). */
int ausm_set_device(int device);
int ausm_device_count(int* count);

/* Creates a solver for an M (around the body, periodic) x N (radial) cell O-grid:
 * replaces main.js:102-151 (texture allocation).  M >= 4, N >= 2. */
int ausm_create(int M, int N, ausm_solver** out);
int ausm_destroy(ausm_solver* h);
/* Message of the last failed call on h (h == NULL: of the calling thread). */
const char* ausm_last_error(const ausm_solver* h);
int ausm_dims(const ausm_solver* h, int* M, int* N);

int ausm_set_engine(ausm_solver* h, int engine);
int ausm_set_params(ausm_solver* h, const AusmParams* p);   /* util.js:162-190 */
int ausm_get_params(const ausm_solver* h, AusmParams* p);
int ausm_set_scheme(ausm_solver* h, int scheme);            /* updateSolver, main.js:629 */

/* Body row j=0, CCW from the trailing edge.  NACA 4-digit formula of grid.js:38-52
 * (size = half chord, chord centred at x_offset; closed_te=1 keeps the reference's
 * -0.1036 quartic coefficient, which closes the trailing edge, 0 uses -0.1015). */
int ausm_set_body_naca4(ausm_solver* h, int digits, double size, double x_offset, int closed_te);
/* Host-only geometry (no handle, no GPU): the same generators as above, into xy[2*M]. */
int ausm_naca4_points(int M, int digits, double size, double x_offset, int closed_te, double* xy);
int ausm_outer_points(int M, int kind, double p0, double p1, double p2, double* xy);
/* Arbitrary body of exactly M points (a .dat airfoil sampled on the host, airfoilDatParser.js:280). */
int ausm_set_body_points(ausm_solver* h, const double* xy, int n);
/* Outer row j=N: AUSM_OUTER_RECT (p0 = half width / half height ratio, grid.js:238-255)
 * or AUSM_OUTER_CIRCLE (p0 = radius, centre (p1, p2)). */
int ausm_set_outer(ausm_solver* h, int kind, double p0, double p1, double p2);
/* Initial guess in j: first_spacing <= 0 is the reference's linear interpolation
 * (shaders/grid.js:24-27); > 0 is a geometric stretch with that first cell height. */
int ausm_set_radial_stretch(ausm_solver* h, double first_spacing);
/* prepareGrid (main.js:658-699): initial guess, `iters` TTM/Winslow sweeps (P=Q=0,
 * update only where the Jacobian is negative, shaders/grid.js:33-110), then metrics.
 * AUSM_GRID_MULTICOLOR stops early once the max vertex move is <= tol. */
int ausm_generate_grid(ausm_solver* h, int iters, int method, double tol, int* iters_done);
/* Vertices float2 M x (N+1) row-major (main.js:110, grid.js:33). */
int ausm_set_vertices(ausm_solver* h, const float* xy);
int ausm_get_vertices(ausm_solver* h, float* xy);

/* prepareState (main.js:631-655): fills the state, then the max wave speed for dt. */
int ausm_init_state(ausm_solver* h, int mode);
/* State in the reference layout: float4 (rho, rho u, rho v, rho E) x M x (N+3), row 0 the
 * wall ghost, rows 1..N interior, rows N+1, N+2 far-field ghosts (main.js:117, util.js:51).
 * set_state reads the interior rows; get_state writes the interior and the ghost rows
 * of the boundary pass applied to that interior (ausm.js:34-120). */
int ausm_set_state(ausm_solver* h, const float* q);
int ausm_get_state(ausm_solver* h, float* q);
/* The same layout in double: the F64 engine's state as it is, the FP32 engines' state
 * widened (no counterpart in the reference, which is FP32 only). */
int ausm_get_state_f64(ausm_solver* h, double* q);

/* step(n): dt = min(maxdt, cfl / max wave speed) of the current state, held for n
 * TVD-RK3 steps, then the max wave speed of the new state (main.js:744-791).  dt_out
 * may be NULL (then the call does not wait for the GPU).  A tile whose bounded wait
 * gave up (AUSM_ERR_TIMEOUT) is reported by this call when it waits (dt_out given),
 * else by the next call on the handle that waits for the GPU (get_state, forces,
 * residual_l2, field, max_wave_speed, synchronize, time_steps or a step with dt_out). */
int ausm_step(ausm_solver* h, int n, float* dt_out);
int ausm_max_wave_speed(ausm_solver* h, float* out);

/* Surface force (per wall face graphs.js:5-41, sum and coefficients graphs.js:43-103)
 * with FP64 accumulation: out[6] = Fx, Fy,
 * |F| sign(F.V), Cl, Cd, Cl/Cd (coefficients per the reference, not divided by chord);
 * cp (may be NULL) gets M wall pressure coefficients (p - p_inf) / q_inf. */
int ausm_forces(ausm_solver* h, double* out6, double* cp);
/* sqrt(mean(R_rho^2)) over the interior of the current state, FP64 accumulation. */
int ausm_residual_l2(ausm_solver* h, double* l2);
/* Headless field output: M x N floats of AUSM_FIELD_* for the interior. */
int ausm_field(ausm_solver* h, int kind, float* out);

/* Surface force and wall Cp without allocating anything (no counterpart in the
 * reference).  For hosts that cannot call cudaMalloc where they need the forces: hosts
 * that own all device memory through their own pool or arena, hosts that must not
 * trigger the implicit synchronisation an allocation can cause, and hosts that keep the
 * state in their own device buffers without a solver handle.  wall_row: device pointer
 * to the M float4 conserved states of the first interior row (row 1 of the reference
 * layout); body_xy: device pointer to the M float2 body vertices (vertex row 0);
 * out6 and cp (M values, may be NULL) are host pointers, filled as by ausm_forces with
 * the inflow speed mach * sqrt(gamma p / rho) of *p.  stream may be NULL (legacy
 * default stream); the call waits for it.  Scratch is one fixed array per device of
 * 3 * 16384 + 2 doubles, so M above 16384 is rejected with AUSM_ERR_INVALID.  The
 * first call on each device looks up that array's device address, so make it before
 * any stream capture.  Calls share the array: two calls that overlap on the GPU race. */
int ausm_forces_noalloc(const void* wall_row, const void* body_xy, int M, const AusmParams* p, double* out6,
                        double* cp, void* stream);

/* Device stream of the handle (cudaStream_t) and a blocking wait on it. */
int ausm_stream(ausm_solver* h, void** stream);
int ausm_synchronize(ausm_solver* h);
/* Device-timed loop for benchmarks: `reps` calls of step(n) bracketed by CUDA events
 * on the handle's stream; ms_out gets the elapsed device time of all of them. */
int ausm_time_steps(ausm_solver* h, int n, int reps, float* ms_out);
/* Test hook (no counterpart in the reference): the number of polls, 0 to 65536 (the
 * default), of the first bounded wait of every TMA box of the stage kernels on the
 * current device, in this process.  0 makes every such wait give up at once, so a test
 * can drive the timeout path without a fault: the tiles report AUSM_ERR_TIMEOUT, write
 * nothing, and still let their copies land (second wait, full bound) before they exit.
 * The call waits for the device to be idle, so work queued before it keeps the bound it
 * was queued under.  Restore 65536 afterwards. */
int ausm_debug_set_wait_polls(unsigned polls);
/* Tile-height autotuner of the fused engine (no counterpart in the reference): times
 * the TMA stage kernel for tiles of 32 x 8, 32 x 16 and 32 x 32 cells on this solve's
 * grid and state and keeps the fastest for its steps (cached per M, N and scheme for the
 * process; force = 1 re-measures).  The first ausm_step of an untuned solve runs it
 * implicitly, so call it before capturing steps in a CUDA graph.  AUSM_TILE_ROWS=8|16|32
 * fixes the height, AUSM_AUTOTUNE=0 keeps 16.  *rows gets the height in use. */
int ausm_autotune(ausm_solver* h, int force, int* rows);

/* ---- batches: many solves advanced together (no counterpart in the reference) ----
 * The reference steps one grid per page.  A batch steps any number of independent
 * fused-engine solvers of any grid sizes and schemes with one kernel launch per RK
 * stage and scheme: the work list is every member's 32 x TY cell tiles end to end (TY
 * chosen by the batch's tile-height tuning), one CTA per tile.  Each
 * member keeps its own dt (from its own max wave speed, held over the n steps as
 * ausm_step does), so a member's results are the same alone or in any batch.  While a
 * solver is a member, its calls run on the batch's stream (ausm_stream returns it) and
 * its engine cannot change; destroying a member removes it first.  A member may belong
 * to one batch.  With graphs on (the default) the n-step sequence is captured once per
 * (membership, n) as a CUDA graph and replayed. */
typedef struct ausm_batch ausm_batch;
/* New empty batch on the current device. */
int ausm_batch_create(ausm_batch** out);
int ausm_batch_destroy(ausm_batch* b);
const char* ausm_batch_last_error(const ausm_batch* b);
/* Add a solver that has a grid and a state (fused engine, same device). */
int ausm_batch_add(ausm_batch* b, ausm_solver* h);
/* Remove a member; AUSM_ERR_NOT_FOUND if h is not one. */
int ausm_batch_remove(ausm_batch* b, ausm_solver* h);
int ausm_batch_size(const ausm_batch* b, int* n);
/* Member k (in order of addition, removals close the gap). */
int ausm_batch_member(const ausm_batch* b, int k, ausm_solver** h);
int ausm_batch_set_graphs(ausm_batch* b, int enable);
/* n RK3 steps of every member.  dt_wave (2 floats per member, may be NULL): the dt used
 * and the max wave speed after the steps; with it the call waits for the GPU and
 * returns AUSM_ERR_DIVERGED (after filling dt_wave) when a member's wave speed is not
 * finite.  Without it the call only enqueues the work. */
int ausm_batch_step(ausm_batch* b, int n, float* dt_wave);
/* Density-residual L2 norm of every member's current state (as ausm_residual_l2), one
 * double per member; waits for the GPU. */
int ausm_batch_residual_l2(ausm_batch* b, double* l2);
int ausm_batch_synchronize(ausm_batch* b);
/* Device-timed loop: `reps` calls of ausm_batch_step(b, n, NULL); ms_out gets the
 * elapsed device time of all of them. */
int ausm_batch_time_steps(ausm_batch* b, int n, int reps, float* ms_out);

/* ---- serving: continuous batching of solve requests (no counterpart in the reference) ----
 * A server admits requests (airfoil, grid size, flow, scheme, stopping rule) as they
 * arrive, in arrival order, while the HBM budget and the slot count allow; keeps their
 * state resident on the device in one batch; advances the batch in rounds of
 * `chunk_steps` RK3 steps (dt held per round, as one reference frame); after each round
 * checks every member's density-residual L2 norm (FP64) against its own stopping rule
 * and retires the finished ones with their forces and surface Cp (FP64), freeing their
 * memory for the next arrivals.  A request's steps are counted from its admission, so
 * its result is the same whether it runs alone or among others.  Requests are rejected
 * at submit on the host (invalid or non-finite fields: AUSM_ERR_INVALID; larger than
 * the whole budget: AUSM_ERR_BUDGET).  A request that diverges ends with state
 * AUSM_ERR_DIVERGED and does not affect the others. */
typedef struct AusmRequest {
  int M, N;              /* cells around the body (periodic) x radial */
  int naca4;             /* NACA 4-digit code, used when body_xy is NULL */
  int closed_te;         /* 1: closed trailing edge (-0.1036 coefficient) */
  const double* body_xy; /* optional M body vertices (x, y) from a .dat loader; copied */
  double chord;          /* NACA chord; the body spans x in [-chord/2, chord/2] */
  double far_radius;     /* circular far field radius, centred at the origin */
  double first_spacing;  /* first radial cell height of the initial grid; 0 = uniform */
  int grid_iters;        /* multicolor TTM sweeps */
  int init_mode;         /* AUSM_INIT_* */
  AusmParams params;
  double residual_drop;  /* stop after this many decades of density-residual L2 drop */
  int max_steps;         /* ... or after this many RK3 steps (rounded up to whole rounds) */
} AusmRequest;

#define AUSM_REQ_DONE 0    /* state: finished (see stop) */
#define AUSM_REQ_QUEUED 1  /* state: waiting for admission */
#define AUSM_REQ_RUNNING 2 /* state: on the device */
#define AUSM_STOP_CONVERGED 1
#define AUSM_STOP_MAX_STEPS 2
#define AUSM_STOP_DIVERGED 3

typedef struct AusmResult {
  int64_t id;
  int state;      /* AUSM_REQ_* or a negative status (the request failed) */
  int stop;       /* AUSM_STOP_* once finished */
  int M, N;
  int steps;      /* RK3 steps taken */
  double l2_first; /* density-residual L2 of the initial state */
  double l2_last;  /* ... after the last round */
  double forces[6]; /* Fx, Fy, |F| sign, Cl, Cd, Cl/Cd as ausm_forces */
  double queue_ms;  /* submit -> admission */
  double run_ms;    /* admission -> finished */
  double latency_ms; /* submit -> finished */
} AusmResult;

typedef struct AusmServerStats {
  int64_t submitted, rejected, admitted, finished, failed, rounds;
  int pending, active;
  double bytes_in_use, peak_bytes, cell_updates;
} AusmServerStats;

#define AUSM_SERVE_PLAIN 1   /* flag: no batch; one solve at a time, ausm_step per round */
#define AUSM_SERVE_NO_GRAPH 2 /* flag: batch without CUDA graphs */

typedef struct ausm_server ausm_server;
/* New server on the current device.  hbm_budget_bytes: device memory its solves may
 * hold at once; max_active: slots (concurrent solves); chunk_steps: RK3 steps per round.
 * No CUDA call happens until the first round. */
int ausm_server_create(double hbm_budget_bytes, int max_active, int chunk_steps, int flags, ausm_server** out);
int ausm_server_destroy(ausm_server* s);
const char* ausm_server_last_error(const ausm_server* s);
/* Device bytes a request holds while admitted (what admission charges to the budget). */
int ausm_request_bytes(const AusmRequest* r, double* bytes);
/* Queues a request; *id identifies it.  Thread-safe. */
int ausm_server_submit(ausm_server* s, const AusmRequest* r, int64_t* id);
/* One round on the calling thread: admit, step, check, retire.  *active gets the
 * number of solves left on the device or queued.  Use either this or the worker. */
int ausm_server_pump(ausm_server* s, int* remaining);
/* Starts / stops a worker thread that pumps whenever requests are queued or active. */
int ausm_server_start(ausm_server* s);
int ausm_server_stop(ausm_server* s);
/* Result of request id (state AUSM_REQ_QUEUED / RUNNING until done); cp (may be NULL)
 * gets the M wall Cp values once done.  AUSM_ERR_NOT_FOUND for an unknown id. */
int ausm_server_poll(ausm_server* s, int64_t id, AusmResult* res, double* cp);
/* Waits until nothing is queued or active (the worker must be running, or the call
 * pumps on this thread); timeout_ms < 0 waits without limit.  AUSM_ERR_TIMEOUT if the
 * time ran out first. */
int ausm_server_drain(ausm_server* s, double timeout_ms);
int ausm_server_stats(ausm_server* s, AusmServerStats* st);

#ifdef __cplusplus
}
#endif
#endif /* AUSM_H */
