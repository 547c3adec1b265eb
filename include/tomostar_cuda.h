/*
 * tomostar_cuda.h — C ABI of libtomostar_cuda.so, the B200 (sm_100a) forward engine of TomoSTAR.
 *
 * The C# host binds it with [DllImport("tomostar_cuda")] (the native-library convention of
 * src/TomoStar.Core/Compute/MpiSession.cs:158-168) behind the interfaces the OpenCL backend
 * implements today:
 *   - src/TomoStar.Core/Forward/EikonalOpenCl.cs (TryCreate, SuggestBatch, TrySolve, SelfTest),
 *   - the per-arrival body of src/TomoStar.Core/Tomography/RayKernels.cs:67-107
 *     (RayTracing.Backtrack + RayTracing.Kernel), which has no device interface in the reference.
 *
 * Conventions: nothing throws or aborts across the boundary. Every entry point returns TS_OK (0)
 * or a TS_E_* code, and ts_last_error() gives the text (the `reason` of TrySolve). Arrays are
 * caller-owned host memory passed by pointer; device memory is owned by the context. Calls on one
 * context are serialised internally (as EikonalOpenCl's lock(_gate), EikonalOpenCl.cs:64,165).
 * There is no CPU fallback inside any entry point: a device failure is returned as an error.
 */
#ifndef TOMOSTAR_CUDA_H
#define TOMOSTAR_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TS_OK 0
#define TS_E_ARG 1        /* invalid argument (sizes, pointers, grid) */
#define TS_E_CUDA 2       /* a CUDA call failed; text in ts_last_error */
#define TS_E_NOMEM 3      /* device memory exhausted */
#define TS_E_UNSETTLED 4  /* "sweeping not settled after N rounds" (EikonalOpenCl.cs:269) */
#define TS_E_CANCELLED 5  /* the cancel flag was raised (CancellationToken, EikonalOpenCl.cs:243,262) */
#define TS_E_TIMEOUT 6    /* a bounded device-side wait ran out; the context stays usable */
#define TS_E_CAPACITY 7   /* an output buffer is too small; the needed size is reported */
#define TS_E_NOSEEDS 8    /* "no seed nodes" (EikonalOpenCl.cs:164) */
#define TS_E_SELFTEST 9   /* the device disagreed with the host solver beyond the gate */
#define TS_E_NODEVICE 10  /* no CUDA device */

#define TS_PRECISION_F64 64
#define TS_PRECISION_F32 32

/* Solve modes of ts_eik_solve. */
#define TS_MODE_ENGINE 0  /* batched tiled engine: tile-wavefront sweeps, one cooperative launch */
#define TS_MODE_PLAIN 1   /* the reference scheme as-is: one launch per diagonal plane, one field at a time */
#define TS_MODE_FAST 2    /* the engine where a node wakes its neighbours only when it dropped by more than
                             TS_WAKE_REL of its time: last-digit changes are not propagated, so far fewer
                             nodes are re-evaluated; FP64 results stay within ~1e-11 relative of
                             TS_MODE_ENGINE's (which equal the reference's to the bit) */
#define TS_WAKE_REL 1e-13

/* Output element types. TS_OUT_NONE keeps the fields on the device (ts_eik_solve_model only). */
#define TS_OUT_F64 0
#define TS_OUT_F32 1
#define TS_OUT_NONE 2

typedef struct ts_ctx ts_ctx;

/* GridDefinition (src/TomoStar.Core/Geo/SphericalGrid.cs:13-31). depth_km (extension, not in the
 * reference): nz increasing depths for a variable vertical spacing, or NULL for the uniform grid. */
typedef struct ts_grid {
    double min_lon, max_lon, min_lat, max_lat, min_depth_km, max_depth_km;
    int32_t nx, ny, nz, reserved;
    const double* depth_km;
} ts_grid;

typedef struct ts_eik_stats {
    int32_t rounds[2];      /* rounds of eight sweeps per phase, largest over the batch (LastStats) */
    int32_t launches;       /* kernel launches made by the solve */
    int32_t reserved;
    int64_t node_updates;   /* node evaluations performed (one per node per tile or plane visit) */
    int64_t tile_visits;    /* tiles processed (engine) or planes launched (plain) */
    double device_ms;       /* CUDA-event time of the solve on the device (set-up kernels included) */
    double kernel_ms;       /* CUDA-event time of the sweeping kernel launches alone */
} ts_eik_stats;

/* ---- context (EikonalOpenCl.TryCreate / Dispose / Device) ----------------------------------- */

/* Creates a context on a CUDA device (EikonalOpenCl.TryCreate, EikonalOpenCl.cs:88-118, without
 * the self-test: call ts_cuda_selftest, as TryCreate does at :109-115, before trusting it). */
int ts_cuda_create(int32_t device, ts_ctx** out);
void ts_cuda_destroy(ts_ctx* ctx);                       /* EikonalOpenCl.Dispose (:376-384) */
const char* ts_last_error(ts_ctx* ctx);                  /* the `reason` strings of TrySolve */
int ts_device_name(ts_ctx* ctx, char* buf, int32_t cap); /* EikonalOpenCl.Device (:83) */
const char* ts_last_stats(ts_ctx* ctx);                  /* EikonalOpenCl.LastStats (:86) */
/* Raises or clears the cancel flag polled between rounds (CancellationToken of TrySolve). */
void ts_set_cancel(ts_ctx* ctx, int32_t cancel);

/* Fields of `nodes` nodes per batch that fit this device (EikonalOpenCl.SuggestBatch, :121-132);
 * the engine caps it at 1024 instead of 32 because it has no per-plane launch cost to amortise. */
int32_t ts_eik_suggest_batch(ts_ctx* ctx, int64_t nodes, int32_t precision);

/* ---- eikonal ----------------------------------------------------------------------------------- */

/* SphericalEikonal.PointSource (Forward/SphericalEikonal.cs:68-100) on the host: the seed nodes
 * of a point source. Returns the seed count; when it exceeds cap, nothing is written past cap and
 * the count needed is returned. radius_cells is the reference's default 3. */
int32_t ts_point_source(const ts_grid* grid, const double* slowness, double lon, double lat, double depth_km,
                        double origin_time, double radius_cells, int32_t* idx_out, double* t_out, int32_t cap);

/* EikonalOpenCl.TrySolve (EikonalOpenCl.cs:138-166): one field per seed set, all on one grid and
 * one slowness (double[n], grid order, x fastest). Seed set f is seed_index/seed_time
 * [seed_offsets[f], seed_offsets[f+1]); out-of-range indices are ignored and duplicates take the
 * smallest time. precision: TS_PRECISION_F64 (result equals SphericalEikonal.Relax to the bit) or
 * TS_PRECISION_F32. mode: TS_MODE_ENGINE or TS_MODE_PLAIN. tol: settle tolerance of a round, s
 * (the reference's 1e-7; 0 runs to the exact fixed point). max_rounds <= 0 uses the reference cap
 * max(32, (nx+ny+nz)/4) per phase. out: n_fields*n values, field-major, of out_type; unreached
 * nodes are +inf. Returns TS_E_UNSETTLED, like TrySolve's refusal, if any field did not settle. */
int ts_eik_solve(ts_ctx* ctx, const ts_grid* grid, const double* slowness, int32_t n_fields,
                 const int32_t* seed_offsets, const int32_t* seed_index, const double* seed_time, int32_t precision,
                 int32_t mode, double tol, int32_t max_rounds, void* out, int32_t out_type, ts_eik_stats* stats);

/* Resident models (ForwardModel, Forward/TravelTimeTable.cs:167-241, kept on the device between
 * solves the way TravelTimeTableSet reuses tables by ModelKey, :176-183, 278-279): the slowness of
 * n_phases phases (phase p at p*n) and the grid's metric, uploaded once in `precision`. */
int ts_model_put(ts_ctx* ctx, const ts_grid* grid, const double* slowness, int32_t n_phases, int32_t precision,
                 int32_t* model_id);
int ts_model_drop(ts_ctx* ctx, int32_t model_id);
/* ts_eik_solve on a resident model's phase (no slowness upload). out_type TS_OUT_NONE leaves the
 * fields on the device (out may be NULL); otherwise as ts_eik_solve. */
int ts_eik_solve_model(ts_ctx* ctx, int32_t model_id, int32_t phase, int32_t n_fields, const int32_t* seed_offsets,
                       const int32_t* seed_index, const double* seed_time, int32_t mode, double tol,
                       int32_t max_rounds, void* out, int32_t out_type, ts_eik_stats* stats);

/* ts_eik_solve_noalloc — no counterpart in the reference. The plain FP64 solve of one field for a
 * caller that cannot allocate device memory: for instance a process whose device memory is all held
 * by another allocator (a framework's caching pool, a serving budget reserved at start-up), a plug-in
 * host that forbids device allocation after initialisation, or a latency-critical path that cannot
 * take an allocation's implicit synchronisation. The caller passes its own device buffers:
 * slowness_dev (nx*ny*nz doubles, grid order) and field_dev (the same size, written), both device memory
 * of the calling thread's current device (anything else is refused with TS_E_ARG); seeds are host
 * arrays as in ts_eik_solve. The function allocates no device memory: its working memory (due and
 * fixed-node flags, axis weights, seeds, the round flag) is one static __device__ array of about
 * 13 MB that every GPU which loads the library holds until the process exits. Limits: uniform grids
 * (depth_km NULL), nx*ny*nz <= TS_NOALLOC_MAX_NODES, ny*nz <= TS_NOALLOC_MAX_ROWS,
 * nz <= TS_NOALLOC_MAX_LEVELS, at most TS_NOALLOC_MAX_SEEDS distinct seed nodes; larger inputs
 * return TS_E_CAPACITY. Every call looks up the array's address (cudaGetSymbolAddress) on the current
 * device, so a device reset leaves no stale address behind; the first call on a device is also where
 * the library's device code is loaded there: make that first call before any stream capture.
 * All calls share the one array, so calls that overlap on the GPU (other host threads, other
 * streams) race: serialise them. The result equals SphericalEikonal.Relax to the bit (the reference
 * scheme, one launch per diagonal plane, on `stream`, NULL for the default stream). rounds_out[2]
 * receives the rounds of each phase. Errors: text in ts_last_error(NULL). */
#define TS_NOALLOC_MAX_NODES 4194304
#define TS_NOALLOC_MAX_ROWS 262144
#define TS_NOALLOC_MAX_LEVELS 8192
#define TS_NOALLOC_MAX_SEEDS 65536
int ts_eik_solve_noalloc(const ts_grid* grid, const double* slowness_dev, int32_t n_seeds, const int32_t* seed_index,
                         const double* seed_time, double* field_dev, double tol, int32_t max_rounds, void* stream,
                         int32_t* rounds_out);

/* EikonalOpenCl.SelfTest (EikonalOpenCl.cs:346-374): the reference's 22x20x16 heterogeneous case
 * solved on the device and by the host sweeping solver; *rel_err = max |dt| / field range. The
 * gate passes when *rel_err <= 1e-6 (SelfTestTolerance, :45); otherwise TS_E_SELFTEST. */
int ts_cuda_selftest(ts_ctx* ctx, int32_t precision, double* rel_err, char* msg, int32_t cap);

/* Engine tile shapes compiled into the library: writes up to cap (id, bx, by, bz) quadruples to
 * shapes and returns how many exist. No reference counterpart (the OpenCL kernel is untiled). */
int32_t ts_engine_shapes(int32_t* shapes, int32_t cap);
/* Selects the engine's tile shape for one precision on this context (the autotuner's knob). */
/* Engine scheduler: 0 = all fields step through the tile diagonals together (one grid-wide barrier
 * per diagonal); 1 = flow: each field advances on its own through a shared tile queue (no barrier).
 * Both give the same fields. No reference counterpart. */
int ts_engine_set_scheduler(ts_ctx* ctx, int32_t scheduler);
int ts_engine_set_tile(ts_ctx* ctx, int32_t precision, int32_t shape_id);

/* Many fields on grids of uneven size in one engine launch (the reference batches only fields of one
 * grid and slowness, EikonalOpenCl.TrySolve). Grid g (grids[g], slowness[g]: its nx*ny*nz values on
 * the host) may have a variable depth array. Field f lies on grid field_grid[f] with seeds
 * [seed_offsets[f], seed_offsets[f+1]). mode: TS_MODE_ENGINE or TS_MODE_FAST. out: the fields one
 * after another, each its grid's nx*ny*nz values of out_type, or nothing with TS_OUT_NONE. */
int ts_eik_solve_multi(ts_ctx* ctx, int32_t n_grids, const ts_grid* grids, const double* const* slowness,
                       int32_t n_fields, const int32_t* field_grid, const int32_t* seed_offsets, const int32_t* seed_index,
                       const double* seed_time, int32_t precision, int32_t mode, double tol, int32_t max_rounds,
                       void* out, int32_t out_type, ts_eik_stats* stats);
/* Captures each one-shot engine solve into a CUDA graph and replays it while the same job (the same
 * grids, fields and seeds on the same buffers) is solved again. No reference counterpart. */
int ts_engine_set_graph(ts_ctx* ctx, int32_t enable);
int32_t ts_engine_graph_replays(ts_ctx* ctx);
/* Times every tile shape under both schedulers on a sample batch (ts_eik_solve_multi arguments, best
 * of `repeats`), selects the fastest pair for `precision` on this context and returns it;
 * ms_per_shape[2q + s] receives shape q's time under scheduler s (up to cap entries). No reference
 * counterpart. */
int ts_engine_autotune(ts_ctx* ctx, int32_t n_grids, const ts_grid* grids, const double* const* slowness,
                       int32_t n_fields, const int32_t* field_grid, const int32_t* seed_offsets, const int32_t* seed_index,
                       const double* seed_time, int32_t precision, int32_t mode, int32_t repeats, int32_t* best_tile,
                       int32_t* best_scheduler, double* ms_per_shape, int32_t cap);

/* ---- serving: a resident request loop with continuous batching (no reference counterpart) ----
 * A server owns its own context on `device` and one loop thread. Models are put once and stay on
 * the device. Requests (fields on one model and phase, optionally rays traced on those fields) are
 * queued in arrival order, admitted while their device footprint (engine buffers and float32
 * tables of their fields) fits in hbm_budget_bytes, and solved by the engine in epochs of
 * rounds_per_epoch sweep rounds over every field in flight, so requests that arrive while others
 * run join the next epoch. A field's result does not depend on the requests it ran with. Rows of
 * a finished request belong to the caller (ts_rows_free) and must be freed before
 * ts_serve_destroy. All calls are thread-safe. */
typedef struct ts_server ts_server;
typedef struct ts_rows ts_rows;  /* ray rows, see below */
typedef struct ts_serve_request {
    int32_t model_id;             /* from ts_serve_model_put */
    int32_t phase;
    int32_t n_fields;
    int32_t n_rays;
    const int32_t* seed_offsets;  /* n_fields + 1, into seed_index / seed_time (copied at submit) */
    const int32_t* seed_index;
    const double* seed_time;
    const double* field_origin;   /* 3 per field (lon, lat, depth km): where rays of the field end */
    const int32_t* ray_field;     /* n_rays: the field each ray is traced on */
    const double* ray_event;      /* 3 per ray: the ray's start (the event) */
    const ts_grid* inv;           /* grid of the rows' columns; NULL: the forward grid coarsened by 2 */
    double step_km;               /* <= 0: the RayKernels step (RayKernels.cs:62) */
    float* tables_out;            /* NULL, or n_fields * nx*ny*nz floats, filled before completion */
} ts_serve_request;
typedef struct ts_serve_result {
    int32_t status;               /* TS_OK or the request's error code */
    int32_t n_fields;
    int32_t rounds[2];            /* sweep rounds per phase, the largest over its fields */
    double queue_ms;              /* submit → admission */
    double latency_ms;            /* submit → completion (tables and rays done) */
    ts_rows* rows;                /* the rays' rows (NULL without rays); the caller frees them */
    char error[160];
} ts_serve_result;
typedef struct ts_serve_stats_t {
    int64_t epochs, fields_done, requests_done, node_updates;
    double device_ms;             /* engine kernel time */
    double epoch_ms;              /* wall time of the epochs (kernel, its set-up and read-back) */
    double complete_ms;           /* wall time of finishing requests (tables, rays, copies) */
    double bytes_in_use, peak_bytes;
    int32_t queued, in_flight;
} ts_serve_stats_t;
int ts_serve_create(int32_t device, int32_t precision, int32_t mode, int32_t tile, int32_t scheduler,
                    double hbm_budget_bytes, int32_t rounds_per_epoch, ts_server** out);
void ts_serve_destroy(ts_server* server);
/* Flow scheduler only: an epoch ends once `ms` have passed, each field pausing at its next round
 * end (and at rounds_per_epoch rounds at the latest), so that fields of small grids keep the device
 * busy while larger ones finish their rounds. 0: rounds only. */
int ts_serve_set_epoch_ms(ts_server* server, double ms);
const char* ts_serve_last_error(ts_server* server);
int ts_serve_model_put(ts_server* server, const ts_grid* grid, const double* slowness, int32_t n_phases,
                       int32_t* model_id);
int ts_serve_submit(ts_server* server, const ts_serve_request* request, int64_t* request_id);
/* Waits up to timeout_s (< 0: for ever) for a request; TS_E_TIMEOUT if it is not done yet. A
 * request can be waited for once: its result (and rows) then pass to the caller. */
int ts_serve_wait(ts_server* server, int64_t request_id, double timeout_s, ts_serve_result* result);
int ts_serve_stats(ts_server* server, ts_serve_stats_t* stats);

/* ---- rays and Jacobian rows (RayKernels.Compute's per-arrival body) ---------------------------- */

typedef struct ts_rows ts_rows;

/* Traces rays on travel-time tables and integrates them on the inversion grid
 * (RayTracing.Backtrack, Forward/RayTracing.cs:73-111; RayTracing.Kernel, :118-159; row
 * finalisation, Tomography/RayKernels.cs:79-97). tables: n_tables float32 fields on fwd (the
 * .qttb values, TravelTimeTable.cs:73); table_station: 3 doubles (lon, lat, depth) per table (the
 * table header's station). Ray a starts at events[3a..3a+2] on table table_of[a]. step_km: the
 * RayKernels step 0.5·min(forward, inversion MinSpacingKm). Produces one CSR row per ray (nodes
 * ascending, float32 lengths), TCalc and the source gradient; a ray the reference drops has ok=0
 * and an empty row. The result stays on the device until ts_rows_copy. */
int ts_rays_trace(ts_ctx* ctx, const ts_grid* fwd, int32_t n_tables, const float* tables, const double* table_station,
                  const ts_grid* inv, int32_t n_rays, const int32_t* table_of, const double* events, double step_km,
                  ts_rows** out);

/* Which kernel traces a call's rays (no counterpart in the reference, whose Backtrack runs one ray
 * per CPU thread, RayKernels.cs:67-107): a call of at most max_rays rays is traced with one warp
 * per ray, whose lanes share each step's corner loads and gradient evaluations (the latency of a
 * small call, such as a serving completion's, is its longest ray's); a larger call with one thread
 * per ray. Both give the same rows to the bit. Default 2048 (one warp per ray is the faster below about
 * 2,500 rays of a 121×121×61 model, a thread per ray above); 0 always uses a thread per ray. */
int ts_rays_set_warp_max(ts_ctx* ctx, int32_t max_rays);

/* RayKernels.Compute for travel times (Tomography/RayKernels.cs:30-115) with the tables built on
 * the device: one field per (station, phase) used, by the engine (precision as ts_eik_solve), each
 * seeded by PointSource at the station and rounded to float32 as TravelTimeTable.Write does, then
 * every arrival traced on its table. slowness: n_phases fields on fwd (ForwardModel, phase p at
 * p*n). stations/events: 3 doubles each. Arrival a: (arr_event[a], arr_station[a], arr_phase[a]).
 * mode: TS_MODE_FAST (the recommended default: fields within 1e-10 relative of the reference's, about
 * half the work) or TS_MODE_ENGINE (the reference's fields to the bit). step_km <= 0 uses the
 * RayKernels step. */
int ts_forward(ts_ctx* ctx, const ts_grid* fwd, const double* slowness, int32_t n_phases, const ts_grid* inv,
               int32_t n_stations, const double* stations, int32_t n_events, const double* events,
               int32_t n_arrivals, const int32_t* arr_event, const int32_t* arr_station, const int32_t* arr_phase,
               int32_t precision, int32_t mode, double step_km, ts_rows** out, ts_eik_stats* stats);

/* ---- LSQR on the device (Numerics/Lsqr.cs:33-152, LsqrOpenCl.cs) ----
 * Damped LSQR, min ‖A x − b‖² + damp² ‖x‖², with the reference's stopping rules (atol, btol,
 * conlim, iteration budget). stop: 0 empty system, 1 zero right-hand side, 2 Aᵀb = 0, 3 iteration
 * budget, 4 btol, 5 atol, 6 conlim, 7–9 machine precision (residual, normal equations, condition),
 * 10 bidiagonalisation terminated. The solve repeats to the bit on a given device and agrees with
 * the sequential host solver to rounding. */
typedef struct ts_lsqr_info {
    int32_t iterations, stop;
    double bnorm, rnorm, acond;   /* ‖b‖, ‖r‖ of the damped system, condition estimate */
    double device_ms;             /* the iteration loop */
} ts_lsqr_info;
/* A as host CSR (row_ptr[m+1], col, val), b[m] on the host; x_out[n]. */
int ts_lsqr_solve(ts_ctx* ctx, int32_t m, int32_t n, const int32_t* row_ptr, const int32_t* col, const double* val,
                  const double* b, double damp, int32_t max_iterations, double atol, double btol, double conlim,
                  double* x_out, ts_lsqr_info* info);
/* A = the rows of a ray result (ts_forward / ts_rays_trace) as they lie on the device, n columns
 * (the inversion grid's nodes); rows the reference drops are empty and their b entries should be 0. */
int ts_lsqr_solve_rows(ts_ctx* ctx, ts_rows* rows, int32_t n, const double* b, double damp, int32_t max_iterations,
                       double atol, double btol, double conlim, double* x_out, ts_lsqr_info* info);
/* The rows' transpose is built on the device in CsrMatrix.Transpose's order (SparseMatrix.cs:79-96);
 * a column index not below n is refused with TS_E_ARG. */

/* Lsqr.Solve's onIteration (Lsqr.cs:43,140; LsqrOpenCl.TrySolve's, LsqrOpenCl.cs:250-256): fn is called
 * on the calling thread after every iteration with the iteration number (from 1) and ‖r‖ of the damped
 * system. NULL removes it. */
typedef void (*ts_lsqr_iteration_fn)(int32_t iteration, double rnorm, void* user);
int ts_lsqr_set_callback(ts_ctx* ctx, ts_lsqr_iteration_fn fn, void* user);
/* LsqrOpenCl.SelfTest (LsqrOpenCl.cs:541-557): a random 3000 x 1200 damped system with 12 non-zeros per
 * row solved on the device and by the sequential host solver (damp 0.05, 300 iterations, atol = btol =
 * 1e-12, conlim 1e10); *rel_err = max |dx| / max |x_host|. TS_OK when <= 1e-8 (SelfTestTolerance, :33),
 * otherwise TS_E_SELFTEST. */
int ts_lsqr_selftest(ts_ctx* ctx, double* rel_err, char* msg, int32_t cap);

/* ---- Forward domain and model (Forward/ForwardDomain.cs:24-137, Forward/TravelTimeTable.cs:213-241) ---- */
/* VelocityModel1D's nodes (Model/VelocityModel1D.cs:8-45): n depths (non-decreasing; a repeated depth is
 * a discontinuity) with Vp and Vs, km/s; piecewise linear, the first node's value above it. */
typedef struct ts_background {
    int32_t n, reserved;
    const double* depth_km;
    const double* vp;
    const double* vs;
} ts_background;
/* ForwardDomain.Covering (:51-107) on the host: the inversion grid refined `refinement` times, or,
 * when some of the points (lon, lat, depth per point) lie outside the inversion grid, the grid that
 * holds them with a margin of two cells, coarsened by 1.25 steps until it has at most max_nodes
 * nodes (<= 0: 12,000,000). *extended: 1 when it reaches beyond the inversion grid; *coarsening: the
 * spacing factor applied. Errors as text in ts_last_error(NULL). */
int ts_domain_covering(const ts_grid* inversion, int32_t refinement, int32_t n_points, const double* points,
                       int64_t max_nodes, ts_grid* out, int32_t* extended, double* coarsening);
/* ForwardModel.FromInversionGrid (TravelTimeTable.cs:217-241) on the device, into a resident model on
 * `forward` (as ts_model_put makes): per phase (1: P, 2: P and S) the inversion grid's velocity
 * 1/inv_slowness interpolated at every forward node (SphericalGrid.ResampleFrom, :241-252), the
 * background's Vp or Vs where a node lies outside the inversion grid (bg non-NULL: the extended
 * domain), then slowness = 1/v. Bitwise the reference's arithmetic. */
int ts_model_put_resampled(ts_ctx* ctx, const ts_grid* forward, const ts_grid* inversion, const double* inv_slowness,
                           int32_t n_phases, const ts_background* bg, int32_t precision, int32_t* model_id);
/* The extended domain's background for the rays (RayKernels.Compute with domain.Extended,
 * RayKernels.cs:63-65): from this call on, ts_forward and the other ray calls integrate only the
 * pieces inside the inversion grid (tolerance 1e-6) and sum the others' length times 1/Vp or 1/Vs of
 * the background (the arrival's phase; ts_rays_trace: Vp) into the row's outside time
 * (RayTracing.Kernel, RayTracing.cs:126-159). NULL or n = 0 restores the plain domain. */
int ts_set_background(ts_ctx* ctx, const ts_background* bg);
/* A resident model's slowness of one phase to the host (grid-count doubles). */
int ts_model_copy_slowness(ts_ctx* ctx, int32_t model_id, int32_t phase, double* out);

/* ---- Travel-time tables kept on the device (TravelTimeTableSet, Forward/TravelTimeTable.cs:247-412) ----
 * n_tables float32 fields on one uniform grid, node-major per table as a .qttb file holds them. A table
 * set belongs to the context that made it: free it (ts_tables_free) before ts_cuda_destroy. */
typedef struct ts_tables ts_tables;
/* TravelTimeTableSet.Build (:264-308): table t is the field of the source sources[3t..3t+2] (lon, lat,
 * depth km; seeds by PointSource, :373) for the slowness of phase source_phase[t] (slowness holds
 * n_phases fields on grid), solved by the engine (bitwise the reference's sweeping) and rounded to
 * float32 (TravelTimeTable.Write, :73). */
int ts_tables_build(ts_ctx* ctx, const ts_grid* grid, const double* slowness, int32_t n_phases, int32_t n_tables,
                    const double* sources, const int32_t* source_phase, int32_t precision, ts_tables** out,
                    ts_eik_stats* stats);
/* Tables from the host (e.g. .qttb files read by TravelTimeTable.Open, :99-111). */
int ts_tables_upload(ts_ctx* ctx, const ts_grid* grid, int32_t n_tables, const float* tables, ts_tables** out);
int ts_tables_info(ts_tables* tables, int32_t* n_tables, int64_t* nodes_per_table);
/* Tables first .. first+count-1 to the host (count * nodes floats). */
int ts_tables_copy(ts_tables* tables, int32_t first, int32_t count, float* out);
void ts_tables_free(ts_tables* tables);
/* TravelTimeTable.Write (Forward/TravelTimeTable.cs:57-80) for tables first .. first+count-1: file k
 * at paths[k] holds the magic "QTTB" 01 00 00 00, header_len[k] as a little-endian int32, the
 * header bytes headers[k] (the caller's TravelTimeTableHeader serialised with TomoJson.Options,
 * Model/Basics.cs:60-75), zero bytes up to a multiple of 64, then the table as little-endian float32
 * with every non-finite value written as +inf; written to path + ".tmp" and renamed over path. */
int ts_tables_write_qttb(ts_tables* tables, int32_t first, int32_t count, const char* const* paths,
                         const char* const* headers, const int32_t* header_len);
/* TravelTimeTable.Open (:99-111) of count files into a resident table set on `grid` (the grid their
 * headers name): the magic is checked and each file must hold the grid's nodes after its header. */
int ts_tables_load_qttb(ts_ctx* ctx, const ts_grid* grid, int32_t count, const char* const* paths, ts_tables** out);

/* ---- Event location on resident tables (Location/EventLocator.cs:59-342, Relocation.cs:48-97) ---- */
typedef struct ts_locator_settings {   /* LocatorSettings (EventLocator.cs:10-36); defaults in brackets */
    int32_t global_search;             /* [1] whole grid on a stride lattice first; 0: within 6 nodes of the start */
    int32_t coarse_candidates;         /* [8000] */
    int32_t max_geiger_iterations;     /* [20] */
    int32_t min_phases;                /* [4] */
    double damping;                    /* [0.01] Levenberg-Marquardt damping relative to the diagonal */
    double outlier_mads;               /* [4] */
    double outlier_floor;              /* [0.5] s */
    int32_t fix_depth;                 /* [0] */
    int32_t reserved;
} ts_locator_settings;
typedef struct ts_location {           /* LocationResult + Hypocentre (EventLocator.cs:38, Model/Catalogue.cs:92-114) */
    double t0;                         /* origin time, s after the event's reference time */
    double lon, lat, depth_km;
    double rms;                        /* s */
    double err_h_km, err_minor_km, err_azimuth_deg, err_depth_km, err_time_s;  /* NaN: singular covariance */
    double gap_deg;                    /* azimuthal gap of the stations in use */
    int32_t used, rejected, iterations;
    int32_t status;                    /* 0 ok; 1 fewer than min_phases observations; 2 local search box outside the grid */
} ts_location;
typedef struct ts_locate_stats {
    double device_ms;                  /* the whole call on the device */
    int64_t candidates;                /* grid-search nodes evaluated */
    int32_t rounds, reserved;          /* location rounds run (outlier rejection relocates) */
} ts_locate_stats;
/* EventLocator.Locate for n_events events. Event e's observations are obs_offsets[e] ..
 * obs_offsets[e+1]-1 (at most 1024): obs_table (its station's table for its phase), obs_seconds (the
 * pick time in s after the event's reference time), obs_weight, obs_correction (the station
 * correction). start: lon, lat, depth per event (the catalogue location). table_station: lon, lat of
 * each table's station (the gap). residual_out[q]: every pick's residual at the solution (rejected
 * picks included; NaN for an event not located). Not located (status != 0): the start is returned. */
int ts_locate(ts_ctx* ctx, ts_tables* tables, const ts_locator_settings* settings, int32_t n_events,
              const double* start, const int32_t* obs_offsets, const int32_t* obs_table, const double* obs_seconds,
              const double* obs_weight, const double* obs_correction, const double* table_station, ts_location* out,
              double* residual_out, ts_locate_stats* stats);

/* Sizes of a result: rows (= rays or arrivals) and total non-zeros. */
int ts_rows_info(ts_rows* rows, int32_t* n_rows, int64_t* nnz);
/* Copies a result to the host: row_ptr[n_rows+1], col[nnz] (int32 node), len[nnz] (float32 km),
 * tcalc_grad[4*n_rows] (TCalc s, Ge, Gn, Gz s/km), ok[n_rows]. Any pointer may be NULL. */
int ts_rows_copy(ts_rows* rows, int32_t* row_ptr, int32_t* col, float* len, double* tcalc_grad, uint8_t* ok);
/* RayRow.OutsideTime (Tomography/RayKernels.cs:15-19, 95) of every row: the time spent outside the
 * inversion grid in the background set by ts_set_background (0 without one); n_rows doubles. */
int ts_rows_outside(ts_rows* rows, double* outside);
void ts_rows_free(ts_rows* rows);

#ifdef __cplusplus
}
#endif

#endif /* TOMOSTAR_CUDA_H */
