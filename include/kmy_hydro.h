/* kmy_hydro.h -- C ABI of the B200 finite-volume update (kamayan hydro path).
 *
 * Plain C types only: no CUDA, torch or C++ types cross this boundary.  Every
 * entry point returns a kmy_status code; no C++ exception escapes.  A context
 * owns one mesh, its device-resident stage containers and one CUDA stream; it
 * is not thread-safe (use one context per host thread).
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the kamayan source tree).
 */
#ifndef KMY_HYDRO_H_
#define KMY_HYDRO_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* TaskStatus / PARTHENON_FAIL analogue (driver/kamayan_driver_types.hpp:19-20). */
typedef enum {
  KMY_OK = 0,
  KMY_ERR_BAD_PARAM = 1, /* unknown option, bad size or name */
  KMY_ERR_OOM = 2,       /* device allocation failed */
  KMY_ERR_NONFINITE = 3, /* NaN/inf or non-positive density/pressure detected */
  KMY_ERR_TIMEOUT = 4,   /* a bounded device wait gave up */
  KMY_ERR_CUDA = 5,      /* CUDA runtime error (see kmy_last_error) */
  KMY_ERR_STATE = 6,     /* call out of order (e.g. no state yet) */
  KMY_ERR_DT_RANGE = 7   /* dt below dt_min for dt_min_cycle_limit cycles, or above dt_max for
                            dt_max_cycle_limit (Parthenon's fatal, kamayan_driver.cpp:43-54) */
} kmy_status;

typedef struct kmy_ctx kmy_ctx;

/* Mesh description returned by kmy_get_info.  Arrays are (i, j, k) ordered. */
typedef struct {
  int ndim;
  int nblocks;
  int nx[3];        /* interior cells per meshblock */
  int nghost;       /* ghost cells in each active dimension */
  int ncells_pad[3];/* ghost-padded cells per block: nx + 2*nghost (1 if inactive) */
  int nfaces_pad[3];/* face array dims: ncells_pad + 1 in active dims */
  int nblocks_dim[3];
  int ncons;        /* cell conserved components: 5 hydro, 8 with CT */
  int mhd;          /* 0 off, 1 constrained transport */
  int nstages;      /* RK stages of the integrator */
  int precision;    /* 64 or 32: arithmetic/storage type of the bulk update */
  double xmin[3], xmax[3], dx[3];
} kmy_info;

/* Create a context from a Parthenon input deck (`<block>` headers with
 * `key = value` lines, and `block/key = value` override lines).  Accepted keys
 * mirror the reference's runtime parameters: <parthenon/mesh> (nx*, x*min/max,
 * *_bc, nghost), <parthenon/meshblock> (nx*), <parthenon/time> (integrator,
 * tlim, nlim, dt_*), <hydro> (reconstruction, slope_limiter, riemann, cfl,
 * ReconstructionVars, ReconstructionStrategy, EMF_averaging), <physics> (MHD),
 * <material/single> (gamma, Abar, eos_type), <eos> (mode_init), plus
 * <kamayan_b200> (precision = fp64|fp32; stage_kernel = auto|brick|slab|tune;
 * slab_rows = auto|8|16; launch = batched|per_block; ct_update =
 * auto|streamed|per_face).  Unknown option values
 * fail with KMY_ERR_BAD_PARAM.
 * Adaptive meshes (hydro and CT): <parthenon/mesh> refinement = adaptive, numlevel
 * (<= 8), derefine_count, and <kamayan/refinement0>, <kamayan/refinement1>, ...
 * blocks, each with field (dens|pres|ener), method = loehner, refine_tol,
 * derefine_tol, filter, max_level (src/grid/grid.cpp:43-48, :90-124;
 * src/grid/grid_refinement.cpp:15-30).  Blocks then carry a level and a logical
 * location (kmy_get_blocks) and the block count changes as the mesh adapts; the
 * step runs the per-task kernels with flux (and, with CT, EMF) correction,
 * Loehner tagging and a remesh after each step.
 * Replaces: InitEnv/InitPackages parameter setup (src/kamayan/kamayan.cpp:20-138),
 * hydro::SetupParams (src/physics/hydro/hydro.cpp:51-92),
 * grid::SetupParams (src/grid/grid.cpp:29-122),
 * driver::SetupParams (src/driver/kamayan_driver.cpp:23-81). */
int kmy_create(const char *deck, int device, kmy_ctx **out);
int kmy_destroy(kmy_ctx *ctx);
/* Message of the last failing call on this context ("" if none). */
const char *kmy_last_error(const kmy_ctx *ctx);
int kmy_get_info(const kmy_ctx *ctx, kmy_info *out);

/* Bind the context to a caller-owned cudaStream_t (NULL = context's own). */
int kmy_set_stream(kmy_ctx *ctx, void *cuda_stream);
/* Block until all work queued on the context's stream is finished. */
int kmy_sync(kmy_ctx *ctx);

/* ---- state in Parthenon MeshData layout -------------------------------------
 * Cell variables: n = nblocks * prod(ncells_pad) doubles, block-major then
 * (k, j, i) with i fastest.  Face variable "mag": comp = face direction, n =
 * nblocks * prod(nfaces_pad).  Names are the reference field names
 * (src/kamayan/fields.hpp:177-210): "dens", "momentum"(3), "ener", "magc"(3),
 * "mag"(face, 3), "velocity"(3), "pres", "bulk modulus", "eint", "temp",
 * "divb".  Containers: "base", the stage names "1", "2", ... and "dUdt"
 * (src/driver/kamayan_driver.cpp:140-143).  Primitives are shared by all
 * containers.  Export fills ghost zones first (boundary exchange semantics). */
int kmy_import_var(kmy_ctx *ctx, const char *container, const char *var, int comp,
                   const double *host, size_t n);
int kmy_export_var(kmy_ctx *ctx, const char *container, const char *var, int comp,
                   double *host, size_t n);
/* Interior cells only: n = nblocks * nx[0]*nx[1]*nx[2] doubles, block-major
 * then (k, j, i) with i fastest and no ghost zones -- the layout of the
 * Parthenon phdf outputs the reference's regression baselines compare
 * (python/kamayan/testing/baselines.py:300).  Cell variables only.  An import
 * leaves the ghost zones to kmy_finalize_import; moving interior cells moves
 * 40 % fewer bytes than the padded arrays on 32^3 blocks with 3 ghosts. */
int kmy_import_interior(kmy_ctx *ctx, const char *container, const char *var, int comp,
                        const double *host, size_t n);
int kmy_export_interior(kmy_ctx *ctx, const char *container, const char *var, int comp,
                        double *host, size_t n);
/* In-place state on caller-owned device memory.  The reference's slots read
 * and write the MeshData they are given (src/kamayan/unit.hpp:56-76,
 * src/grid/grid.hpp:133-135); kmy_bind_container makes a caller's device
 * arrays the storage of a named container, so every slot above and below
 * (kmy_compute_fluxes, kmy_flux_divergence, kmy_apply_dudt, kmy_task_stage,
 * kmy_rk_stage, kmy_step, ...) works on them directly, with no copies.
 *   cons:    [ncons][nblocks][ncells_pad] of the context's precision (double, or
 *            float with fp32), i fastest: each conserved component a contiguous
 *            nblocks x prod(ncells_pad) array, components in the order dens,
 *            momentum 0-2, ener (, magc 0-2); cons_bytes its size
 *   ener_lo: fp32 only (else NULL/0): [nblocks][ncells_pad] floats, the low word
 *            of the total energy (E = ener + ener_lo); zeros for an FP32 energy
 *   mag:     CT only (else NULL/0): [3][nblocks][nfaces_pad] face field
 * Arrays start on 16-byte boundaries.  The caller keeps them alive until
 * kmy_destroy; the context's own arrays for the container are released.
 * After writing bound arrays from outside, call kmy_finalize_import (ghosts,
 * primitives, dt).  Single-level meshes only (an adaptive mesh reallocates its
 * containers as it remeshes).  kmy_bind_primitives does the same for the
 * primitives shared by all containers, [7][nblocks][ncells_pad] in the order
 * velocity 0-2, pres, bulk modulus, eint, temp. */
int kmy_bind_container(kmy_ctx *ctx, const char *container, void *cons, size_t cons_bytes,
                       void *ener_lo, size_t ener_lo_bytes, void *mag, size_t mag_bytes);
int kmy_bind_primitives(kmy_ctx *ctx, void *prim, size_t bytes);
/* Mark imported state complete: prims of "base" are taken as given (as after
 * the reference's MeshPostInitialization) or, when no primitive variable was
 * imported since the last finalize, derived from the conserved state
 * (PreparePrimitive); ghosts are filled, dt is estimated.
 * Replaces: the driver initialisation path (EstimateTimestep after pgen). */
int kmy_finalize_import(kmy_ctx *ctx);

/* Device problem generators: "isentropic_vortex", "kelvin_helmholtz",
 * "orszag_tang", "blast", "sedov".  Problem parameters come from the deck.
 * Replaces: ProblemGenerator + MeshPostInitialization
 * (src/problems/isentropic_vortex.cpp:105-175, src/problems/sedov.cpp:104-143,
 *  src/physics/hydro/primconsflux.cpp:145-148, src/physics/material_properties/eos/eos.cpp:165-168). */
int kmy_pgen(kmy_ctx *ctx, const char *problem);

/* ---- per-task entry points (KamayanUnit callback slots) -------------------- */
/* hydro::AddFluxTasks -> CalculateFluxes (src/physics/hydro/hydro_add_flux_tasks.cpp:36-264) */
int kmy_compute_fluxes(kmy_ctx *ctx, const char *md0);
/* hydro::AddFluxTasks -> CalculateEMF (src/physics/hydro/hydro_add_flux_tasks.cpp:405-442) */
int kmy_compute_emf(kmy_ctx *ctx, const char *md0);
/* grid::FluxesToDuDt (src/grid/grid.cpp:208-211; src/grid/grid_update.hpp:15-137) */
int kmy_flux_divergence(kmy_ctx *ctx, const char *md0, const char *dudt);
/* grid::ApplyDuDt (src/grid/grid.cpp:213-283) */
int kmy_apply_dudt(kmy_ctx *ctx, const char *base, const char *md0, const char *md1,
                   const char *dudt, double beta, double dt);
/* hydro::PreparePrimitive + eos::PreparePrimitive (src/physics/hydro/primconsflux.cpp:152-155,
 * src/physics/material_properties/eos/eos.cpp:164) */
int kmy_prepare_primitive(kmy_ctx *ctx, const char *md1);
/* Parthenon AddBoundaryExchangeTasks on one level (kamayan_driver.cpp:150-151) */
int kmy_fill_ghosts(kmy_ctx *ctx, const char *md);
/* hydro::EstimateTimeStepMesh (src/physics/hydro/hydro_time_step.cpp:67-70) */
int kmy_estimate_dt(kmy_ctx *ctx, const char *md, double *dt_out);
/* hydro::FillDerived, div B (src/physics/hydro/hydro.cpp:191-194) */
int kmy_fill_derived(kmy_ctx *ctx, const char *md);
/* One RK stage through the per-task kernels above, in the reference task order
 * (KamayanDriver::BuildTaskListRKStage, src/driver/kamayan_driver.cpp:186-248). */
int kmy_task_stage(kmy_ctx *ctx, int stage, double dt);

/* ---- fused path -----------------------------------------------------------
 * One RK stage in a single fused launch (reconstruction, Riemann flux, flux
 * divergence and the low-storage update; dt estimate fused into the last
 * stage).  Same results as kmy_task_stage within FP64 rounding. */
int kmy_rk_stage(kmy_ctx *ctx, int stage, double dt);
/* One time step at the current dt (all stages) followed by the dt controller
 * (Parthenon EvolutionDriver semantics).  dt_taken may be NULL. */
int kmy_step(kmy_ctx *ctx, double *dt_taken);
/* Step until tlim or nlim steps (nlim < 0: no limit). */
int kmy_evolve(kmy_ctx *ctx, double tlim, int nlim, int *nsteps);
/* Close a step driven stage by stage with kmy_rk_stage: advance the clock by
 * the step's dt and choose the next dt on the device, without a host round
 * trip.  Replaces: Parthenon EvolutionDriver time update + SetGlobalTimeStep
 * after the stage task collections (src/driver/kamayan_driver.cpp:121-155). */
int kmy_end_step(kmy_ctx *ctx);
/* Simulation clock: time, next dt, last dt estimate, cycle count. */
int kmy_get_time(const kmy_ctx *ctx, double *time, double *dt, double *dt_est, int *ncycle);
/* Zone-cycles since set-up: the interior cells of each completed step's mesh
 * (before its remesh), summed over the steps.  Divided by wall time it is the
 * zone-cycles/wall_second figure the reference's driver prints every
 * ncycle_out cycles (src/driver/kamayan_driver.cpp:63-78). */
int kmy_zone_cycles(const kmy_ctx *ctx, int64_t *out);
/* Leaf blocks in block order: refinement level (levels[b]) and logical
 * location at that level (locations[3b..3b+2], i j k).  Fills at most
 * max_blocks entries; *nblocks receives the block count.  Single-level meshes
 * report level 0 and the lexicographic location.
 * Replaces: Parthenon MeshBlock::loc / LogicalLocation of each block of the
 * MeshData (used by the refinement tasks, src/grid/grid_refinement.cpp:30-152). */
int kmy_get_blocks(const kmy_ctx *ctx, int *levels, int *locations, int max_blocks, int *nblocks);

/* ---- restart files ----------------------------------------------------------
 * kmy_save_restart writes the context's state to `path`: the deck, the "base"
 * container as stored, the shared primitives, the face field and div B with
 * CT, the device clock and time limits, and the leaf list of an adaptive
 * mesh.  kmy_load_restart creates a new context on `device` from such a file;
 * it continues exactly as the saved context would have (same bits).  Files
 * are for the same build of the library (native byte order, raw arrays).
 * Replaces: Parthenon restart outputs (<parthenon/output*> file_type = rst,
 * src/problems/isentropic_vortex.in:40-43, variables flagged Metadata::Restart
 * in src/kamayan/fields.hpp:160-161) and the driver's restart path (-r). */
int kmy_save_restart(kmy_ctx *ctx, const char *path);
int kmy_load_restart(const char *path, int device, kmy_ctx **out);
/* Override the dt used by the next kmy_step (e.g. to replay a reference run). */
int kmy_set_dt(kmy_ctx *ctx, double dt);
/* Select the stepping path used by kmy_step/kmy_evolve: 0 = fused, 1 = tasks. */
int kmy_set_path(kmy_ctx *ctx, int path);

/* ---- diagnostics ----------------------------------------------------------- */
/* L1 error of dens/velocity/pres/magc against the initial isentropic vortex
 * (src/problems/isentropic_vortex.hpp:150-200).  var: 0 dens, 1 velocity,
 * 2 pres, 3 magc (CT only). */
int kmy_vortex_error(kmy_ctx *ctx, int var, int comp, double *out);
/* Compensated (Kahan-Babuska) FP64 sums of the conserved variables over the
 * interior of `md` times the cell volume: out[0..ncons-1]. */
int kmy_conserved_sums(kmy_ctx *ctx, const char *md, double *out);

/* Face values (vM at i-1/2, vP at i+1/2) of n five-cell stencils (stencils[5i
 * .. 5i+4] = cells i-2 .. i+2) from the library's device reconstruction
 * functions: out[3i] = vM, out[3i+1] = vP, out[3i+2] = 1 when the two lanes of
 * a packed FP32 form disagreed (else 0).  impl selects the form each stage
 * kernel uses: 0 FP64 per-task kernels, 1 FP64 brick and batched stages
 * (two-division WENO-Z, Newton-Raphson reciprocals), 2 FP32 per lane,
 * 3 FP32 brick stage (packed), 4 FP32 z-streamed stage (packed), 5 FP64
 * z-streamed stage (lane by lane, WENO-Z dividing by Newton-Raphson
 * reciprocals); impl 6 returns the FP64 stages' Newton-Raphson reciprocal
 * of stencils[5i] in out[3i] and square root of stencils[5i+1] in
 * out[3i+1].  Needs no context; runs on the current device and
 * synchronises it.  Counterpart of the reference's device-side Reconstruct
 * (src/physics/hydro/reconstruction.hpp:11-142) as its unit tests call it
 * (src/physics/hydro/tests/test_reconstruction.cpp:13-194). */
int kmy_reconstruct_stencils(const char *reconstruction, const char *slope_limiter, int impl,
                             const double *stencils, int n, double *out);

/* Number of this library's kernels launched on the context since creation. */
int kmy_launch_count(const kmy_ctx *ctx, int64_t *out);
/* Failure-path test hook.  what = "stage_wait", value = 1: the next
 * z-streamed stage's staged-pair barrier expects more bytes than its tensor
 * loads deliver and its bounded wait is shortened, so the wait runs out; the
 * stage stops, sets the device clock's status, and the step returns
 * KMY_ERR_TIMEOUT.  Nothing faults or hangs; the CUDA context stays usable.
 * No counterpart in the reference. */
int kmy_set_fault(kmy_ctx *ctx, const char *what, int value);
/* Number of kmy_evolve chunks (or adaptive steps) that replayed a cached CUDA
 * graph instead of launching their kernels one by one. */
int kmy_graph_replays(const kmy_ctx *ctx, int64_t *out);
/* Device time (ms) of the last kmy_evolve call: from before each group of
 * queued steps to after their last kernel, summed; the host's read-backs and
 * tree updates between groups are not counted, so wall time over this is the
 * host's share of the loop. */
int kmy_evolve_device_ms(const kmy_ctx *ctx, double *ms);

/* ---- stage-kernel autotuner -------------------------------------------------
 * The reference chooses its flux loop strategy by a runtime parameter
 * (<hydro> ReconstructionStrategy, src/physics/hydro/hydro.cpp:75-79).  Here
 * the stage kernel is chosen by measurement: "brick" (brick-tiled fused
 * stage), "slab16" / "slab8" (z-streamed 3D stage with TMA-staged plane
 * pairs, tiles of 16 or 8 rows; FP64 runs 8 only).  kmy_autotune times every candidate that
 * applies to the context on its current state (stage 1 into a scratch
 * container, so the solve does not advance), applies the fastest and caches
 * it under (device name, configuration key).  The deck option
 * <kamayan_b200> stage_kernel = tune does the same at the first stage (from
 * the cache when it holds the key).  results[i]: candidate name, mean stage
 * time in ms, and whether it applies (ms < 0 when it does not). */
typedef struct {
  char name[16];
  double ms;
  int applies;
} kmy_tune_result;
int kmy_autotune(kmy_ctx *ctx, int reps, kmy_tune_result *results, int max_results, int *n_results);
/* The stage kernel the context's next fused stage runs: "brick", "slab16",
 * "slab8", "tune" (not yet chosen) or "tasks". */
int kmy_stage_kernel(const kmy_ctx *ctx, char *name, size_t n);
/* Configuration part of the tuner's cache key for a deck (host only: parses
 * the deck, needs no GPU).  The cache key is "<device name> | <this>". */
int kmy_tune_key(const char *deck, char *buf, size_t n);
/* The process-wide tuning cache: put/get one entry (choice must be a
 * candidate name), clear, and save to / load from a text file with one
 * "key<TAB>choice<TAB>ms" line per entry (malformed lines are skipped).
 * kmy_tune_cache_get returns KMY_ERR_STATE when the key is absent. */
int kmy_tune_cache_put(const char *key, const char *choice, double ms);
int kmy_tune_cache_get(const char *key, char *choice, size_t n, double *ms);
int kmy_tune_cache_clear(void);
int kmy_tune_cache_save(const char *path);
int kmy_tune_cache_load(const char *path);

/* ---- serving loop: continuously batched independent solves ----------------
 * No counterpart in the reference (which runs one mesh per process).  A
 * server owns one CUDA stream and an HBM budget (a fraction of the free
 * device memory at creation).  Requests are a deck, a problem generator and a
 * step count; kmy_server_tick admits queued requests whose footprint fits the
 * budget, then advances every admitted solve by one RK step with one
 * persistent launch per stage per kernel class (precision, dimensionality,
 * reconstruction, Riemann solver), replayed from a CUDA graph.  Hydro decks
 * with rk2/rk3 only.  Times are host seconds. */
typedef struct kmy_server kmy_server;
int kmy_server_create(int device, double hbm_fraction, int use_graphs, kmy_server **out);
int kmy_server_destroy(kmy_server *srv);
const char *kmy_server_last_error(const kmy_server *srv);
int kmy_server_submit(kmy_server *srv, const char *deck, const char *problem, int nsteps,
                      int64_t *id);
/* Admit, step every active solve once, retire finished ones. */
int kmy_server_tick(kmy_server *srv, int *nactive, int *nqueued);
/* Finished requests since the last poll: id, time-to-solution (submit to
 * completion), status (KMY_OK or the failure code). */
int kmy_server_poll(kmy_server *srv, int64_t *ids, double *seconds, int *status, int max, int *n);
/* Final state of a finished request (MeshData layout, like kmy_export_var). */
int kmy_server_export(kmy_server *srv, int64_t id, const char *var, int comp, double *host,
                      size_t n);
/* Free a finished request's device state. */
int kmy_server_release(kmy_server *srv, int64_t id);
/* out[0..7]: active, queued, finished, bytes in use, byte budget, ticks,
 * cell updates done, kernel launches. */
int kmy_server_stats(const kmy_server *srv, double *out);

/* Compensated FP64 sums of conserved variables for callers that cannot
 * allocate device memory (a framework that owns all device memory through its
 * own pool, or code where an allocation is not allowed or would synchronise
 * the device).  No counterpart in the reference.  Needs no context and calls
 * no cudaMalloc/cudaFree: its scratch is a static device array of fixed size
 * held by every GPU that loads the library.
 *   cons:   device pointer, [ncons][nblocks][ncells_pad] doubles (MeshData layout)
 *   out_dev: device pointer to ncons doubles, out_dev[v] = sum over interior
 *           cells of cons[v] * cell_volume
 *   stream: cudaStream_t to launch on (NULL = default stream)
 * ncons above 8 (the scratch array's capacity) returns KMY_ERR_BAD_PARAM.
 * The first call in a CUDA context looks up the scratch array's device
 * address in that context (the address is valid for that context only; a
 * device reset starts a new context, whose first call looks it up again);
 * make that first call before any stream capture.  Calls
 * share the scratch array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int kmy_conserved_sums_noalloc(const double *cons, int ncons, int nblocks,
                               const int ncells_pad[3], const int nx[3], const int nghost[3],
                               double cell_volume, double *out_dev, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* KMY_HYDRO_H_ */
