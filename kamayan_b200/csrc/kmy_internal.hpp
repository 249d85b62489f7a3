// kmy_internal.hpp -- host-side context, mesh description and kernel entry
// points shared by the translation units of libkmy_hydro.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "kmy_device.cuh"

namespace kmy {

// Uniform single-level mesh, passed by value to every kernel.  Block b sits at
// logical location (b % nbx0, (b / nbx0) % nbx1, b / (nbx0 nbx1)); arrays are
// Parthenon MeshData layout: [var][block][k][j][i] over the ghost-padded block.
struct MeshDesc {
  int ndim;
  int nb;
  int nx[3];       // interior cells per block
  int g[3];        // ghosts per dim (0 if inactive)
  int np[3];       // padded cells per dim
  int nf[3];       // padded face dims (np + 1 in active dims)
  int nbx[3];      // blocks per dim
  int mesh_nx[3];  // cells across the mesh
  int bc[3][2];    // BoundaryKind per dim and side
  long long P;     // padded cells per block
  long long Pf;    // padded faces per block (one element)
  double dx[3];
  double xmin[3];
  // cartesian geometry (Parthenon UniformCartesian products)
  double area[3];  // dy*dz, dx*dz, dx*dy
  double vol;      // dx*dy*dz
  // adaptive mesh: per-block level and logical location, and per level a
  // table of (leaf id | -1 covered by finer | -2 covered by coarser) over the
  // level's block positions.  All null / zero on a single-level mesh, where
  // block b sits at lexicographic location b at level 0.
  const int *blev;
  const int *bloc;
  const int *tabs;
  int nlev;
  int tab_off[8];
  int tab_dim[8][3];
};

__host__ __device__ __forceinline__ int blk_level(const MeshDesc &m, int b) { return m.blev ? m.blev[b] : 0; }
__host__ __device__ __forceinline__ int blk_loc(const MeshDesc &m, int b, int d) {
  if (m.bloc) return m.bloc[3 * b + d];
  if (d == 0) return b % m.nbx[0];
  if (d == 1) return (b / m.nbx[0]) % m.nbx[1];
  return b / (m.nbx[0] * m.nbx[1]);
}
// cell size of block b (only active dimensions refine)
__host__ __device__ __forceinline__ double blk_dx(const MeshDesc &m, int b, int d) {
  return d < m.ndim ? m.dx[d] / double(1 << blk_level(m, b)) : m.dx[d];
}
__host__ __device__ __forceinline__ double blk_area(const MeshDesc &m, int b, int d) {
  if (!m.blev) return m.area[d];
  if (d == 0) return blk_dx(m, b, 1) * blk_dx(m, b, 2);
  if (d == 1) return blk_dx(m, b, 0) * blk_dx(m, b, 2);
  return blk_dx(m, b, 0) * blk_dx(m, b, 1);
}
__host__ __device__ __forceinline__ double blk_vol(const MeshDesc &m, int b) {
  if (!m.blev) return m.vol;
  return blk_dx(m, b, 0) * blk_dx(m, b, 1) * blk_dx(m, b, 2);
}

// Device-resident simulation clock.  The dt controller runs on the device so
// that a whole step (all stages + controller) needs no host round trip.
struct DevClock {
  double time;
  double dt;        // dt of the next step
  double dt_est;    // last CFL estimate (already times cfl/ndim)
  double dt_taken;  // dt of the last completed step
  unsigned long long dtmin_bits;  // atomic min of dx/(|v|+c) (bit pattern of a positive double)
  int ncycle;
  int done;         // time >= tlim: stage kernels become no-ops
  int status;       // KMY_ERR_NONFINITE when the estimate was not finite/positive,
                    // KMY_ERR_DT_RANGE when dt left [dt_min, dt_max] too long,
                    // KMY_ERR_TIMEOUT when a stage kernel's bounded wait gave up
  unsigned long long zone_cycles;  // interior cells x completed steps, summed over the steps
  int below_min;    // consecutive cycles with dt < dt_min
  int above_max;    // consecutive cycles with dt > dt_max
};

struct TimeParams {
  double tlim, dt_factor, dt_init, dt_ceil, dt_user, dt_floor;
  double cfl_over_ndim;
  // Parthenon's dt sanity limits: a dt below dt_min for dt_min_cycle_limit
  // cycles (or above dt_max for dt_max_cycle_limit) ends the run
  double dt_min, dt_max;
  int nlim;
  int dt_min_cycle_limit, dt_max_cycle_limit;
};

// Parthenon EvolutionDriver time update + SetGlobalTimeStep after a step,
// restated: time += dt, then dt <- min(dt * dt_factor, CFL estimate, ceilings),
// clamped so the run ends exactly at tlim.  The estimate is the atomic minimum
// of dx/(|v|+c_f) left by the last stage.
__device__ __forceinline__ void advance_clock(DevClock *clk, const TimeParams &tp) {
  const double dtmin = __longlong_as_double((long long)clk->dtmin_bits);
  const double big = 1.7976931348623157e308;
  clk->dt_taken = clk->dt;
  clk->time += clk->dt;
  clk->ncycle += 1;
  const double est = dtmin * tp.cfl_over_ndim;
  clk->dt_est = est;
  // the first failure stays: a stage that stopped early (a wait that ran
  // out) leaves no estimate, which is not the cause to report
  if (clk->status == 0 && (!(est > 0.0) || !(est < big))) clk->status = 3;  // KMY_ERR_NONFINITE
  double nd = clk->dt;
  if (nd < 0.1 * big) nd *= tp.dt_factor;
  nd = fmin(nd, est);
  nd = fmin(nd, tp.dt_ceil);
  nd = fmin(nd, tp.dt_user);
  if (clk->time < tp.tlim && (tp.tlim - clk->time) < nd) nd = tp.tlim - clk->time;
  clk->dt = nd;
  clk->done = clk->time >= tp.tlim;
  // the dt sanity limits (the reference's parthenon/time dt_min, dt_max and
  // their cycle limits, src/driver/kamayan_driver.cpp:43-54): the step that
  // was just taken counts
  clk->below_min = clk->dt_taken < tp.dt_min ? clk->below_min + 1 : 0;
  clk->above_max = clk->dt_taken > tp.dt_max ? clk->above_max + 1 : 0;
  if (clk->status == 0 && (clk->below_min >= tp.dt_min_cycle_limit || clk->above_max >= tp.dt_max_cycle_limit))
    clk->status = 7;  // KMY_ERR_DT_RANGE
}

struct Params {
  int recon = FOG, limiter = MINMOD, riemann = HLL;
  bool mhd = false;
  double cfl = 0.8, gamma = 5.0 / 3.0, Abar = 1.0;
  std::vector<double> beta;
  std::vector<std::string> stage_name;
  int precision = 64;
  // fused hydro stage kernel: 0 auto (the z-streamed stage where it applies),
  // 1 brick stage, 2 z-streamed stage (error where it does not apply),
  // 3 tune (the autotuner's cached or measured choice, kmy_tune.cu)
  int stage_kernel = 0;
  // rows per tile of the z-streamed stage: 0 auto, 8 or 16
  int slab_rows = 0;
  // hydro brick stage launched once per meshblock instead of once per mesh
  // (<kamayan_b200> launch = per_block; the plain per-block GPU baseline)
  bool per_block = false;
  // face update of a constrained-transport stage (<kamayan_b200> ct_update):
  // 0 auto (streamed where it applies), 1 streamed (kmy_ct.cu), 2 one kernel
  // per face direction plus the primitive pass (kmy_tasks.cu)
  int ct_update = 0;
  TimeParams tp{};
  std::map<std::string, std::string> deck;
  double real(const std::string &k, double d) const;
  int integer(const std::string &k, int d) const;
  std::string str(const std::string &k, const std::string &d) const;
};

struct Container {
  void *cc = nullptr;     // [ncc][nb][P] of S
  void *ener_lo = nullptr;// [nb][P] float low word of E (FP32 path only)
  void *fc = nullptr;     // [3][nb][Pf] face "mag" (CT only)
  void *emf = nullptr;    // [3][nb][Pf] edge EMFs (CT only)
  // the face ghosts of the conserved state hold their owners' values (set by
  // a ghost fill or a z-streamed stage that wrote this container, cleared by
  // every other writer); the z-streamed stage stages its input through them
  bool ghosts = false;
  // the arrays are the caller's (kmy_bind_container): never freed or moved
  bool bound = false;
};

// Host side of an adaptive mesh: the leaf list and the refinement parameters.
struct AmrCriterion {
  std::string field = "dens";
  double refine_tol = 0.8, derefine_tol = 0.2, filter = 0.01;
  int max_level = 0;
};
struct AmrHost {
  bool on = false;
  int numlevel = 1, max_level = 0, derefine_count = 10;  // max_level = numlevel - 1
  std::vector<AmrCriterion> crits;  // one per <kamayan/refinementN> block with a field
  std::vector<int> lev;  // per leaf
  std::vector<int> loc;  // 3 per leaf
  std::vector<int> cnt;  // consecutive derefine tags per leaf
  bool balanced = false;  // the leaf list is known to be 2:1 balanced
  int *d_blev = nullptr, *d_bloc = nullptr, *d_tabs = nullptr, *d_tags = nullptr;
  int *d_err = nullptr;  // set by a level-value recursion that ran out of depth
  void *d_emf_tmp = nullptr;  // EMFs as computed, read by the edge correction
  // ghost cells whose position is not a leaf at their level, with the cells
  // their restriction or prolongation reads (rebuilt at every table upload)
  // (entries [0, plan_n) are read directly, the next plan_deep evaluated
  // recursively, the last plan_inner are inner entries whose values the
  // direct ones read from d_plan_scr, [variable][plan_inner] doubles)
  void *d_plan = nullptr;
  int *d_plan_n = nullptr;  // four counters: direct, recursive, inner, copies
  double *d_plan_scr = nullptr;
  int plan_n = 0, plan_deep = 0, plan_inner = 0;
  // ghost cells whose same-level position holds a leaf, with that leaf cell
  void *d_copy = nullptr;
  int copy_n = 0;
  // coarse boundary faces whose neighbour is finer, with the fine faces their
  // flux is restricted from
  void *d_fix = nullptr;
  int fix_n = 0;
  int64_t gen = 0;  // table uploads so far (a captured step is only valid for one)
  size_t emf_tmp_bytes = 0;
};

}  // namespace kmy

struct kmy_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  kmy::Params prm;
  kmy::MeshDesc m{};
  kmy::EosParams eos{};
  int ncc = 5;
  size_t esz = 8;  // bytes per stored real
  std::map<std::string, kmy::Container> md;
  void *prim = nullptr;   // [NPRIM][nb][P] shared primitives (S)
  // Fused path: the stage reads the primitives of its input from `prim` and
  // writes those of its output to `prim_alt`; the two swap after the stage.
  void *prim_alt = nullptr;
  bool prims_interior = false;  // `prim` holds the interior primitives of "base" (ghosts stale)
  bool prims_imported = false;  // a primitive was imported since the last finalize
  bool prim_bound = false;      // `prim` is the caller's (kmy_bind_primitives): never swapped or freed
  void *flux = nullptr;   // [3][ncc][nb][Pf] face fluxes (S), shared by all containers
  double *divb = nullptr; // [nb][P]
  kmy::DevClock *clock = nullptr;  // device
  double *scratch = nullptr;       // reduction scratch (device)
  bool prims_valid = false;  // stored prims match "base" (after pgen/import/tasks)
  int path = 0;              // 0 fused, 1 tasks
  kmy::AmrHost amr;          // adaptive mesh (task path only)
  int64_t launches = 0;
  // kmy_evolve's chunk of fused steps as a CUDA graph, and the host-side
  // state it was captured from (kmy_api.cu:graph_run)
  cudaGraphExec_t evolve_exec = nullptr;
  std::string evolve_key, evolve_seen;
  int64_t evolve_launches = 0;
  int64_t graph_replays = 0;  // launches of a cached graph (kmy_graph_replays)
  // kmy_evolve's device time: events around each iteration's queued steps
  cudaEvent_t ev_evolve[2] = {nullptr, nullptr};
  double evolve_device_ms = 0.0;
  // kmy_evolve on an adaptive mesh queues the next step before it reads the
  // tags of the current one (kmy_api.cu:evolve_amr): the base state before
  // that speculative step is kept here (conserved, energy low words, faces,
  // primitives, div B, clock; sized for bak_cells padded cells per array),
  // and each step in flight has a pinned slot for its tags and clock and a
  // pair of timing events
  void *bak_cc = nullptr, *bak_lo = nullptr, *bak_fc = nullptr, *bak_prim = nullptr, *bak_divb = nullptr,
       *bak_clock = nullptr;
  size_t bak_cells = 0;
  char *pipe_pin[2] = {nullptr, nullptr};
  size_t pipe_pin_bytes = 0;
  cudaEvent_t pipe_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int fault_wait = 0;  // kmy_set_fault "stage_wait": the next z-streamed stage's waits run out
  // pinned host staging for the per-step reads (clock, tags), grown on demand
  void *h_pin = nullptr;
  size_t h_pin_bytes = 0;
  // the clock as an adaptive step's tag read brought it back, valid while no
  // kernel has been launched since (launches == clock_host_launches)
  kmy::DevClock clock_host{};
  int64_t clock_host_launches = -1;
  std::string err;
  std::string deck_text;  // the deck the context was created from (restart files carry it)
  std::vector<void *> allocations;
};

namespace kmy {

// ---- kernels (kmy_tasks.cu) ----
int launch_fill_ghosts(kmy_ctx *c, Container &ct);
// Pinned host staging of at least `bytes` (kmy_api.cu); valid until the next
// call, so every user synchronizes before it returns.
void *host_pin(kmy_ctx *c, size_t bytes);
int launch_compute_fluxes(kmy_ctx *c, Container &md0);
int launch_compute_emf(kmy_ctx *c, Container &md0);
int launch_flux_divergence(kmy_ctx *c, Container &md0, Container &dudt);
// Flux divergence and the cell update in one pass (adaptive hydro meshes).
int launch_div_apply(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta, double dt,
                     const double *dt_dev);
int launch_apply_dudt(kmy_ctx *c, Container &base, Container &md0, Container &md1,
                      Container &dudt, double beta, double dt, const double *dt_dev);
// constrained-transport pieces of a stage that the fused stage leaves to
// separate kernels
int ensure_flux(kmy_ctx *c);
const char *fused_ct_unsupported(const kmy_ctx *c);  // kmy_fused.cu
int launch_flux_halo(kmy_ctx *c);
int launch_flux_stokes(kmy_ctx *c, Container &md0, Container &dudt);
int launch_apply_faces(kmy_ctx *c, Container &base, Container &md0, Container &md1, Container &dudt,
                       double beta, double dt, const double *dt_dev);
int launch_ct_faces(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta);
int launch_prepare_primitive(kmy_ctx *c, Container &md1);
int launch_estimate_dt(kmy_ctx *c, Container &md, bool reset);
int launch_fill_derived(kmy_ctx *c, Container &md);
int launch_eos_init(kmy_ctx *c, Container &md);
int launch_convert_to_conserved(kmy_ctx *c, Container &md);
// mode 0: after a step; 1: initial dt from the estimate; 2: clamp pending dt to tlim
// cells: interior cells of the step the controller completes (mode 0); -1
// takes the current mesh's.
int launch_dt_controller(kmy_ctx *c, int mode, long long cells = -1);
int launch_conserved_sums(kmy_ctx *c, Container &md, double *host_out);
int launch_vortex_error(kmy_ctx *c, int var, int comp, double *host_out);
int launch_set_energy_split(kmy_ctx *c, Container &ct);
// ---- fused stage (kmy_fused.cu) ----
int launch_fused_stage(kmy_ctx *c, Container &base, Container &md0, Container &md1,
                       double beta, bool stored_prims, bool last);
// ---- z-streamed 3D stage (kmy_slab_host.cu; kernels in kmy_slab_f32.cu, kmy_slab_f64.cu) ----
// Why the z-streamed stage cannot run this context, or null.
const char *slab_unsupported(const kmy_ctx *c);
// Rows per tile the z-streamed stage uses for this context (8 or 16).
int slab_rows(const kmy_ctx *c);
int launch_slab_stage(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta, bool last);
// Whether the fused stage runs the z-streamed kernel (it applies, the deck
// allows it, and in auto mode the mesh has enough work items), and whether a
// constrained-transport stage runs its cells through it.
bool slab_runs(const kmy_ctx *c);
bool ct_cells_on_slab(const kmy_ctx *c);
// ---- streamed constrained-transport face update (kmy_ct.cu) ----
// Why the streamed face update cannot run this context, or null.
const char *ct_stream_unsupported(const kmy_ctx *c);
// Edge EMFs, Stokes sums and face update of md1, then the cell-centred field
// and primitives of md1; with fold_last also the CFL estimate into the clock
// and div B of md1 (the last stage, md1 being "base").
int launch_ct_stream(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta, bool fold_last);
// ---- stage-kernel autotuner (kmy_tune.cu) ----
std::string tune_config_key(const kmy_ctx *c);
int tune_apply(kmy_ctx *c, const std::string &choice);
int tune_run(kmy_ctx *c, int reps, std::vector<std::pair<std::string, double>> *results);
bool tune_lookup(kmy_ctx *c);
// Parse and validate a deck into a context that owns no device resources.
int parse_deck(kmy_ctx *tmp, const char *deck);
// ---- problem generators (kmy_pgen.cu) ----
int launch_pgen(kmy_ctx *c, const std::string &problem);

int cuda_check(kmy_ctx *c, cudaError_t e, const char *what);
// Zeroed device allocation from the stream-ordered pool, freed with the context.
int dalloc(kmy_ctx *c, void **p, size_t bytes);
// Return one allocation of the context to the pool before the context ends.
void dfree(kmy_ctx *c, void *p);
int make_container(kmy_ctx *c, const std::string &name);

// ---- adaptive mesh (kmy_amr.cu) ----
int amr_setup(kmy_ctx *c);
int amr_upload(kmy_ctx *c);
int launch_amr_fill_ghosts(kmy_ctx *c, Container &ct);
int launch_flux_correct(kmy_ctx *c);
int launch_emf_correct(kmy_ctx *c, Container &md0);
int launch_amr_tag(kmy_ctx *c, Container &ct);
// The tree update from the last tags; with clock_out, the device clock comes
// back in the same read (one host sync).
int amr_remesh(kmy_ctx *c, bool allow_derefine, bool *changed, DevClock *clock_out = nullptr);
// The two halves of amr_remesh on tags already read back: the derefinement
// counters and whether anything is due (call once per step's tags), then the
// tree update and remap.
int amr_count_tags(kmy_ctx *c, const std::vector<int> &tags, int err, bool *any);
// before_change runs once the new tree is known to differ, before any device
// work.
int amr_remesh_apply(kmy_ctx *c, bool allow_derefine, const std::vector<int> &tags, bool *changed,
                     const std::function<int()> &before_change = nullptr);
// Storage for the leaf list already in c->amr (lev, loc, cnt): level tables,
// every stage container, the primitives and div B at the new block count.
int amr_adopt_leaves(kmy_ctx *c);

// Device footprint and kernel class of a deck (kmy_api.cu), for admission.
struct Footprint {
  size_t bytes;
  int esz, ndim, recon, riemann, nstages, mhd;
  long long cells;
};
int deck_footprint(const char *deck, Footprint *out, std::string *err);

}  // namespace kmy
