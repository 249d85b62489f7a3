// kmy_server.cu -- serving loop: many independent solves, continuously batched.
//
// Requests (a deck, a problem generator and a step count) queue on the host.
// Each tick the server admits queued requests while their device footprint
// fits the HBM budget (first fit over the queue), creates their device state
// (a fused-path kmy_ctx on the server's stream) and adds them to the batch of
// their kernel class (precision, dimensionality, reconstruction, Riemann
// solver, stage count).  Then every batch advances all its solves by one RK
// step: one persistent launch per stage over the batch's (solve, block, brick)
// work list, then one controller launch that moves each solve's clock.  A
// solve leaves its batch when it reaches its step count; its state stays on
// the device until the caller exports and releases it.  The work list, its
// length and each solve's clock live in device memory, so a batch's launches
// are captured once in a CUDA graph and replayed whatever the membership.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/kmy_hydro.h"
#include "kmy_batch.cuh"

namespace kmy {

int batch_stage_f64(cudaStream_t, int, int, int, const void *, const long long *, const int *, int, int *);
int batch_stage_f32(cudaStream_t, int, int, int, const void *, const long long *, const int *, int, int *);
int batch_controller_f64(cudaStream_t, void *, const int *, int, BatchStatus *);
int batch_controller_f32(cudaStream_t, void *, const int *, int, BatchStatus *);

struct Request {
  int64_t id = 0;
  std::string deck, problem;
  int nsteps = 0;
  Footprint fp{};
  kmy_ctx *ctx = nullptr;
  double t_submit = 0, t_admit = -1, t_done = -1;
  int state = 0;  // 0 queued, 1 active, 2 finished, 3 failed
  int status = 0;
  bool first = true;
  int batch = -1;
};

struct Batch {
  int esz, ndim, recon, riemann, nstages;
  std::vector<Request *> members;
  bool dirty = true;
  int capacity = 0;
  cudaStream_t stream = nullptr;  // one stream per class: classes overlap on the GPU
  void *d_desc = nullptr;
  long long *d_prefix = nullptr;
  int *d_n = nullptr;
  BatchStatus *d_status = nullptr;
  BatchStatus *h_status = nullptr;  // pinned
  int grid = 0;
  cudaGraphExec_t graph = nullptr;
  bool key_match(const Footprint &f) const {
    return esz == f.esz && ndim == f.ndim && recon == f.recon && riemann == f.riemann &&
           nstages == f.nstages;
  }
};

}  // namespace kmy

struct kmy_server {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool graphs = true;
  size_t budget = 0, used = 0;
  int64_t next_id = 1;
  std::deque<kmy::Request *> queue;
  std::map<int64_t, std::unique_ptr<kmy::Request>> reqs;
  std::vector<std::unique_ptr<kmy::Batch>> batches;
  std::vector<kmy::Request *> finished;  // not yet polled
  std::chrono::steady_clock::time_point t0;
  int64_t ticks = 0, launches = 0, finished_total = 0;
  double cell_updates = 0.0;
  std::string err;
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

using namespace kmy;

static int srv_fail(kmy_server *s, int code, const std::string &msg) {
  s->err = msg;
  return code;
}

static void free_batch_buffers(Batch &b) {
  if (b.graph) cudaGraphExecDestroy(b.graph);
  if (b.d_desc) cudaFree(b.d_desc);
  if (b.d_prefix) cudaFree(b.d_prefix);
  if (b.d_n) cudaFree(b.d_n);
  if (b.d_status) cudaFree(b.d_status);
  if (b.h_status) cudaFreeHost(b.h_status);
  b.graph = nullptr;
  b.d_desc = nullptr;
  b.d_prefix = nullptr;
  b.capacity = 0;
  b.d_n = nullptr;
  b.d_status = nullptr;
  b.h_status = nullptr;
}

template <typename S>
static void fill_desc(kmy_ctx *c, const Request &r, SolveDesc<S> &q) {
  std::memset(&q, 0, sizeof(q));
  q.m = c->m;
  q.eos = c->eos;
  q.tp = c->prm.tp;
  q.limiter = c->prm.limiter;
  q.nstages = int(c->prm.beta.size());
  q.nlim = r.nsteps;
  q.stored = r.first ? 1 : 0;
  for (int s = 0; s < q.nstages && s < 3; s++) {
    Container &ct = c->md[c->prm.stage_name[s]];
    q.cont[s] = static_cast<S *>(ct.cc);
    q.lo[s] = static_cast<float *>(ct.ener_lo);
    q.beta[s] = c->prm.beta[s];
  }
  q.prim = static_cast<const S *>(c->prim);
  q.clock = c->clock;
  const int B3[3] = {c->m.ndim == 3 ? 8 : c->m.ndim == 2 ? 16 : 128,
                     c->m.ndim == 3 ? 8 : c->m.ndim == 2 ? 16 : 1, c->m.ndim == 3 ? 8 : 1};
  for (int d = 0; d < 3; d++) q.nbr[d] = (c->m.nx[d] + B3[d] - 1) / B3[d];
}

// Upload a batch's work list (descriptors, offsets, count) after a membership change.
static int upload(kmy_server *s, Batch &b) {
  const int n = int(b.members.size());
  const size_t dsz = b.esz == 8 ? sizeof(SolveDesc<double>) : sizeof(SolveDesc<float>);
  if (n > b.capacity) {
    free_batch_buffers(b);
    b.capacity = std::max(64, 2 * n);
    if (cudaMalloc(&b.d_desc, dsz * b.capacity) != cudaSuccess ||
        cudaMalloc((void **)&b.d_prefix, sizeof(long long) * (b.capacity + 1)) != cudaSuccess ||
        cudaMalloc((void **)&b.d_n, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void **)&b.d_status, sizeof(BatchStatus) * b.capacity) != cudaSuccess ||
        cudaMallocHost((void **)&b.h_status, sizeof(BatchStatus) * b.capacity) != cudaSuccess) {
      cudaGetLastError();
      return srv_fail(s, KMY_ERR_OOM, "batch work-list allocation failed");
    }
  }
  std::vector<unsigned char> desc(dsz * std::max(n, 1));
  std::vector<long long> prefix(n + 1, 0);
  for (int i = 0; i < n; i++) {
    Request *r = b.members[i];
    kmy_ctx *c = r->ctx;
    long long nbrick;
    if (b.esz == 8) {
      SolveDesc<double> *q = reinterpret_cast<SolveDesc<double> *>(desc.data()) + i;
      fill_desc(c, *r, *q);
      nbrick = (long long)q->nbr[0] * q->nbr[1] * q->nbr[2];
    } else {
      SolveDesc<float> *q = reinterpret_cast<SolveDesc<float> *>(desc.data()) + i;
      fill_desc(c, *r, *q);
      nbrick = (long long)q->nbr[0] * q->nbr[1] * q->nbr[2];
    }
    prefix[i + 1] = prefix[i] + nbrick * c->m.nb;
  }
  cudaError_t e = cudaMemcpyAsync(b.d_desc, desc.data(), dsz * n, cudaMemcpyHostToDevice, b.stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b.d_prefix, prefix.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice,
                        b.stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b.d_n, &n, sizeof(int), cudaMemcpyHostToDevice, b.stream);
  // the host vectors are released on return: finish the copies first
  if (e == cudaSuccess) e = cudaStreamSynchronize(b.stream);
  if (e != cudaSuccess) return srv_fail(s, KMY_ERR_CUDA, cudaGetErrorString(e));
  b.dirty = false;
  return KMY_OK;
}

// One RK step of every solve in the batch: ns stage launches + the controller.
static int launch_step(kmy_server *s, Batch &b) {
  int rc = 0;
  for (int st = 1; st <= b.nstages && !rc; st++) {
    rc = b.esz == 8 ? batch_stage_f64(b.stream, b.ndim, b.recon, b.riemann, b.d_desc, b.d_prefix, b.d_n,
                                      st, &b.grid)
                    : batch_stage_f32(b.stream, b.ndim, b.recon, b.riemann, b.d_desc, b.d_prefix, b.d_n,
                                      st, &b.grid);
  }
  if (!rc)
    rc = b.esz == 8 ? batch_controller_f64(b.stream, b.d_desc, b.d_n, b.capacity, b.d_status)
                    : batch_controller_f32(b.stream, b.d_desc, b.d_n, b.capacity, b.d_status);
  return rc ? srv_fail(s, KMY_ERR_CUDA, "batched stage launch failed") : KMY_OK;
}

static int run_batch(kmy_server *s, Batch &b) {
  if (b.dirty) {
    // a capacity change reallocates the work list and drops the graph
    int rc = upload(s, b);
    if (rc) return rc;
  }
  if (!s->graphs) {
    s->launches += b.nstages + 1;
    return launch_step(s, b);
  }
  if (!b.graph) {
    // occupancy query and smem attributes must happen outside capture
    if (b.grid <= 0) {
      int rc = launch_step(s, b);  // first step runs directly and sizes the grid
      s->launches += b.nstages + 1;
      return rc;
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal);
    int rc = e == cudaSuccess ? launch_step(s, b) : KMY_ERR_CUDA;
    e = cudaStreamEndCapture(b.stream, &g);
    if (rc || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return srv_fail(s, KMY_ERR_CUDA, "graph capture failed");
    }
    e = cudaGraphInstantiate(&b.graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return srv_fail(s, KMY_ERR_CUDA, "graph instantiation failed");
  }
  s->launches += b.nstages + 1;
  const cudaError_t e = cudaGraphLaunch(b.graph, b.stream);
  return e == cudaSuccess ? KMY_OK : srv_fail(s, KMY_ERR_CUDA, cudaGetErrorString(e));
}

static int admit(kmy_server *s) {
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    Request *r = *it;
    if (s->used + r->fp.bytes > s->budget) {
      ++it;  // first fit: a smaller request behind may still fit
      continue;
    }
    kmy_ctx *c = nullptr;
    int rc = kmy_create(r->deck.c_str(), s->device, &c);
    if (!rc) rc = kmy_set_stream(c, s->stream);
    if (!rc) rc = kmy_pgen(c, r->problem.c_str());
    if (rc) {
      if (c) kmy_destroy(c);
      if (rc == KMY_ERR_OOM) return KMY_OK;  // fragmentation: retry on a later tick
      r->state = 3;
      r->status = rc;
      r->t_done = s->now();
      s->finished.push_back(r);
      it = s->queue.erase(it);
      continue;
    }
    r->ctx = c;
    r->state = 1;
    r->t_admit = s->now();
    s->used += r->fp.bytes;
    int bi = -1;
    for (size_t k = 0; k < s->batches.size(); k++)
      if (s->batches[k]->key_match(r->fp)) bi = int(k);
    if (bi < 0) {
      auto b = std::make_unique<Batch>();
      b->esz = r->fp.esz;
      b->ndim = r->fp.ndim;
      b->recon = r->fp.recon;
      b->riemann = r->fp.riemann;
      b->nstages = r->fp.nstages;
      if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return srv_fail(s, KMY_ERR_CUDA, "stream creation failed");
      s->batches.push_back(std::move(b));
      bi = int(s->batches.size()) - 1;
    }
    r->batch = bi;
    s->batches[bi]->members.push_back(r);
    s->batches[bi]->dirty = true;
    it = s->queue.erase(it);
  }
  return KMY_OK;
}

extern "C" {

int kmy_server_create(int device, double hbm_fraction, int use_graphs, kmy_server **out) {
  if (!out || !(hbm_fraction > 0.0) || hbm_fraction > 1.0) return KMY_ERR_BAD_PARAM;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return KMY_ERR_CUDA;
  auto *s = new kmy_server();
  s->device = device;
  s->graphs = use_graphs != 0;
  s->t0 = std::chrono::steady_clock::now();
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    return KMY_ERR_CUDA;
  }
  s->budget = size_t(double(fr) * hbm_fraction);
  *out = s;
  return KMY_OK;
}

int kmy_server_destroy(kmy_server *s) {
  if (!s) return KMY_OK;
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->stream);
  for (auto &kv : s->reqs)
    if (kv.second->ctx) kmy_destroy(kv.second->ctx);
  for (auto &b : s->batches) {
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_batch_buffers(*b);
    if (b->stream) cudaStreamDestroy(b->stream);
  }
  cudaStreamDestroy(s->stream);
  delete s;
  return KMY_OK;
}

const char *kmy_server_last_error(const kmy_server *s) { return s ? s->err.c_str() : "null server"; }

int kmy_server_submit(kmy_server *s, const char *deck, const char *problem, int nsteps, int64_t *id) {
  if (!s || !deck || !problem || nsteps < 1) return KMY_ERR_BAD_PARAM;
  auto r = std::make_unique<Request>();
  std::string err;
  int rc = deck_footprint(deck, &r->fp, &err);
  if (rc) return srv_fail(s, rc, err);
  if (r->fp.mhd) return srv_fail(s, KMY_ERR_BAD_PARAM, "the serving loop batches hydro solves only");
  if (r->fp.nstages < 2)
    return srv_fail(s, KMY_ERR_BAD_PARAM, "the serving loop needs a two- or three-stage integrator");
  if (r->fp.bytes > s->budget) return srv_fail(s, KMY_ERR_OOM, "request larger than the HBM budget");
  r->id = s->next_id++;
  r->deck = deck;
  r->problem = problem;
  r->nsteps = nsteps;
  r->t_submit = s->now();
  if (id) *id = r->id;
  s->queue.push_back(r.get());
  s->reqs[r->id] = std::move(r);
  return KMY_OK;
}

int kmy_server_tick(kmy_server *s, int *nactive, int *nqueued) {
  if (!s) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(s->device);
  int rc = admit(s);
  if (rc) return rc;
  bool any = false;
  for (auto &b : s->batches) {
    if (b->members.empty()) continue;
    rc = run_batch(s, *b);
    if (rc) return rc;
    cudaMemcpyAsync(b->h_status, b->d_status, sizeof(BatchStatus) * b->members.size(),
                    cudaMemcpyDeviceToHost, b->stream);
    any = true;
  }
  if (any) {
    for (auto &b : s->batches) {
      if (b->members.empty()) continue;
      const cudaError_t e = cudaStreamSynchronize(b->stream);
      if (e != cudaSuccess) return srv_fail(s, KMY_ERR_CUDA, cudaGetErrorString(e));
    }
    s->ticks++;
  }
  const double t = s->now();
  int active = 0;
  for (auto &b : s->batches) {
    if (b->members.empty()) continue;
    std::vector<Request *> keep;
    for (size_t i = 0; i < b->members.size(); i++) {
      Request *r = b->members[i];
      const BatchStatus &st = b->h_status[i];
      if (r->first) {
        r->first = false;  // the controller cleared the device copy of the flag
        b->dirty = true;   // re-upload so the host copy agrees
      }
      s->cell_updates += double(r->fp.cells);
      if (st.done || st.status) {
        // the batched stages advanced the conserved state only: export must
        // rebuild primitives and ghost zones
        r->ctx->prims_valid = false;
        r->state = st.status ? 3 : 2;
        r->status = st.status;
        r->t_done = t;
        s->finished.push_back(r);
        s->finished_total++;
        b->dirty = true;
      } else {
        keep.push_back(r);
      }
    }
    b->members.swap(keep);
    active += int(b->members.size());
  }
  if (nactive) *nactive = active;
  if (nqueued) *nqueued = int(s->queue.size());
  return KMY_OK;
}

int kmy_server_poll(kmy_server *s, int64_t *ids, double *seconds, int *status, int max, int *n) {
  if (!s || !n) return KMY_ERR_BAD_PARAM;
  int k = 0;
  while (k < max && !s->finished.empty()) {
    Request *r = s->finished.front();
    s->finished.erase(s->finished.begin());
    if (ids) ids[k] = r->id;
    if (seconds) seconds[k] = r->t_done - r->t_submit;
    if (status) status[k] = r->status;
    k++;
  }
  *n = k;
  return KMY_OK;
}

int kmy_server_export(kmy_server *s, int64_t id, const char *var, int comp, double *host, size_t n) {
  if (!s) return KMY_ERR_BAD_PARAM;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end() || !it->second->ctx) return srv_fail(s, KMY_ERR_BAD_PARAM, "unknown request");
  if (it->second->state == 1) return srv_fail(s, KMY_ERR_STATE, "request still running");
  const int rc = kmy_export_var(it->second->ctx, "base", var, comp, host, n);
  if (rc) s->err = kmy_last_error(it->second->ctx);
  return rc;
}

int kmy_server_release(kmy_server *s, int64_t id) {
  if (!s) return KMY_ERR_BAD_PARAM;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return srv_fail(s, KMY_ERR_BAD_PARAM, "unknown request");
  Request *r = it->second.get();
  if (r->state == 1 || r->state == 0) return srv_fail(s, KMY_ERR_STATE, "request not finished");
  if (r->ctx) {
    kmy_destroy(r->ctx);
    r->ctx = nullptr;
    s->used -= r->fp.bytes;
  }
  s->reqs.erase(it);
  return KMY_OK;
}

int kmy_server_stats(const kmy_server *s, double *out) {
  if (!s || !out) return KMY_ERR_BAD_PARAM;
  int active = 0;
  for (auto &b : s->batches) active += int(b->members.size());
  out[0] = double(active);
  out[1] = double(s->queue.size());
  out[2] = double(s->finished_total);
  out[3] = double(s->used);
  out[4] = double(s->budget);
  out[5] = double(s->ticks);
  out[6] = s->cell_updates;
  out[7] = double(s->launches);
  return KMY_OK;
}

}  // extern "C"
