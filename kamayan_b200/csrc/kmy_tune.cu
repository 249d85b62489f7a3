// kmy_tune.cu -- autotuner of the hydro stage kernel.
//
// The reference picks its flux loop strategy as a runtime parameter
// (<hydro> ReconstructionStrategy, src/physics/hydro/hydro.cpp:75-79).  Here
// the choice that matters for speed is how a stage stages and tiles its
// cells, and it is measured rather than configured:
//
//   brick   -- the brick-tiled fused stage (8^3 / 16^2 / 128 bricks, halos
//              read from neighbouring interiors through address tables);
//   slab16  -- the z-streamed 3D stage, TMA-staged plane pairs, tiles of
//              16 rows (FP32: one 512-thread CTA per SM);
//   slab8   -- the same with tiles of 8 rows (FP32: two 256-thread CTAs per
//              SM; FP64, whose plan does not fit 16 rows: one).
//
// A tuning run times every candidate that applies to the context, on its own
// state: stage 1 (beta = 1) reads "base" and writes a scratch container, so
// the solve does not advance.  The fastest candidate is applied and cached
// under (device name, configuration key), for the process and, through
// kmy_tune_cache_save / _load, across processes.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>

#include "../../include/kmy_hydro.h"
#include "kmy_internal.hpp"

namespace kmy {

namespace {

struct Cand {
  const char *name;
  int kernel;  // Params::stage_kernel: 1 brick, 2 z-streamed
  int rows;    // Params::slab_rows
};
constexpr Cand kCands[] = {{"brick", 1, 0}, {"slab16", 2, 16}, {"slab8", 2, 8}};

const Cand *find_cand(const std::string &name) {
  for (const auto &c : kCands)
    if (name == c.name) return &c;
  return nullptr;
}

struct Entry {
  std::string choice;
  double ms;
};
std::mutex g_mu;
std::map<std::string, Entry> g_cache;

const char *recon_name(int r) { return r == FOG ? "fog" : r == PLM ? "plm" : r == PPM ? "ppm" : "wenoz"; }
const char *limiter_name(int l) { return l == MINMOD ? "minmod" : l == VAN_LEER ? "van_leer" : "mc"; }

std::string device_name(int device) {
  cudaDeviceProp p{};
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) {
    cudaGetLastError();
    return "device" + std::to_string(device);
  }
  return p.name;
}

}  // namespace

// Configuration part of a cache key: everything the stage kernels' speed
// depends on (precision, dimensionality, method, block shape, block count).
std::string tune_config_key(const kmy_ctx *c) {
  const MeshDesc &m = c->m;
  std::ostringstream o;
  o << (c->esz == 4 ? "fp32" : "fp64") << " d" << m.ndim << " " << recon_name(c->prm.recon) << "-"
    << (c->prm.riemann == HLL ? "hll" : "hllc") << "-" << limiter_name(c->prm.limiter) << (c->prm.mhd ? " ct" : "")
    << " n" << m.nx[0] << "x" << m.nx[1] << "x" << m.nx[2] << " g" << m.g[0] << " b" << m.nb;
  return o.str();
}

int tune_apply(kmy_ctx *c, const std::string &choice) {
  const Cand *k = find_cand(choice);
  if (!k) {
    c->err = "unknown stage kernel " + choice;
    return KMY_ERR_BAD_PARAM;
  }
  c->prm.stage_kernel = k->kernel;
  c->prm.slab_rows = k->rows;
  return KMY_OK;
}

// Time every candidate stage kernel on the context's state; apply and cache
// the fastest.  results: (name, ms per stage, applies).
int tune_run(kmy_ctx *c, int reps, std::vector<std::pair<std::string, double>> *results) {
  if (c->prm.mhd || c->amr.on) {
    // constrained transport takes the z-streamed stage where it runs (FP32,
    // enough blocks) and the brick stage elsewhere, without tuning; adaptive
    // meshes run the per-task kernels
    if (results) results->push_back({"brick", -1.0});
    return tune_apply(c, "brick");
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(c->stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
    c->err = "the stage kernel cannot be tuned inside a stream capture";
    return KMY_ERR_STATE;
  }
  reps = std::max(1, std::min(reps, 50));
  const int saved_kernel = c->prm.stage_kernel, saved_rows = c->prm.slab_rows;
  if (!c->md.count("tune") && make_container(c, "tune")) return KMY_ERR_OOM;
  if (c->esz == 4 && !c->prim_alt && dalloc(c, &c->prim_alt, c->esz * NPRIM * size_t(c->m.nb) * c->m.P))
    return KMY_ERR_OOM;
  Container &base = c->md["base"], &out = c->md["tune"];
  const bool stored = c->prims_valid || c->prims_interior;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = cuda_check(c, cudaEventCreate(&e0), "tune event");
  if (!rc) rc = cuda_check(c, cudaEventCreate(&e1), "tune event");
  std::string best;
  double best_ms = 1e300;
  for (const auto &k : kCands) {
    if (rc) break;
    c->prm.stage_kernel = k.kernel;
    c->prm.slab_rows = k.rows;
    if (k.kernel == 2 && slab_unsupported(c)) {
      if (results) results->push_back({k.name, -1.0});
      continue;
    }
    auto launch = [&]() {
      return k.kernel == 2 ? launch_slab_stage(c, base, base, out, 1.0, false)
                           : launch_fused_stage(c, base, base, out, 1.0, stored, false);
    };
    rc = launch();  // warm-up (first-use attributes, caches)
    if (!rc) rc = cuda_check(c, cudaEventRecord(e0, c->stream), "tune record");
    for (int r = 0; r < reps && !rc; r++) rc = launch();
    if (!rc) rc = cuda_check(c, cudaEventRecord(e1, c->stream), "tune record");
    if (!rc) rc = cuda_check(c, cudaEventSynchronize(e1), "tune sync");
    float ms = 0.f;
    if (!rc) rc = cuda_check(c, cudaEventElapsedTime(&ms, e0, e1), "tune elapsed");
    if (rc) break;
    const double per = double(ms) / reps;
    if (results) results->push_back({k.name, per});
    if (per < best_ms) {
      best_ms = per;
      best = k.name;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  // the scratch container goes back to the pool
  dfree(c, out.cc);
  dfree(c, out.ener_lo);
  c->md.erase("tune");
  c->prm.stage_kernel = saved_kernel;
  c->prm.slab_rows = saved_rows;
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache[device_name(c->device) + " | " + tune_config_key(c)] = Entry{best, best_ms};
  }
  return tune_apply(c, best);
}

// The cached choice for this context, if any (applied when found).
bool tune_lookup(kmy_ctx *c) {
  const std::string key = device_name(c->device) + " | " + tune_config_key(c);
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cache.find(key);
  if (it == g_cache.end()) return false;
  return tune_apply(c, it->second.choice) == KMY_OK;
}

}  // namespace kmy

using namespace kmy;

extern "C" {

int kmy_tune_key(const char *deck, char *buf, size_t n) {
  if (!deck || !buf || n == 0) return KMY_ERR_BAD_PARAM;
  kmy_ctx tmp;
  std::string err;
  const int rc = parse_deck(&tmp, deck);
  if (rc) return rc;
  const std::string k = tune_config_key(&tmp);
  if (k.size() + 1 > n) return KMY_ERR_BAD_PARAM;
  std::memcpy(buf, k.c_str(), k.size() + 1);
  return KMY_OK;
}

int kmy_tune_cache_put(const char *key, const char *choice, double ms) {
  if (!key || !choice || !find_cand(choice) || std::strchr(key, '\t') || std::strchr(key, '\n'))
    return KMY_ERR_BAD_PARAM;
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache[key] = Entry{choice, ms};
  return KMY_OK;
}

int kmy_tune_cache_get(const char *key, char *choice, size_t n, double *ms) {
  if (!key || !choice || n == 0) return KMY_ERR_BAD_PARAM;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cache.find(key);
  if (it == g_cache.end()) return KMY_ERR_STATE;
  if (it->second.choice.size() + 1 > n) return KMY_ERR_BAD_PARAM;
  std::memcpy(choice, it->second.choice.c_str(), it->second.choice.size() + 1);
  if (ms) *ms = it->second.ms;
  return KMY_OK;
}

int kmy_tune_cache_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache.clear();
  return KMY_OK;
}

int kmy_tune_cache_save(const char *path) {
  if (!path) return KMY_ERR_BAD_PARAM;
  std::lock_guard<std::mutex> lk(g_mu);
  std::ofstream f(path);
  if (!f) return KMY_ERR_BAD_PARAM;
  for (const auto &kv : g_cache) f << kv.first << '\t' << kv.second.choice << '\t' << kv.second.ms << '\n';
  return f.good() ? KMY_OK : KMY_ERR_BAD_PARAM;
}

int kmy_tune_cache_load(const char *path) {
  if (!path) return KMY_ERR_BAD_PARAM;
  std::ifstream f(path);
  if (!f) return KMY_ERR_BAD_PARAM;
  std::string line;
  std::lock_guard<std::mutex> lk(g_mu);
  while (std::getline(f, line)) {
    const size_t a = line.find('\t'), b = a == std::string::npos ? a : line.find('\t', a + 1);
    if (b == std::string::npos) continue;  // not three fields
    const std::string key = line.substr(0, a), choice = line.substr(a + 1, b - a - 1);
    char *end = nullptr;
    const double ms = std::strtod(line.c_str() + b + 1, &end);
    if (key.empty() || !find_cand(choice) || end == line.c_str() + b + 1) continue;
    g_cache[key] = Entry{choice, ms};
  }
  return KMY_OK;
}

int kmy_autotune(kmy_ctx *c, int reps, kmy_tune_result *out, int max_out, int *n_out) {
  if (!c) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  std::vector<std::pair<std::string, double>> res;
  const int rc = tune_run(c, reps, &res);
  if (n_out) *n_out = int(res.size());
  for (int i = 0; out && i < int(res.size()) && i < max_out; i++) {
    std::snprintf(out[i].name, sizeof(out[i].name), "%s", res[size_t(i)].first.c_str());
    out[i].ms = res[size_t(i)].second;
    out[i].applies = res[size_t(i)].second >= 0.0 ? 1 : 0;
  }
  return rc;
}

int kmy_stage_kernel(const kmy_ctx *c, char *name, size_t n) {
  if (!c || !name || n == 0) return KMY_ERR_BAD_PARAM;
  const char *s = "tasks";
  if (c->path == 0 && !c->amr.on) {
    if (c->prm.stage_kernel == 3 && !c->prm.mhd) s = "tune";
    else if (slab_runs(c)) s = slab_rows(c) == 8 ? "slab8" : "slab16";
    else s = c->prm.stage_kernel == 2 ? "slab (does not apply)" : "brick";
  }
  std::snprintf(name, n, "%s", s);
  return KMY_OK;
}

}  // extern "C"
