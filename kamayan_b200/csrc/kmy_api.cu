// kmy_api.cu -- C ABI of libkmy_hydro: contexts, deck parameters, MeshData
// import/export and the RK driver (stage sequencing + device dt controller).
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <sstream>

#include "../../include/kmy_hydro.h"
#include "kmy_internal.hpp"

using kmy::Container;

namespace kmy {

int cuda_check(kmy_ctx *c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return KMY_OK;
  c->err = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return KMY_ERR_OOM;
  return KMY_ERR_CUDA;
}

double Params::real(const std::string &k, double d) const {
  auto it = deck.find(k);
  return it == deck.end() ? d : std::strtod(it->second.c_str(), nullptr);
}
int Params::integer(const std::string &k, int d) const {
  auto it = deck.find(k);
  return it == deck.end() ? d : std::atoi(it->second.c_str());
}
std::string Params::str(const std::string &k, const std::string &d) const {
  auto it = deck.find(k);
  return it == deck.end() ? d : it->second;
}

// Parthenon input-deck syntax: "<block>" headers, "key = value" lines, '#'
// comments, and "block/key = value" lines that name their block themselves.
static void parse_deck(const char *text, std::map<std::string, std::string> &kv) {
  std::istringstream in(text ? text : "");
  std::string line, block;
  auto trim = [](const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return std::string();
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
  };
  while (std::getline(in, line)) {
    auto hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    line = trim(line);
    if (line.empty()) continue;
    if (line.front() == '<' && line.back() == '>') {
      block = trim(line.substr(1, line.size() - 2));
      continue;
    }
    auto eq = line.find('=');
    if (eq == std::string::npos) continue;
    std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
    if (key.find('/') != std::string::npos) kv[key] = val;
    else kv[block + "/" + key] = val;
  }
}

static int bc_kind(const std::string &s, bool &ok) {
  if (s == "periodic") return BC_PERIODIC;
  if (s == "outflow") return BC_OUTFLOW;
  if (s == "reflect" || s == "reflecting") return BC_REFLECT;
  ok = false;
  return BC_OUTFLOW;
}

static bool one_of(const std::string &v, std::initializer_list<const char *> opts) {
  for (auto o : opts)
    if (v == o) return true;
  return false;
}

// Validates and fills ctx->prm / ctx->m.  Mirrors the option lists of the
// reference's AddParm calls (hydro.cpp:55-90, grid.cpp:175-228,
// kamayan_driver.cpp:25-80, eos.cpp:32-49, physics.cpp:20-23).
static int setup_params(kmy_ctx *c, const char *deck) {
  Params &p = c->prm;
  parse_deck(deck, p.deck);
  auto bad = [&](const std::string &msg) {
    c->err = msg;
    return int(KMY_ERR_BAD_PARAM);
  };
  const std::string rc = p.str("hydro/reconstruction", "fog");
  if (!one_of(rc, {"fog", "plm", "ppm", "wenoz"})) return bad("hydro/reconstruction: " + rc);
  p.recon = rc == "plm" ? PLM : rc == "ppm" ? PPM : rc == "wenoz" ? WENOZ : FOG;
  const std::string sl = p.str("hydro/slope_limiter", "minmod");
  if (!one_of(sl, {"minmod", "van_leer", "mc"})) return bad("hydro/slope_limiter: " + sl);
  p.limiter = sl == "mc" ? MC : sl == "van_leer" ? VAN_LEER : MINMOD;
  const std::string rs = p.str("hydro/riemann", "hll");
  if (!one_of(rs, {"hll", "hllc"})) return bad("hydro/riemann: " + rs);
  p.riemann = rs == "hllc" ? HLLC : HLL;
  if (!one_of(p.str("hydro/ReconstructionVars", "primitive"), {"primitive"}))
    return bad("hydro/ReconstructionVars");
  if (!one_of(p.str("hydro/ReconstructionStrategy", "scratchpad"), {"scratchpad", "scratchvar"}))
    return bad("hydro/ReconstructionStrategy");
  if (!one_of(p.str("hydro/EMF_averaging", "arithmetic"), {"arithmetic"}))
    return bad("hydro/EMF_averaging");
  p.cfl = p.real("hydro/cfl", 0.8);
  const std::string mhd = p.str("physics/MHD", "off");
  if (!one_of(mhd, {"off", "ct"})) return bad("physics/MHD: " + mhd);
  p.mhd = mhd == "ct";
  if (p.str("physics/fluid", "oneT") != "oneT") return bad("physics/fluid: only oneT is implemented");
  if (p.str("geometry/geometry", "cartesian") != "cartesian")
    return bad("geometry/geometry: only cartesian is supported");
  if (p.str("material/single/eos_type", "gamma") != "gamma") return bad("material/single/eos_type");
  if (!one_of(p.str("eos/mode_init", "dens_pres"), {"dens_pres"}))
    return bad("eos/mode_init: only dens_pres is supported");
  p.gamma = p.real("material/single/gamma", 5.0 / 3.0);
  p.Abar = p.real("material/single/Abar", 1.0);
  const std::string prec = p.str("kamayan_b200/precision", "fp64");
  if (!one_of(prec, {"fp64", "fp32"})) return bad("kamayan_b200/precision: " + prec);
  p.precision = prec == "fp32" ? 32 : 64;
  const std::string sk = p.str("kamayan_b200/stage_kernel", "auto");
  if (!one_of(sk, {"auto", "brick", "slab", "tune"})) return bad("kamayan_b200/stage_kernel: " + sk);
  p.stage_kernel = sk == "auto" ? 0 : sk == "brick" ? 1 : sk == "slab" ? 2 : 3;
  const std::string sr = p.str("kamayan_b200/slab_rows", "auto");
  if (!one_of(sr, {"auto", "8", "16"})) return bad("kamayan_b200/slab_rows: " + sr);
  p.slab_rows = sr == "auto" ? 0 : std::stoi(sr);
  const std::string ln = p.str("kamayan_b200/launch", "batched");
  if (!one_of(ln, {"batched", "per_block"})) return bad("kamayan_b200/launch: " + ln);
  p.per_block = ln == "per_block";
  if (p.per_block && p.stage_kernel == 0) p.stage_kernel = 1;  // the per-block launches are of the brick stage
  const std::string cu = p.str("kamayan_b200/ct_update", "auto");
  if (!one_of(cu, {"auto", "streamed", "per_face"})) return bad("kamayan_b200/ct_update: " + cu);
  p.ct_update = cu == "auto" ? 0 : cu == "streamed" ? 1 : 2;

  const std::string integ = p.str("parthenon/time/integrator", "rk2");
  if (integ == "rk1") p.beta = {1.0};
  else if (integ == "rk2") p.beta = {1.0, 0.5};
  else if (integ == "rk3") p.beta = {1.0, 0.25, 2.0 / 3.0};
  else return bad("parthenon/time/integrator: " + integ);
  const int ns = int(p.beta.size());
  p.stage_name.assign(ns + 1, "base");
  for (int s = 1; s < ns; s++) p.stage_name[s] = std::to_string(s);

  const double big = std::numeric_limits<double>::max();
  p.tp.tlim = p.real("parthenon/time/tlim", big);
  p.tp.nlim = p.integer("parthenon/time/nlim", -1);
  p.tp.dt_factor = p.real("parthenon/time/dt_factor", 2.0);
  p.tp.dt_init = p.real("parthenon/time/dt_init", big);
  p.tp.dt_ceil = p.real("parthenon/time/dt_ceil", big);
  p.tp.dt_user = p.real("parthenon/time/dt_user", big);
  p.tp.dt_floor = p.real("parthenon/time/dt_floor", std::numeric_limits<double>::min());
  p.tp.dt_min = p.real("parthenon/time/dt_min", std::numeric_limits<double>::lowest());
  p.tp.dt_max = p.real("parthenon/time/dt_max", std::numeric_limits<double>::max());
  p.tp.dt_min_cycle_limit = p.integer("parthenon/time/dt_min_cycle_limit", 10);
  p.tp.dt_max_cycle_limit = p.integer("parthenon/time/dt_max_cycle_limit", 1);
  if (p.tp.dt_min_cycle_limit < 1 || p.tp.dt_max_cycle_limit < 1)
    return bad("parthenon/time/dt_min_cycle_limit and dt_max_cycle_limit must be positive");

  const std::string refine = p.str("parthenon/mesh/refinement", "none");
  if (!one_of(refine, {"none", "static", "adaptive"})) return bad("parthenon/mesh/refinement");
  const int numlevel = p.integer("parthenon/mesh/numlevel", 1);
  if (refine == "static" && numlevel > 1)
    return bad("parthenon/mesh/refinement = static with numlevel > 1 is not supported");
  // adaptive mesh: one criterion per <kamayan/refinementN> block, N = 0, 1, ...
  // while the blocks exist; a block without a field adds none
  // (grid.cpp:43-48, :90-124, :127-141)
  AmrHost &amr = c->amr;
  amr.crits.clear();
  if (refine == "adaptive") {
    for (int n = 0;; n++) {
      const std::string b = "kamayan/refinement" + std::to_string(n) + "/";
      auto it = p.deck.lower_bound(b);
      if (it == p.deck.end() || it->first.compare(0, b.size(), b) != 0) break;
      if (!p.deck.count(b + "field")) continue;
      AmrCriterion cr;
      cr.field = p.str(b + "field", "dens");
      if (!one_of(cr.field, {"dens", "pres", "ener"})) return bad(b + "field: " + cr.field);
      if (p.str(b + "method", "loehner") != "loehner") return bad(b + "method: only loehner is implemented");
      cr.refine_tol = p.real(b + "refine_tol", 0.8);
      cr.derefine_tol = p.real(b + "derefine_tol", 0.2);
      cr.filter = p.real(b + "filter", 0.01);
      cr.max_level = std::min(numlevel - 1, p.integer(b + "max_level", numlevel - 1));
      amr.crits.push_back(cr);
    }
  }
  amr.on = numlevel > 1 && !amr.crits.empty();
  if (amr.on) {
    if (numlevel > 8) return bad("parthenon/mesh/numlevel: at most 8 levels");
    amr.numlevel = numlevel;
    amr.max_level = numlevel - 1;
    amr.derefine_count = p.integer("parthenon/mesh/derefine_count", 10);
  }

  MeshDesc &m = c->m;
  const char *ax[3] = {"1", "2", "3"};
  for (int i = 0; i < 3; i++) {
    m.mesh_nx[i] = p.integer(std::string("parthenon/mesh/nx") + ax[i], 32);
    m.nx[i] = p.integer(std::string("parthenon/meshblock/nx") + ax[i], m.mesh_nx[i]);
    m.xmin[i] = p.real(std::string("parthenon/mesh/x") + ax[i] + "min", 0.0);
    const double xmax = p.real(std::string("parthenon/mesh/x") + ax[i] + "max", 1.0);
    bool ok = true;
    m.bc[i][0] = bc_kind(p.str(std::string("parthenon/mesh/ix") + ax[i] + "_bc", "outflow"), ok);
    m.bc[i][1] = bc_kind(p.str(std::string("parthenon/mesh/ox") + ax[i] + "_bc", "outflow"), ok);
    if (!ok) return bad(std::string("parthenon/mesh boundary condition along x") + ax[i]);
    m.dx[i] = xmax - m.xmin[i];  // divided below
  }
  m.ndim = m.mesh_nx[2] > 1 ? 3 : (m.mesh_nx[1] > 1 ? 2 : 1);
  for (int i = m.ndim; i < 3; i++) m.nx[i] = m.mesh_nx[i] = 1;
  const int ng = p.integer("parthenon/mesh/nghost", 4);
  const int need = ReconWidthRuntime(p.recon) + 1 + (p.mhd ? 1 : 0);
  if (ng < need) return bad("parthenon/mesh/nghost too small for the reconstruction");
  // the refinement estimator takes second differences across the block edge
  if (c->amr.on && ng < 2) return bad("parthenon/mesh/nghost: adaptive meshes need at least 2");
  m.nb = 1;
  for (int i = 0; i < 3; i++) {
    if (m.nx[i] <= 0 || m.mesh_nx[i] % m.nx[i] != 0)
      return bad("parthenon/mesh nx must be a multiple of parthenon/meshblock nx");
    if (i < m.ndim && m.nx[i] < ng) return bad("meshblock smaller than nghost");
    if ((m.bc[i][0] == BC_PERIODIC) != (m.bc[i][1] == BC_PERIODIC))
      return bad("periodic boundaries must be periodic on both sides");
    m.nbx[i] = m.mesh_nx[i] / m.nx[i];
    m.nb *= m.nbx[i];
    m.g[i] = i < m.ndim ? ng : 0;
    m.np[i] = m.nx[i] + 2 * m.g[i];
    m.nf[i] = m.np[i] + (i < m.ndim ? 1 : 0);
    m.dx[i] = m.dx[i] / double(m.mesh_nx[i]);
  }
  m.P = (long long)m.np[0] * m.np[1] * m.np[2];
  m.Pf = (long long)m.nf[0] * m.nf[1] * m.nf[2];
  m.area[0] = m.dx[1] * m.dx[2];
  m.area[1] = m.dx[0] * m.dx[2];
  m.area[2] = m.dx[0] * m.dx[1];
  m.vol = m.dx[0] * m.dx[1] * m.dx[2];
  p.tp.cfl_over_ndim = p.cfl / double(m.ndim);

  const double kboltz = 1.380649e-16;
  c->eos.cv = p.gamma * kboltz / p.Abar;
  c->eos.gm1 = p.gamma - 1.0;
  c->ncc = p.mhd ? 8 : 5;
  c->esz = p.precision == 32 ? 4 : 8;
  return KMY_OK;
}

int parse_deck(kmy_ctx *tmp, const char *deck) { return setup_params(tmp, deck); }

// Device bytes a fused-path context for `deck` allocates at kmy_create, and
// the deck's kernel class.  Host-only: parses and validates the deck.
int deck_footprint(const char *deck, Footprint *out, std::string *err) {
  kmy_ctx tmp;
  const int rc = setup_params(&tmp, deck);
  if (rc) {
    if (err) *err = tmp.err;
    return rc;
  }
  if (tmp.amr.on) {
    if (err) *err = "adaptive meshes are not batched: the block count changes between steps";
    return KMY_ERR_BAD_PARAM;
  }
  const MeshDesc &m = tmp.m;
  const size_t n = size_t(m.nb) * m.P, nf = size_t(m.nb) * m.Pf;
  const size_t ns = tmp.prm.beta.size();
  size_t per = tmp.esz * tmp.ncc * n + (tmp.esz == 4 ? 4 * n : 0);
  if (tmp.prm.mhd) per += 2 * tmp.esz * 3 * nf;
  out->bytes = ns * per + tmp.esz * NPRIM * n + (tmp.prm.mhd ? 8 * n : 0) + sizeof(DevClock) + 512;
  out->esz = int(tmp.esz);
  out->ndim = m.ndim;
  out->recon = tmp.prm.recon;
  out->riemann = tmp.prm.riemann;
  out->nstages = int(ns);
  out->mhd = tmp.prm.mhd ? 1 : 0;
  out->cells = (long long)m.mesh_nx[0] * m.mesh_nx[1] * m.mesh_nx[2];
  return KMY_OK;
}

// Context memory comes from the device's stream-ordered pool.  The pool keeps
// freed blocks for reuse (release threshold raised once per device, for this
// process only), so creating and destroying contexts -- one per request in
// the serving loop -- does not synchronise the device or return to the driver.
static void keep_pool(int device) {
  static bool done[64] = {};
  if (device < 0 || device >= 64 || done[device]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t threshold = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  done[device] = true;
}

int dalloc(kmy_ctx *c, void **p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return KMY_OK;
  cudaError_t e = cudaMallocAsync(p, bytes, c->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    c->err = "device allocation of " + std::to_string(bytes) + " bytes failed";
    return KMY_ERR_OOM;
  }
  c->allocations.push_back(*p);
  return cuda_check(c, cudaMemsetAsync(*p, 0, bytes, c->stream), "memset");
}

void *host_pin(kmy_ctx *c, size_t bytes) {
  if (bytes <= c->h_pin_bytes) return c->h_pin;
  if (c->h_pin) cudaFreeHost(c->h_pin);
  c->h_pin = nullptr;
  c->h_pin_bytes = 0;
  const size_t n = std::max(bytes, size_t(4096));
  if (cudaMallocHost(&c->h_pin, n) != cudaSuccess) {
    cudaGetLastError();
    c->h_pin = nullptr;
    c->err = "pinned host allocation of " + std::to_string(n) + " bytes failed";
    return nullptr;
  }
  c->h_pin_bytes = n;
  return c->h_pin;
}

void dfree(kmy_ctx *c, void *p) {
  if (!p) return;
  for (size_t i = 0; i < c->allocations.size(); i++)
    if (c->allocations[i] == p) {
      c->allocations.erase(c->allocations.begin() + long(i));
      cudaFreeAsync(p, c->stream);
      return;
    }
}

int make_container(kmy_ctx *c, const std::string &name) {
  Container ct;
  const MeshDesc &m = c->m;
  const size_t n = size_t(m.nb) * m.P, nf = size_t(m.nb) * m.Pf;
  int rc = dalloc(c, &ct.cc, c->esz * c->ncc * n);
  if (!rc && c->esz == 4) rc = dalloc(c, &ct.ener_lo, 4 * n);
  if (!rc && c->prm.mhd) rc = dalloc(c, &ct.fc, c->esz * 3 * nf);
  if (!rc && c->prm.mhd) rc = dalloc(c, &ct.emf, c->esz * 3 * nf);
  if (rc) return rc;
  c->md[name] = ct;
  return KMY_OK;
}

}  // namespace kmy

using namespace kmy;

// Containers by name.  "dUdt" is only needed by the per-task path and is
// allocated on first use, so fused-only contexts (the serving path) never
// hold it.
static Container *find_container(kmy_ctx *c, const char *name) {
  const std::string n(name ? name : "");
  auto it = c->md.find(n);
  if (it == c->md.end() && n == "dUdt") {
    if (make_container(c, "dUdt")) return nullptr;
    it = c->md.find(n);
  }
  if (it == c->md.end()) {
    c->err = "unknown container " + n;
    return nullptr;
  }
  return &it->second;
}

// ----------------------------------------------------------------------------
// staging conversions between host doubles and device storage
__global__ void k_store_cells(const double *src, void *dst, float *lo, size_t n, int f32) {
  size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const double v = src[i];
  if (f32) {
    const float hi = float(v);
    static_cast<float *>(dst)[i] = hi;
    if (lo) lo[i] = float(v - double(hi));
  } else {
    static_cast<double *>(dst)[i] = v;
  }
}
__global__ void k_load_cells(const void *src, const float *lo, double *dst, size_t n, int f32) {
  size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  if (f32) {
    double v = double(static_cast<const float *>(src)[i]);
    if (lo) v += double(lo[i]);
    dst[i] = v;
  } else {
    dst[i] = static_cast<const double *>(src)[i];
  }
}

// Resolve (container, var, comp) to device storage.
struct VarRef {
  void *p = nullptr;
  float *lo = nullptr;
  bool is_double = false;
  size_t n = 0;
};

static int resolve(kmy_ctx *c, const char *container, const char *var, int comp, VarRef &r) {
  const MeshDesc &m = c->m;
  const size_t n = size_t(m.nb) * m.P, nf = size_t(m.nb) * m.Pf;
  const std::string v(var ? var : "");
  auto shared = [&](int slot) {
    r.p = static_cast<char *>(c->prim) + c->esz * n * slot;
    r.n = n;
    return int(KMY_OK);
  };
  if (v == "velocity" && comp >= 0 && comp < 3) return shared(PVEL0 + comp);
  if (v == "pres") return shared(PPRES);
  if (v == "bulk modulus") return shared(PBMOD);
  if (v == "eint") return shared(PEINT);
  if (v == "temp") return shared(PTEMP);
  if (v == "divb" && c->prm.mhd) {
    r.p = c->divb;
    r.is_double = true;
    r.n = n;
    return KMY_OK;
  }
  Container *ct = find_container(c, container);
  if (!ct) return KMY_ERR_BAD_PARAM;
  auto cell = [&](int slot) {
    r.p = static_cast<char *>(ct->cc) + c->esz * n * slot;
    r.n = n;
    return int(KMY_OK);
  };
  if (v == "dens") return cell(CDENS);
  if (v == "momentum" && comp >= 0 && comp < 3) return cell(CMOM0 + comp);
  if (v == "ener") {
    r.lo = static_cast<float *>(ct->ener_lo);
    return cell(CENER);
  }
  if (v == "magc" && c->prm.mhd && comp >= 0 && comp < 3) return cell(CMAGC0 + comp);
  if (v == "mag" && c->prm.mhd && comp >= 0 && comp < 3) {
    r.p = static_cast<char *>(ct->fc) + c->esz * nf * comp;
    r.n = nf;
    return KMY_OK;
  }
  c->err = "unknown variable " + v + " (comp " + std::to_string(comp) + ")";
  return KMY_ERR_BAD_PARAM;
}

// Materialise the reference-visible state of "base" after fused steps:
// primitives from PreparePrimitive and filled ghosts.
static int materialize(kmy_ctx *c) {
  if (c->prims_valid) return KMY_OK;
  Container &b = c->md["base"];
  int rc = launch_prepare_primitive(c, b);
  if (!rc) rc = launch_fill_ghosts(c, b);
  if (!rc) c->prims_valid = true;
  return rc;
}

extern "C" {

int kmy_create(const char *deck, int device, kmy_ctx **out) {
  if (!out) return KMY_ERR_BAD_PARAM;
  *out = nullptr;
  auto *c = new kmy_ctx();
  c->device = device;
  c->deck_text = deck ? deck : "";
  int rc = setup_params(c, deck);
  if (rc) {
    std::fprintf(stderr, "kmy_create: %s\n", c->err.c_str());
    delete c;
    return rc;
  }
  rc = cuda_check(c, cudaSetDevice(device), "cudaSetDevice");
  if (!rc) rc = cuda_check(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
  if (rc) {
    std::fprintf(stderr, "kmy_create: %s\n", c->err.c_str());
    delete c;
    return rc;
  }
  c->own_stream = true;
  keep_pool(device);
  const size_t n = size_t(c->m.nb) * c->m.P;
  for (size_t s = 0; s + 1 < c->prm.stage_name.size() && !rc; s++)
    if (!c->md.count(c->prm.stage_name[s])) rc = make_container(c, c->prm.stage_name[s]);
  if (!rc) rc = dalloc(c, &c->prim, c->esz * NPRIM * n);
  if (!rc && c->prm.mhd) rc = dalloc(c, reinterpret_cast<void **>(&c->divb), 8 * n);
  if (!rc) rc = dalloc(c, reinterpret_cast<void **>(&c->clock), sizeof(DevClock));
  if (!rc) rc = dalloc(c, reinterpret_cast<void **>(&c->scratch), 8 * 64);
  if (!rc && c->amr.on) rc = amr_setup(c);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "create sync");
  if (rc) {
    std::fprintf(stderr, "kmy_create: %s\n", c->err.c_str());
    kmy_destroy(c);
    return rc;
  }
  *out = c;
  return KMY_OK;
}

int kmy_destroy(kmy_ctx *c) {
  if (!c) return KMY_OK;
  cudaSetDevice(c->device);
  if (c->evolve_exec) cudaGraphExecDestroy(c->evolve_exec);
  for (cudaEvent_t &e : c->ev_evolve)
    if (e) cudaEventDestroy(e);
  for (auto &pair : c->pipe_ev)
    for (cudaEvent_t &e : pair)
      if (e) cudaEventDestroy(e);
  for (void *p : c->allocations) cudaFreeAsync(p, c->stream);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (char *&p : c->pipe_pin)
    if (p) cudaFreeHost(p);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  if (c->h_pin) cudaFreeHost(c->h_pin);
  delete c;
  return KMY_OK;
}

const char *kmy_last_error(const kmy_ctx *c) { return c ? c->err.c_str() : "null context"; }

int kmy_get_info(const kmy_ctx *c, kmy_info *o) {
  if (!c || !o) return KMY_ERR_BAD_PARAM;
  const MeshDesc &m = c->m;
  o->ndim = m.ndim;
  o->nblocks = m.nb;
  for (int i = 0; i < 3; i++) {
    o->nx[i] = m.nx[i];
    o->ncells_pad[i] = m.np[i];
    o->nfaces_pad[i] = m.nf[i];
    o->nblocks_dim[i] = m.nbx[i];
    o->xmin[i] = m.xmin[i];
    o->dx[i] = m.dx[i];
    o->xmax[i] = m.xmin[i] + m.dx[i] * m.mesh_nx[i];
  }
  o->nghost = m.g[0];
  o->ncons = c->ncc;
  o->mhd = c->prm.mhd ? 1 : 0;
  o->nstages = int(c->prm.beta.size());
  o->precision = c->prm.precision;
  return KMY_OK;
}

int kmy_set_stream(kmy_ctx *c, void *s) {
  if (!c) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  if (s) {
    cudaStreamSynchronize(c->stream);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->stream = static_cast<cudaStream_t>(s);
    c->own_stream = false;
  }
  return KMY_OK;
}

int kmy_sync(kmy_ctx *c) {
  if (!c) return KMY_ERR_BAD_PARAM;
  return cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
}

int kmy_import_var(kmy_ctx *c, const char *container, const char *var, int comp,
                   const double *host, size_t n) {
  if (!c || !host) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  VarRef r;
  int rc = resolve(c, container, var, comp, r);
  if (rc) return rc;
  if (n != r.n) {
    c->err = "size mismatch: expected " + std::to_string(r.n);
    return KMY_ERR_BAD_PARAM;
  }
  const std::string vn(var);
  if (vn == "velocity" || vn == "pres" || vn == "bulk modulus" || vn == "eint" || vn == "temp")
    c->prims_imported = true;
  if (Container *w = find_container(c, container)) w->ghosts = false;
  if (r.is_double || c->esz == 8) {
    rc = cuda_check(c, cudaMemcpyAsync(r.p, host, n * 8, cudaMemcpyHostToDevice, c->stream), "import copy");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "import sync");
    c->prims_valid = true;
    return rc;
  }
  double *stage = nullptr;
  rc = cuda_check(c, cudaMallocAsync(reinterpret_cast<void **>(&stage), n * 8, c->stream), "stage");
  if (rc) return rc;
  rc = cuda_check(c, cudaMemcpyAsync(stage, host, n * 8, cudaMemcpyHostToDevice, c->stream), "import");
  if (!rc) {
    k_store_cells<<<unsigned((n + 255) / 256), 256, 0, c->stream>>>(stage, r.p, r.lo, n, 1);
    c->launches++;
    rc = cuda_check(c, cudaGetLastError(), "k_store_cells");
  }
  cudaFreeAsync(stage, c->stream);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "import sync");
  c->prims_valid = true;
  return rc;
}

int kmy_export_var(kmy_ctx *c, const char *container, const char *var, int comp, double *host,
                   size_t n) {
  if (!c || !host) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  VarRef r;
  int rc = resolve(c, container, var, comp, r);
  if (rc) return rc;
  if (n != r.n) {
    c->err = "size mismatch: expected " + std::to_string(r.n);
    return KMY_ERR_BAD_PARAM;
  }
  rc = materialize(c);
  if (rc) return rc;
  if (r.is_double || c->esz == 8) {
    rc = cuda_check(c, cudaMemcpyAsync(host, r.p, n * 8, cudaMemcpyDeviceToHost, c->stream), "export copy");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "export sync");
    return rc;
  }
  double *stage = nullptr;
  rc = cuda_check(c, cudaMallocAsync(reinterpret_cast<void **>(&stage), n * 8, c->stream), "stage");
  if (rc) return rc;
  k_load_cells<<<unsigned((n + 255) / 256), 256, 0, c->stream>>>(r.p, r.lo, stage, n, 1);
  c->launches++;
  rc = cuda_check(c, cudaGetLastError(), "k_load_cells");
  if (!rc) rc = cuda_check(c, cudaMemcpyAsync(host, stage, n * 8, cudaMemcpyDeviceToHost, c->stream), "export");
  cudaFreeAsync(stage, c->stream);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "export sync");
  return rc;
}

// Interior cells only, packed block-major then (k, j, i): scatter from a
// host-order staging buffer into the ghost-padded layout, and the gather
// back.  One thread per interior cell.
__global__ void k_store_interior(MeshDesc m, const double *src, void *dst, float *lo, int f32) {
  const size_t per = size_t(m.nx[0]) * m.nx[1] * m.nx[2];
  const size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (t >= per * m.nb) return;
  const size_t b = t / per, r = t - b * per;
  const size_t i = r % m.nx[0], q = r / m.nx[0], j = q % m.nx[1], k = q / m.nx[1];
  const size_t n = b * m.P + ((k + m.g[2]) * m.np[1] + (j + m.g[1])) * m.np[0] + (i + m.g[0]);
  const double v = src[t];
  if (f32) {
    const float hi = float(v);
    static_cast<float *>(dst)[n] = hi;
    if (lo) lo[n] = float(v - double(hi));
  } else {
    static_cast<double *>(dst)[n] = v;
  }
}
__global__ void k_load_interior(MeshDesc m, const void *src, const float *lo, double *dst, int f32) {
  const size_t per = size_t(m.nx[0]) * m.nx[1] * m.nx[2];
  const size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (t >= per * m.nb) return;
  const size_t b = t / per, r = t - b * per;
  const size_t i = r % m.nx[0], q = r / m.nx[0], j = q % m.nx[1], k = q / m.nx[1];
  const size_t n = b * m.P + ((k + m.g[2]) * m.np[1] + (j + m.g[1])) * m.np[0] + (i + m.g[0]);
  if (f32) {
    double v = double(static_cast<const float *>(src)[n]);
    if (lo) v += double(lo[n]);
    dst[t] = v;
  } else {
    dst[t] = static_cast<const double *>(src)[n];
  }
}

// Shared checks of the interior transfers: a cell variable and the interior
// cell count.
static int resolve_interior(kmy_ctx *c, const char *container, const char *var, int comp, size_t n,
                            VarRef &r) {
  int rc = resolve(c, container, var, comp, r);
  if (rc) return rc;
  const MeshDesc &m = c->m;
  if (r.n != size_t(m.nb) * m.P) {
    c->err = "interior transfers cover cell variables";
    return KMY_ERR_BAD_PARAM;
  }
  const size_t ni = size_t(m.nb) * m.nx[0] * m.nx[1] * m.nx[2];
  if (n != ni) {
    c->err = "size mismatch: expected " + std::to_string(ni) + " interior cells";
    return KMY_ERR_BAD_PARAM;
  }
  return KMY_OK;
}

int kmy_import_interior(kmy_ctx *c, const char *container, const char *var, int comp, const double *host,
                        size_t n) {
  if (!c || !host) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  VarRef r;
  int rc = resolve_interior(c, container, var, comp, n, r);
  if (rc) return rc;
  const std::string vn(var);
  if (vn == "velocity" || vn == "pres" || vn == "bulk modulus" || vn == "eint" || vn == "temp")
    c->prims_imported = true;
  if (Container *w = find_container(c, container)) w->ghosts = false;
  double *stage = nullptr;
  rc = cuda_check(c, cudaMallocAsync(reinterpret_cast<void **>(&stage), n * 8, c->stream), "stage");
  if (rc) return rc;
  rc = cuda_check(c, cudaMemcpyAsync(stage, host, n * 8, cudaMemcpyHostToDevice, c->stream), "import");
  if (!rc) {
    const int f32 = (r.is_double || c->esz == 8) ? 0 : 1;
    k_store_interior<<<unsigned((n + 255) / 256), 256, 0, c->stream>>>(c->m, stage, r.p, f32 ? r.lo : nullptr, f32);
    c->launches++;
    rc = cuda_check(c, cudaGetLastError(), "k_store_interior");
  }
  cudaFreeAsync(stage, c->stream);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "import sync");
  c->prims_valid = true;
  return rc;
}

int kmy_export_interior(kmy_ctx *c, const char *container, const char *var, int comp, double *host, size_t n) {
  if (!c || !host) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  VarRef r;
  int rc = resolve_interior(c, container, var, comp, n, r);
  if (rc) return rc;
  rc = materialize(c);
  if (rc) return rc;
  double *stage = nullptr;
  rc = cuda_check(c, cudaMallocAsync(reinterpret_cast<void **>(&stage), n * 8, c->stream), "stage");
  if (rc) return rc;
  const int f32 = (r.is_double || c->esz == 8) ? 0 : 1;
  k_load_interior<<<unsigned((n + 255) / 256), 256, 0, c->stream>>>(c->m, r.p, f32 ? r.lo : nullptr, stage, f32);
  c->launches++;
  rc = cuda_check(c, cudaGetLastError(), "k_load_interior");
  if (!rc) rc = cuda_check(c, cudaMemcpyAsync(host, stage, n * 8, cudaMemcpyDeviceToHost, c->stream), "export");
  cudaFreeAsync(stage, c->stream);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "export sync");
  return rc;
}

int kmy_finalize_import(kmy_ctx *c) {
  if (!c) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  Container &b = c->md["base"];
  int rc = KMY_OK;
  // primitives that were not imported come from the conserved state
  if (!c->prims_imported) rc = launch_prepare_primitive(c, b);
  c->prims_imported = false;
  if (!rc) rc = launch_fill_ghosts(c, b);
  if (!rc && c->prm.mhd) rc = launch_fill_derived(c, b);
  if (!rc) rc = launch_estimate_dt(c, b, true);
  if (!rc) rc = launch_dt_controller(c, 1);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "finalize");
  c->prims_valid = true;
  return rc;
}

int kmy_pgen(kmy_ctx *c, const char *problem) {
  if (!c || !problem) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  auto generate = [&]() {
    int r = launch_pgen(c, problem);
    if (!r) r = launch_eos_init(c, c->md["base"]);
    if (!r) r = launch_convert_to_conserved(c, c->md["base"]);
    if (!r) r = launch_fill_ghosts(c, c->md["base"]);
    return r;
  };
  int rc = KMY_OK;
  if (c->amr.on) {
    // initial refinement: generate, tag, refine (no derefinement) until the
    // mesh stops changing, then generate on the final mesh
    for (int it = 0; it < c->amr.numlevel && !rc; it++) {
      bool changed = false;
      rc = generate();
      if (!rc) rc = launch_amr_tag(c, c->md["base"]);
      if (!rc) rc = amr_remesh(c, false, &changed);
      if (!changed) break;
    }
    if (rc) return rc;
  }
  rc = generate();
  if (rc) return rc;
  if (c->amr.on) c->amr.cnt.assign(c->amr.cnt.size(), 0);
  Container &b = c->md["base"];
  if (c->prm.mhd) rc = launch_fill_derived(c, b);
  if (!rc) rc = launch_estimate_dt(c, b, true);
  if (!rc) rc = launch_dt_controller(c, 1);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "pgen");
  c->prims_valid = true;
  return rc;
}

#define KMY_CONTAINER(var, name)          \
  Container *var = find_container(c, name); \
  if (!var) return KMY_ERR_BAD_PARAM;

int kmy_compute_fluxes(kmy_ctx *c, const char *md0) {
  if (!c) return KMY_ERR_BAD_PARAM;
  KMY_CONTAINER(a, md0);
  return launch_compute_fluxes(c, *a);
}
int kmy_compute_emf(kmy_ctx *c, const char *md0) {
  if (!c) return KMY_ERR_BAD_PARAM;
  KMY_CONTAINER(a, md0);
  return launch_compute_emf(c, *a);
}
int kmy_flux_divergence(kmy_ctx *c, const char *md0, const char *dudt) {
  if (!c) return KMY_ERR_BAD_PARAM;
  KMY_CONTAINER(a, md0);
  KMY_CONTAINER(d, dudt);
  return launch_flux_divergence(c, *a, *d);
}
int kmy_apply_dudt(kmy_ctx *c, const char *base, const char *md0, const char *md1,
                   const char *dudt, double beta, double dt) {
  if (!c) return KMY_ERR_BAD_PARAM;
  KMY_CONTAINER(b, base);
  KMY_CONTAINER(a0, md0);
  KMY_CONTAINER(a1, md1);
  KMY_CONTAINER(d, dudt);
  a1->ghosts = false;
  return launch_apply_dudt(c, *b, *a0, *a1, *d, beta, dt, nullptr);
}
int kmy_prepare_primitive(kmy_ctx *c, const char *md1) {
  if (!c) return KMY_ERR_BAD_PARAM;
  KMY_CONTAINER(a, md1);
  return launch_prepare_primitive(c, *a);
}
int kmy_fill_ghosts(kmy_ctx *c, const char *md) {
  if (!c) return KMY_ERR_BAD_PARAM;
  KMY_CONTAINER(a, md);
  return launch_fill_ghosts(c, *a);
}
int kmy_estimate_dt(kmy_ctx *c, const char *md, double *dt_out) {
  if (!c) return KMY_ERR_BAD_PARAM;
  KMY_CONTAINER(a, md);
  int rc = launch_estimate_dt(c, *a, true);
  if (rc) return rc;
  DevClock h;
  rc = cuda_check(c, cudaMemcpyAsync(&h, c->clock, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "dt");
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "dt sync");
  if (rc) return rc;
  double dtmin;
  std::memcpy(&dtmin, &h.dtmin_bits, 8);
  if (dt_out) *dt_out = dtmin * c->prm.tp.cfl_over_ndim;
  return KMY_OK;
}
int kmy_fill_derived(kmy_ctx *c, const char *md) {
  if (!c) return KMY_ERR_BAD_PARAM;
  KMY_CONTAINER(a, md);
  return launch_fill_derived(c, *a);
}

// One stage through the per-task kernels, reference task order.  dt is read
// from the device clock when dt < 0.
static int task_stage(kmy_ctx *c, int stage, double dt) {
  const auto &nm = c->prm.stage_name;
  const int ns = int(c->prm.beta.size());
  Container *dup = find_container(c, "dUdt");
  if (!dup) return KMY_ERR_OOM;
  Container &base = c->md[nm[0]], &md0 = c->md[nm[stage - 1]], &md1 = c->md[nm[stage]];
  Container &du = *dup;
  if (!c->prims_valid) {
    // primitives of md0 are needed with ghosts (fused steps leave them stale)
    int rc = launch_prepare_primitive(c, md0);
    if (!rc) rc = launch_fill_ghosts(c, md0);
    if (rc) return rc;
    c->prims_valid = true;
  }
  md1.ghosts = false;
  int rc = launch_compute_fluxes(c, md0);
  if (!rc && c->amr.on) rc = launch_flux_correct(c);
  if (!rc) rc = launch_compute_emf(c, md0);
  if (!rc && c->amr.on) rc = launch_emf_correct(c, md0);
  // An adaptive hydro mesh has no fused stage; its divergence and update
  // share one pass.  Elsewhere the task list's kernels stay separate.
  if (c->amr.on && !c->prm.mhd) {
    if (!rc) rc = launch_div_apply(c, base, md0, md1, c->prm.beta[stage - 1], dt, dt < 0 ? &c->clock->dt : nullptr);
  } else {
    if (!rc) rc = launch_flux_divergence(c, md0, du);
    if (!rc) rc = launch_apply_dudt(c, base, md0, md1, du, c->prm.beta[stage - 1], dt,
                                    dt < 0 ? &c->clock->dt : nullptr);
  }
  if (!rc) rc = launch_prepare_primitive(c, md1);
  if (!rc && stage == ns) {
    rc = launch_estimate_dt(c, base, true);
    if (!rc && c->prm.mhd) rc = launch_fill_derived(c, base);
    // RefinementTagging runs before this stage's boundary exchange
    if (!rc && c->amr.on) rc = launch_amr_tag(c, base);
  }
  if (!rc) rc = launch_fill_ghosts(c, md1);
  return rc;
}

// After the stages of a step on an adaptive mesh (the dt controller has run):
// the tree update and remap.  The tags and the advanced clock come back in one
// read, and a step that leaves the mesh as it is keeps that clock for
// read_clock, so it syncs with the host once.  When the mesh changed, the next
// dt also respects the new blocks' CFL limit (controller mode 3).
static int amr_after_step(kmy_ctx *c) {
  bool changed = false;
  DevClock h{};
  int rc = amr_remesh(c, true, &changed, &h);
  if (rc) return rc;
  if (changed) {
    rc = launch_estimate_dt(c, c->md["base"], true);
    if (!rc) rc = launch_dt_controller(c, 3);
  } else {
    c->clock_host = h;
    c->clock_host_launches = c->launches;
  }
  return rc;
}

int kmy_task_stage(kmy_ctx *c, int stage, double dt) {
  if (!c || stage < 1 || stage > int(c->prm.beta.size())) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  return task_stage(c, stage, dt);
}

// A fused stage stages the primitives of its input from c->prim when they
// are current (after set-up, an import, the task path or a previous fused
// stage) and writes those of its output to c->prim_alt; the buffers swap.
// Constrained transport: the fused stage updates the cells and writes the
// transverse field fluxes; the face update (edge EMFs, Stokes, ApplyDuDt)
// and the primitives (which need the new cell-centred field) follow, in the order of the task list
// (hydro_add_flux_tasks.cpp, grid.cpp:213-241, primconsflux.cpp:82-142): in
// 3D blocks of 32-cell rows as the streamed face update and one cell pass
// (kmy_ct.cu), else one kernel per face direction and a primitive pass.
static int fused_stage_ct(kmy_ctx *c, int stage) {
  const auto &nm = c->prm.stage_name;
  const int ns = int(c->prm.beta.size());
  Container &base = c->md[nm[0]], &md0 = c->md[nm[stage - 1]], &md1 = c->md[nm[stage]];
  const bool stored = c->prims_valid || c->prims_interior;
  const double beta = c->prm.beta[stage - 1];
  md1.ghosts = false;
  // the cells: the z-streamed stage (FP32, 3D blocks of 32-cell rows) by
  // default, else the brick stage; both write the transverse field fluxes
  const char *no_slab = slab_unsupported(c);
  if (c->prm.stage_kernel == 2 && no_slab) {
    c->err = std::string("stage_kernel = slab: ") + no_slab;
    return KMY_ERR_BAD_PARAM;
  }
  int rc = ct_cells_on_slab(c) ? launch_slab_stage(c, base, md0, md1, beta, false)
                               : launch_fused_stage(c, base, md0, md1, beta, stored, false);
  if (!rc) rc = launch_flux_halo(c);
  if (!ct_stream_unsupported(c)) {
    // the streamed face update and cell pass (kmy_ct.cu); on the last stage,
    // whose output is "base", the cell pass also takes the CFL estimate and div B
    const bool fold = stage == ns && &md1 == &base;
    if (!rc) rc = launch_ct_stream(c, base, md0, md1, beta, fold);
    if (!rc && stage == ns && !fold) {
      rc = launch_estimate_dt(c, base, true);
      if (!rc) rc = launch_fill_derived(c, base);
    }
  } else {
    if (!rc) rc = launch_ct_faces(c, base, md0, md1, beta);
    if (!rc) rc = launch_prepare_primitive(c, md1);
    if (!rc && stage == ns) {
      rc = launch_estimate_dt(c, base, true);
      if (!rc) rc = launch_fill_derived(c, base);
    }
  }
  // interior primitives of md1 are current (ghost zones are not), unless the
  // z-streamed stage ran the cells (its cell pass stores no primitives)
  c->prims_interior = !rc && !ct_cells_on_slab(c);
  c->prims_valid = false;
  return rc;
}

// rk1 stages write the scratch container "1" (the stage reads neighbouring
// blocks of its input while it writes); "1" then becomes "base".  A base
// bound to caller memory keeps its arrays: the result is copied into them.
static int adopt_rk1_output(kmy_ctx *c) {
  Container &base = c->md["base"], &out = c->md["1"];
  if (!base.bound) {
    std::swap(c->md["base"], c->md["1"]);
    return KMY_OK;
  }
  const size_t n = size_t(c->m.nb) * c->m.P;
  int rc = cuda_check(c, cudaMemcpyAsync(base.cc, out.cc, c->esz * c->ncc * n, cudaMemcpyDeviceToDevice, c->stream),
                      "rk1 copy");
  if (!rc && base.ener_lo)
    rc = cuda_check(c, cudaMemcpyAsync(base.ener_lo, out.ener_lo, 4 * n, cudaMemcpyDeviceToDevice, c->stream),
                    "rk1 copy");
  base.ghosts = out.ghosts;
  return rc;
}

// Whether the hydro stage runs the z-streamed kernel (kmy_slab_host.cu): by
// default where it applies (3D, 32-cell rows) on meshes large enough to fill
// the GPU with its work items, or as the deck's <kamayan_b200> stage_kernel
// asks.
static bool use_slab(const kmy_ctx *c) { return slab_runs(c); }

// One stage through the z-streamed kernel.  rk1 updates base in place, and
// the kernel reads its input's neighbouring blocks while it writes, so rk1
// writes a scratch container and the two swap roles afterwards.
static int slab_stage(kmy_ctx *c, int stage) {
  const auto &nm = c->prm.stage_name;
  const int ns = int(c->prm.beta.size());
  int rc;
  if (ns == 1) {
    if (!c->md.count("1") && make_container(c, "1")) return KMY_ERR_OOM;
    Container &base = c->md["base"], &out = c->md["1"];
    rc = launch_slab_stage(c, base, base, out, c->prm.beta[0], true);
    if (!rc) rc = adopt_rk1_output(c);
  } else {
    Container &base = c->md[nm[0]], &md0 = c->md[nm[stage - 1]], &md1 = c->md[nm[stage]];
    rc = launch_slab_stage(c, base, md0, md1, c->prm.beta[stage - 1], stage == ns);
  }
  c->prims_interior = false;
  c->prims_valid = false;
  return rc;
}

static int fused_stage(kmy_ctx *c, int stage) {
  if (c->prm.mhd) return fused_stage_ct(c, stage);
  if (c->prm.stage_kernel == 3) {
    // stage_kernel = tune: the cached choice for this device and
    // configuration, else a tuning run now (never inside a stream capture:
    // kmy_evolve runs its first chunk uncaptured, and a capture keeps the
    // default choice until then)
    if (!tune_lookup(c)) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      cudaStreamIsCapturing(c->stream, &cs);
      if (cs == cudaStreamCaptureStatusNone) {
        if (const int rc = tune_run(c, 5, nullptr)) return rc;
      }
    }
  }
  if (c->prm.stage_kernel == 2) {
    if (const char *why = slab_unsupported(c)) {
      c->err = std::string("stage_kernel = slab: ") + why;
      return KMY_ERR_BAD_PARAM;
    }
  }
  if (use_slab(c)) return slab_stage(c, stage);
  const auto &nm = c->prm.stage_name;
  const int ns = int(c->prm.beta.size());
  // FP32 stages keep their output's primitives (kmy_fused.cu) in a second
  // buffer that swaps with the first; primitives bound to caller memory stay
  // where they are, so there every stage converts its input instead
  const bool keep = c->esz == 4 && !c->prim_bound;
  const bool stored = c->prims_valid || c->prims_interior;
  if (keep && !c->prim_alt && dalloc(c, &c->prim_alt, c->esz * NPRIM * size_t(c->m.nb) * c->m.P))
    return KMY_ERR_OOM;
  int rc;
  if (ns == 1) {
    // rk1 updates base in place (stage names base -> base).  The fused stage
    // reads neighbouring bricks' halos while it writes, so it writes a scratch
    // container and the two swap roles afterwards.
    if (!c->md.count("1") && make_container(c, "1")) return KMY_ERR_OOM;
    Container &base = c->md["base"], &out = c->md["1"];
    out.ghosts = false;
    rc = launch_fused_stage(c, base, base, out, c->prm.beta[0], stored, true);
    if (!rc) rc = adopt_rk1_output(c);
  } else {
    Container &base = c->md[nm[0]], &md0 = c->md[nm[stage - 1]], &md1 = c->md[nm[stage]];
    md1.ghosts = false;
    rc = launch_fused_stage(c, base, md0, md1, c->prm.beta[stage - 1], stored, stage == ns);
  }
  if (!rc && keep) std::swap(c->prim, c->prim_alt);
  c->prims_interior = !rc && keep;
  c->prims_valid = false;
  return rc;
}

int kmy_rk_stage(kmy_ctx *c, int stage, double dt) {
  if (!c || stage < 1 || stage > int(c->prm.beta.size())) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  if (dt >= 0) {
    int rc = cuda_check(c, cudaMemcpyAsync(&c->clock->dt, &dt, 8, cudaMemcpyHostToDevice, c->stream), "dt");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "dt sync");
    if (rc) return rc;
  }
  if (c->prm.mhd) {
    c->err = "the fused stage covers hydro; use kmy_task_stage for constrained transport";
    return KMY_ERR_BAD_PARAM;
  }
  if (c->amr.on) {
    c->err = "the fused stage covers single-level meshes; use kmy_task_stage on an adaptive mesh";
    return KMY_ERR_BAD_PARAM;
  }
  return fused_stage(c, stage);
}

// Whole steps go through the fused stage unless the path was set to tasks,
// the mesh is adaptive, or it carries CT in a configuration the fused stage
// does not cover.
static bool steps_fused(const kmy_ctx *c) {
  return c->path == 0 && !c->amr.on && (!c->prm.mhd || !fused_ct_unsupported(c));
}

static long long interior_cells(const kmy_ctx *c) {
  return (long long)c->m.nb * c->m.nx[0] * c->m.nx[1] * c->m.nx[2];
}

static int stages_async(kmy_ctx *c) {
  const int ns = int(c->prm.beta.size());
  int rc = KMY_OK;
  const bool fused = steps_fused(c);
  for (int s = 1; s <= ns && !rc; s++) rc = fused ? fused_stage(c, s) : task_stage(c, s, -1.0);
  return rc;
}

// After a step's stages: the dt controller, which counts the step's cells,
// then the tree update on an adaptive mesh.
static int finish_step(kmy_ctx *c, long long cells) {
  int rc = launch_dt_controller(c, 0, cells);
  if (!rc && c->amr.on) rc = amr_after_step(c);
  return rc;
}

static int step_async(kmy_ctx *c) {
  const long long cells = interior_cells(c);
  int rc = stages_async(c);
  if (!rc) rc = finish_step(c, cells);
  return rc;
}

// The device clock through the pinned staging (synchronizes the stream),
// unless an adaptive step's tag read just brought it back.
static int read_clock(kmy_ctx *c, DevClock &h, const char *what) {
  if (c->clock_host_launches == c->launches) {
    h = c->clock_host;
    c->clock_host_launches = -1;
    return KMY_OK;
  }
  DevClock *pin = static_cast<DevClock *>(host_pin(c, sizeof(DevClock)));
  if (!pin) return KMY_ERR_OOM;
  int rc = cuda_check(c, cudaMemcpyAsync(pin, c->clock, sizeof(DevClock), cudaMemcpyDeviceToHost, c->stream), what);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), what);
  if (!rc) h = *pin;
  return rc;
}

// The device clock's status word: a non-finite or non-positive CFL estimate
// (the dt controller), or a stage kernel's bounded wait that gave up.
static int clock_status(kmy_ctx *c, int status) {
  if (status == KMY_ERR_TIMEOUT) {
    c->err = "a stage kernel's bounded wait for its staged tiles gave up";
    return KMY_ERR_TIMEOUT;
  }
  if (status == KMY_ERR_DT_RANGE) {
    c->err = "the time step stayed outside [dt_min, dt_max] for the cycle limit";
    return KMY_ERR_DT_RANGE;
  }
  c->err = "non-finite or non-positive time-step estimate";
  return KMY_ERR_NONFINITE;
}

int kmy_step(kmy_ctx *c, double *dt_taken) {
  if (!c) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  int rc = step_async(c);
  if (rc) return rc;
  DevClock h;
  rc = read_clock(c, h, "step");
  if (rc) return rc;
  if (dt_taken) *dt_taken = h.dt_taken;
  if (h.status) return clock_status(c, h.status);
  return KMY_OK;
}

// kmy_evolve queues fused hydro steps in chunks of kChunk; the chunk runs as
// one CUDA graph (its 4 x kChunk or so launches cost one submission).  A
// graph replays the kernel arguments it was captured with, so it is keyed by
// the host-side state those arguments come from: the primitive buffers and
// containers (an even number of stages swaps them back), the flags that pick
// stored primitives, and the time parameters of the dt controller.  The first
// chunk after any change of that state runs uncaptured (first-use
// allocations, flags settling); the next one is captured and replayed until
// the state changes again.  An adaptive mesh steps one at a time (the host
// reads its tags after every step), so there the graph holds the stages of
// one step, and its key adds the mesh generation (every table upload changes
// the block list, the ghost plan and the buffers) and the flux buffer.
static constexpr int kChunk = 8;

static std::string evolve_key(const kmy_ctx *c) {
  std::string k;
  auto add = [&](const void *p, size_t n) { k.append(static_cast<const char *>(p), n); };
  const char kind = c->amr.on ? 'a' : 'f';
  add(&kind, 1);
  add(&c->prim, sizeof(c->prim));
  add(&c->prim_alt, sizeof(c->prim_alt));
  for (const auto &kv : c->md) add(&kv.second.cc, sizeof(kv.second.cc));
  const bool flags[2] = {c->prims_valid, c->prims_interior};
  add(flags, sizeof(flags));
  // the time parameters field by field (the struct's tail padding is not state)
  const TimeParams &tp = c->prm.tp;
  for (const double *d : {&tp.tlim, &tp.dt_factor, &tp.dt_init, &tp.dt_ceil, &tp.dt_user, &tp.dt_floor,
                          &tp.cfl_over_ndim, &tp.dt_min, &tp.dt_max})
    add(d, sizeof(double));
  for (const int *i : {&tp.nlim, &tp.dt_min_cycle_limit, &tp.dt_max_cycle_limit}) add(i, sizeof(int));
  // the stage kernel (the tuner may change it after the first chunk)
  add(&c->prm.stage_kernel, sizeof(int));
  add(&c->prm.slab_rows, sizeof(int));
  add(&c->stream, sizeof(c->stream));
  if (c->amr.on) {
    add(&c->amr.gen, sizeof(c->amr.gen));
    add(&c->flux, sizeof(c->flux));
  }
  return k;
}

// Run `body` through the cached graph, capturing it first when the state is
// steady.  *ran is false when the caller should run it uncaptured instead.
static int graph_run(kmy_ctx *c, const std::function<int()> &body, bool *ran) {
  *ran = false;
  const std::string key = evolve_key(c);
  if (c->evolve_exec && key == c->evolve_key) {
    c->launches += c->evolve_launches;
    c->graph_replays++;
    *ran = true;
    return cuda_check(c, cudaGraphLaunch(c->evolve_exec, c->stream), "evolve graph");
  }
  if (c->evolve_exec) {
    cudaGraphExecDestroy(c->evolve_exec);
    c->evolve_exec = nullptr;
  }
  if (key != c->evolve_seen) {  // first run in this state: uncaptured
    c->evolve_seen = key;
    return KMY_OK;
  }
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();  // e.g. the legacy default stream, which cannot be captured
    return KMY_OK;
  }
  const int64_t l0 = c->launches;
  int rc = body();
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (!rc) rc = cuda_check(c, e, "evolve capture");
  cudaGraphExec_t exec = nullptr;
  if (!rc) rc = cuda_check(c, cudaGraphInstantiate(&exec, g, 0), "evolve instantiate");
  if (g) cudaGraphDestroy(g);
  if (rc) return rc;
  // the captured work has not run yet; it runs now, and is kept when the
  // state after it is the state it started from
  rc = cuda_check(c, cudaGraphLaunch(exec, c->stream), "evolve graph");
  if (!rc && evolve_key(c) == key) {
    c->evolve_exec = exec;
    c->evolve_key = key;
    c->evolve_launches = c->launches - l0;
  } else {
    cudaGraphExecDestroy(exec);
  }
  *ran = !rc;
  return rc;
}

// ---------------------------------------------------------------------------
// kmy_evolve on an adaptive mesh.  Each step's stages and dt controller run
// as one graph; its tags, error flag and clock then come back to the host,
// which decides whether the mesh changes.  The host queues the next step
// before it waits for those reads, so the GPU does not idle while the host
// decides: that step is speculative.  Before it the base state (conserved,
// energy low words, faces, primitives, div B, clock) is copied aside on the
// device; when the current step's tags ask for a remesh, or the run ends
// with it (t_end, the step limit, a status), the speculative step is undone
// from that copy before the host goes on, so the results are those of
// stepping one at a time.

// Pinned slots, events and backup arrays for the current mesh (grown by half
// again when it outgrows them).  Called only with nothing in flight.
static int pipe_reserve(kmy_ctx *c) {
  // padded cells (or faces, the larger) of one array over all blocks
  const size_t cells = size_t(c->m.nb) * size_t(std::max<long long>(c->m.P, c->m.Pf));
  const size_t nb = size_t(c->m.nb);
  // pinned slots: [clock][error flag][tags]
  const size_t pin = sizeof(DevClock) + sizeof(int) * (nb + 1);
  if (pin > c->pipe_pin_bytes) {
    const size_t want = pin + pin / 2;
    for (char *&p : c->pipe_pin) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      if (cudaMallocHost(reinterpret_cast<void **>(&p), want) != cudaSuccess) {
        cudaGetLastError();
        c->err = "pinned host allocation failed";
        return KMY_ERR_OOM;
      }
    }
    c->pipe_pin_bytes = want;
  }
  for (auto &pair : c->pipe_ev)
    for (cudaEvent_t &e : pair)
      if (!e && cudaEventCreate(&e) != cudaSuccess) return cuda_check(c, cudaGetLastError(), "pipeline event");
  if (cells > c->bak_cells) {
    const size_t want = cells + cells / 2;
    for (void **p : {&c->bak_cc, &c->bak_lo, &c->bak_fc, &c->bak_prim, &c->bak_divb, &c->bak_clock}) {
      dfree(c, *p);
      *p = nullptr;
    }
    int rc = dalloc(c, &c->bak_cc, c->esz * c->ncc * want);
    if (!rc && c->esz == 4) rc = dalloc(c, &c->bak_lo, 4 * want);
    if (!rc && c->prm.mhd) rc = dalloc(c, &c->bak_fc, c->esz * 3 * want);
    if (!rc) rc = dalloc(c, &c->bak_prim, c->esz * NPRIM * want);
    if (!rc && c->prm.mhd) rc = dalloc(c, &c->bak_divb, 8 * want);
    if (!rc) rc = dalloc(c, &c->bak_clock, sizeof(DevClock));
    if (rc) return rc;
    c->bak_cells = want;
  }
  return KMY_OK;
}

// copy the base state's step-changed arrays aside (to_bak) or back
static int pipe_copy(kmy_ctx *c, bool to_bak) {
  Container &base = c->md["base"];
  const size_t n = size_t(c->m.nb) * size_t(c->m.P), nf = size_t(c->m.nb) * size_t(c->m.Pf);
  struct Arr {
    void *live, *bak;
    size_t bytes;
  };
  const Arr arrs[] = {{base.cc, c->bak_cc, c->esz * c->ncc * n},
                      {base.ener_lo, c->bak_lo, c->esz == 4 ? 4 * n : 0},
                      {base.fc, c->bak_fc, c->prm.mhd ? c->esz * 3 * nf : 0},
                      {c->prim, c->bak_prim, c->esz * NPRIM * n},
                      {c->divb, c->bak_divb, c->prm.mhd ? 8 * n : 0},
                      {c->clock, c->bak_clock, sizeof(DevClock)}};
  for (const Arr &a : arrs) {
    if (!a.bytes || !a.live) continue;
    void *dst = to_bak ? a.bak : a.live;
    const void *src = to_bak ? a.live : a.bak;
    if (int rc = cuda_check(c, cudaMemcpyAsync(dst, src, a.bytes, cudaMemcpyDeviceToDevice, c->stream), "pipeline copy"))
      return rc;
  }
  return KMY_OK;
}

static int evolve_amr(kmy_ctx *c, int nlim, int *n_out, DevClock &h) {
  AmrHost &a = c->amr;
  int rc = pipe_reserve(c);
  if (rc) return rc;
  // queue one step into slot k: timing event, (backup), stages + controller,
  // the reads of its tags, error flag and clock, timing event
  auto enqueue = [&](int k, bool speculative) -> int {
    int r = cuda_check(c, cudaEventRecord(c->pipe_ev[k][0], c->stream), "pipeline event");
    if (!r && speculative) r = pipe_copy(c, true);
    const long long cells = interior_cells(c);
    auto body = [&] {
      int q = stages_async(c);
      if (!q) q = launch_dt_controller(c, 0, cells);
      return q;
    };
    bool ran = false;
    if (!r) r = graph_run(c, body, &ran);
    if (!r && !ran) r = body();
    char *pin = c->pipe_pin[k];
    int *ip = reinterpret_cast<int *>(pin + sizeof(DevClock));
    if (!r)
      r = cuda_check(c, cudaMemcpyAsync(pin, c->clock, sizeof(DevClock), cudaMemcpyDeviceToHost, c->stream),
                     "pipeline clock");
    if (!r) r = cuda_check(c, cudaMemcpyAsync(ip, a.d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "pipeline err");
    if (!r)
      r = cuda_check(c, cudaMemcpyAsync(ip + 1, a.d_tags, sizeof(int) * size_t(c->m.nb), cudaMemcpyDeviceToHost,
                                        c->stream),
                     "pipeline tags");
    if (!r) r = cuda_check(c, cudaEventRecord(c->pipe_ev[k][1], c->stream), "pipeline event");
    return r;
  };
  int n = 0, cur = 0;
  rc = enqueue(cur, false);
  while (!rc) {
    // the speculative next step, unless the current one is the last allowed
    const bool spec = nlim < 0 || n + 1 < nlim;
    if (spec) rc = enqueue(1 - cur, true);
    if (!rc) rc = cuda_check(c, cudaEventSynchronize(c->pipe_ev[cur][1]), "pipeline wait");
    if (rc) break;
    float ms = 0.f;
    rc = cuda_check(c, cudaEventElapsedTime(&ms, c->pipe_ev[cur][0], c->pipe_ev[cur][1]), "pipeline event");
    if (rc) break;
    c->evolve_device_ms += double(ms);
    // the current step's reads
    const char *pin = c->pipe_pin[cur];
    std::memcpy(&h, pin, sizeof(DevClock));
    const int *ip = reinterpret_cast<const int *>(pin + sizeof(DevClock));
    const int nbt = c->m.nb;
    const std::vector<int> tags(ip + 1, ip + 1 + nbt);
    n++;
    bool any = false;
    rc = amr_count_tags(c, tags, ip[0], &any);
    const bool stop = rc || h.status || h.done || (nlim >= 0 && n >= nlim);
    // undo the speculative step (once): before a remap, or when the run ends
    bool undone = !spec;
    auto undo = [&]() -> int {
      if (undone) return KMY_OK;
      undone = true;
      int r = cuda_check(c, cudaStreamSynchronize(c->stream), "pipeline sync");
      if (!r) r = pipe_copy(c, false);
      return r;
    };
    bool changed = false;
    if (!rc && any) rc = amr_remesh_apply(c, true, tags, &changed, undo);
    if (!rc && (stop || changed)) rc = undo();
    if (!rc && changed) {
      rc = launch_estimate_dt(c, c->md["base"], true);
      if (!rc) rc = launch_dt_controller(c, 3);
      if (!rc) rc = read_clock(c, h, "evolve remesh");
    }
    if (rc) {
      undo();
      break;
    }
    if (!stop && !changed) {
      // the speculative step stands and becomes the current one
      cur = 1 - cur;
      continue;
    }
    if (rc || stop || h.status) break;
    if (!rc) rc = pipe_reserve(c);
    if (!rc) rc = enqueue(cur, false);
  }
  // nothing stays in flight
  const int r = cuda_check(c, cudaStreamSynchronize(c->stream), "pipeline end");
  if (!rc) rc = r;
  *n_out = n;
  return rc;
}

int kmy_evolve(kmy_ctx *c, double tlim, int nlim, int *nsteps) {
  if (!c) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  c->prm.tp.tlim = tlim;
  int rc = launch_dt_controller(c, 2);  // clamp the pending dt to tlim
  int n = 0;
  DevClock h{};
  // device time: from before each iteration's steps to after their last
  // kernel (the host's read-back and tree update excluded)
  for (cudaEvent_t &e : c->ev_evolve)
    if (!rc && !e) rc = cuda_check(c, cudaEventCreate(&e), "evolve event");
  c->evolve_device_ms = 0.0;
  if (!rc && c->amr.on) {
    if (nlim != 0) {
      rc = evolve_amr(c, nlim, &n, h);
    } else {
      rc = read_clock(c, h, "evolve");
    }
    if (!rc && h.status) rc = clock_status(c, h.status);
    if (nsteps) *nsteps = h.ncycle;
    return rc;
  }
  while (!rc) {
    rc = cuda_check(c, cudaEventRecord(c->ev_evolve[0], c->stream), "evolve event");
    if (rc) break;

    // Fused hydro steps queue ahead in chunks: a step queued after the clock
    // reached tlim leaves the state unchanged.  The per-task kernels (the
    // tasks path, and the primitives of a constrained-transport stage) do
    // not check the clock, so those step one at a time.  Adaptive meshes run
    // evolve_amr above.
    const int chunk = steps_fused(c) && !c->prm.mhd ? kChunk : 1;
    bool ran = false;
    if (chunk == kChunk && (nlim < 0 || nlim - n >= kChunk)) {
      rc = graph_run(c, [&] {
        int r = KMY_OK;
        for (int i = 0; i < kChunk && !r; i++) r = step_async(c);
        return r;
      }, &ran);
      if (ran) n += kChunk;
    }
    for (int i = 0; !ran && i < chunk && !rc && (nlim < 0 || n < nlim); i++, n++) rc = step_async(c);
    if (!rc) rc = cuda_check(c, cudaEventRecord(c->ev_evolve[1], c->stream), "evolve event");
    if (rc) break;
    rc = read_clock(c, h, "evolve");
    if (rc) break;
    float ms = 0.f;
    rc = cuda_check(c, cudaEventElapsedTime(&ms, c->ev_evolve[0], c->ev_evolve[1]), "evolve event");
    if (rc) break;
    c->evolve_device_ms += double(ms);
    if (h.status) {
      rc = clock_status(c, h.status);
      break;
    }
    if (h.done || (nlim >= 0 && n >= nlim)) break;
  }
  if (nsteps) *nsteps = h.ncycle;
  return rc;
}

int kmy_end_step(kmy_ctx *c) {
  if (!c) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  return finish_step(c, interior_cells(c));
}

int kmy_get_blocks(const kmy_ctx *c, int *levels, int *locations, int max_blocks, int *nblocks) {
  if (!c) return KMY_ERR_BAD_PARAM;
  const MeshDesc &m = c->m;
  if (nblocks) *nblocks = m.nb;
  for (int b = 0; b < m.nb && b < max_blocks; b++) {
    if (levels) levels[b] = c->amr.on ? c->amr.lev[b] : 0;
    for (int d = 0; d < 3 && locations; d++) locations[3 * b + d] = c->amr.on ? c->amr.loc[3 * b + d] : blk_loc(m, b, d);
  }
  return KMY_OK;
}

int kmy_get_time(const kmy_ctx *c, double *time, double *dt, double *dt_est, int *ncycle) {
  if (!c) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  DevClock h;
  cudaError_t e = cudaMemcpyAsync(&h, c->clock, sizeof(h), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return KMY_ERR_CUDA;
  if (time) *time = h.time;
  if (dt) *dt = h.dt;
  if (dt_est) *dt_est = h.dt_est;
  if (ncycle) *ncycle = h.ncycle;
  return KMY_OK;
}

int kmy_zone_cycles(const kmy_ctx *c, int64_t *out) {
  if (!c || !out) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  DevClock h;
  cudaError_t e = cudaMemcpyAsync(&h, c->clock, sizeof(h), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return KMY_ERR_CUDA;
  *out = int64_t(h.zone_cycles);
  return KMY_OK;
}

int kmy_set_dt(kmy_ctx *c, double dt) {
  if (!c || !(dt > 0)) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  int rc = cuda_check(c, cudaMemcpyAsync(&c->clock->dt, &dt, 8, cudaMemcpyHostToDevice, c->stream), "dt");
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "dt");
  return rc;
}

int kmy_set_path(kmy_ctx *c, int path) {
  if (!c || (path != 0 && path != 1)) return KMY_ERR_BAD_PARAM;
  c->path = path;
  return KMY_OK;
}

int kmy_vortex_error(kmy_ctx *c, int var, int comp, double *out) {
  if (!c || !out || var < 0 || var > 3 || (var == 3 && !c->prm.mhd)) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  int rc = materialize(c);
  if (!rc) rc = launch_vortex_error(c, var, comp, out);
  return rc;
}

int kmy_conserved_sums(kmy_ctx *c, const char *md, double *out) {
  if (!c || !out) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  KMY_CONTAINER(a, md);
  return launch_conserved_sums(c, *a, out);
}

static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int kmy_bind_container(kmy_ctx *c, const char *container, void *cons, size_t cons_bytes, void *ener_lo,
                       size_t ener_lo_bytes, void *mag, size_t mag_bytes) {
  if (!c || !container || !cons) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  if (c->amr.on) {
    c->err = "an adaptive mesh reallocates its containers when it remeshes; bind a single-level mesh";
    return KMY_ERR_BAD_PARAM;
  }
  const size_t n = size_t(c->m.nb) * c->m.P, nf = size_t(c->m.nb) * c->m.Pf;
  const size_t want_cc = c->esz * c->ncc * n, want_lo = c->esz == 4 ? 4 * n : 0,
               want_mag = c->prm.mhd ? c->esz * 3 * nf : 0;
  if (cons_bytes != want_cc || ener_lo_bytes != (ener_lo ? want_lo : 0) || (want_lo && !ener_lo) ||
      mag_bytes != (mag ? want_mag : 0) || (want_mag && !mag)) {
    c->err = "bind sizes: conserved " + std::to_string(want_cc) + " bytes, energy low words " +
             std::to_string(want_lo) + ", face field " + std::to_string(want_mag);
    return KMY_ERR_BAD_PARAM;
  }
  if (!aligned16(cons) || (ener_lo && !aligned16(ener_lo)) || (mag && !aligned16(mag))) {
    c->err = "bound arrays must start on a 16-byte boundary";
    return KMY_ERR_BAD_PARAM;
  }
  Container *ct = find_container(c, container);
  if (!ct) return KMY_ERR_BAD_PARAM;
  // the context's own arrays for this container go back to the pool
  if (!ct->bound) {
    dfree(c, ct->cc);
    dfree(c, ct->ener_lo);
    dfree(c, ct->fc);
  }
  ct->cc = cons;
  ct->ener_lo = ener_lo;
  if (c->prm.mhd) ct->fc = mag;
  ct->bound = true;
  ct->ghosts = false;
  c->prims_valid = false;
  c->prims_interior = false;
  if (c->evolve_exec) {
    cudaGraphExecDestroy(c->evolve_exec);
    c->evolve_exec = nullptr;
  }
  return KMY_OK;
}

int kmy_bind_primitives(kmy_ctx *c, void *prim, size_t bytes) {
  if (!c || !prim) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  const size_t want = c->esz * NPRIM * size_t(c->m.nb) * c->m.P;
  if (c->amr.on || bytes != want || !aligned16(prim)) {
    c->err = "bind primitives: " + std::to_string(want) + " bytes, 16-byte aligned, single-level mesh";
    return KMY_ERR_BAD_PARAM;
  }
  if (!c->prim_bound) dfree(c, c->prim);
  c->prim = prim;
  c->prim_bound = true;
  c->prims_valid = false;
  c->prims_interior = false;
  return KMY_OK;
}

int kmy_set_fault(kmy_ctx *c, const char *what, int value) {
  if (!c || !what) return KMY_ERR_BAD_PARAM;
  if (std::string(what) == "stage_wait") {
    if (slab_unsupported(c)) {
      c->err = "stage_wait applies to the z-streamed stage";
      return KMY_ERR_BAD_PARAM;
    }
    c->fault_wait = value ? 1 : 0;
    return KMY_OK;
  }
  c->err = std::string("unknown fault ") + what;
  return KMY_ERR_BAD_PARAM;
}

int kmy_evolve_device_ms(const kmy_ctx *c, double *ms) {
  if (!c || !ms) return KMY_ERR_BAD_PARAM;
  *ms = c->evolve_device_ms;
  return KMY_OK;
}

int kmy_graph_replays(const kmy_ctx *c, int64_t *out) {
  if (!c || !out) return KMY_ERR_BAD_PARAM;
  *out = c->graph_replays;
  return KMY_OK;
}

int kmy_launch_count(const kmy_ctx *c, int64_t *out) {
  if (!c || !out) return KMY_ERR_BAD_PARAM;
  *out = c->launches;
  return KMY_OK;
}

}  // extern "C"
