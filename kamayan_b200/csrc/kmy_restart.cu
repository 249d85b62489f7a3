// kmy_restart.cu -- restart files: a snapshot of a context's device state
// that a new context resumes from bit for bit.
//
// The reference writes Parthenon restart outputs (`file_type = rst`,
// src/problems/isentropic_vortex.in:40-43) holding every variable flagged
// Metadata::Restart (src/kamayan/fields.hpp:160-161) and reads them back with
// `-r`.  Here the snapshot holds what a step reads from its input: the "base"
// container as stored (FP32 keeps its energy low words), the shared
// primitives, the face field and div B with CT, the device clock and time
// parameters, and on an adaptive mesh the leaf list with its derefinement
// counters.  Stage containers, fluxes and EMFs are rebuilt by every step and
// are not saved.  The file carries the deck, so a restart needs nothing else.
//
// Layout (native byte order): magic "KMYRST02", then int32 fields, int64
// sizes, the deck text, the leaf list, raw structs, raw device arrays.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/kmy_hydro.h"
#include "kmy_internal.hpp"

using kmy::Container;

namespace {

constexpr char kMagic[8] = {'K', 'M', 'Y', 'R', 'S', 'T', '0', '2'};
constexpr size_t kChunk = size_t(64) << 20;  // device <-> file staging chunk

struct Header {
  int32_t esz, ncc, mhd, ndim, nb, amr;
  int64_t P, Pf;
  int32_t prims_valid, prims_interior, path, pad;
};

struct File {
  std::FILE *f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

int put(kmy_ctx *c, std::FILE *f, const void *p, size_t n) {
  if (n && std::fwrite(p, 1, n, f) != n) {
    c->err = "restart: write failed";
    return KMY_ERR_STATE;
  }
  return KMY_OK;
}
int get(kmy_ctx *c, std::FILE *f, void *p, size_t n) {
  if (n && std::fread(p, 1, n, f) != n) {
    c->err = "restart: file is truncated";
    return KMY_ERR_STATE;
  }
  return KMY_OK;
}

// Device array -> file and file -> device array, in chunks through host memory.
int save_array(kmy_ctx *c, std::FILE *f, const void *dev, size_t bytes) {
  std::vector<char> h(bytes < kChunk ? bytes : kChunk);
  for (size_t o = 0; o < bytes; o += kChunk) {
    const size_t n = bytes - o < kChunk ? bytes - o : kChunk;
    int rc = kmy::cuda_check(c, cudaMemcpyAsync(h.data(), static_cast<const char *>(dev) + o, n,
                                                cudaMemcpyDeviceToHost, c->stream), "restart read");
    if (!rc) rc = kmy::cuda_check(c, cudaStreamSynchronize(c->stream), "restart read sync");
    if (!rc) rc = put(c, f, h.data(), n);
    if (rc) return rc;
  }
  return KMY_OK;
}
int load_array(kmy_ctx *c, std::FILE *f, void *dev, size_t bytes) {
  std::vector<char> h(bytes < kChunk ? bytes : kChunk);
  for (size_t o = 0; o < bytes; o += kChunk) {
    const size_t n = bytes - o < kChunk ? bytes - o : kChunk;
    int rc = get(c, f, h.data(), n);
    if (!rc)
      rc = kmy::cuda_check(c, cudaMemcpyAsync(static_cast<char *>(dev) + o, h.data(), n, cudaMemcpyHostToDevice,
                                              c->stream), "restart write");
    if (!rc) rc = kmy::cuda_check(c, cudaStreamSynchronize(c->stream), "restart write sync");
    if (rc) return rc;
  }
  return KMY_OK;
}

}  // namespace

extern "C" {

int kmy_save_restart(kmy_ctx *c, const char *path) {
  if (!c || !path) return KMY_ERR_BAD_PARAM;
  cudaSetDevice(c->device);
  int rc = kmy::cuda_check(c, cudaStreamSynchronize(c->stream), "restart sync");
  if (rc) return rc;
  File out;
  out.f = std::fopen(path, "wb");
  if (!out.f) {
    c->err = std::string("restart: cannot open ") + path + " for writing";
    return KMY_ERR_BAD_PARAM;
  }
  const kmy::MeshDesc &m = c->m;
  Header h{};
  h.esz = int32_t(c->esz);
  h.ncc = c->ncc;
  h.mhd = c->prm.mhd ? 1 : 0;
  h.ndim = m.ndim;
  h.nb = m.nb;
  h.amr = c->amr.on ? 1 : 0;
  h.P = m.P;
  h.Pf = m.Pf;
  h.prims_valid = c->prims_valid ? 1 : 0;
  h.prims_interior = c->prims_interior ? 1 : 0;
  h.path = c->path;
  const int64_t deck_len = int64_t(c->deck_text.size());
  rc = put(c, out.f, kMagic, sizeof(kMagic));
  if (!rc) rc = put(c, out.f, &h, sizeof(h));
  if (!rc) rc = put(c, out.f, &deck_len, sizeof(deck_len));
  if (!rc) rc = put(c, out.f, c->deck_text.data(), c->deck_text.size());
  if (!rc && h.amr) {
    rc = put(c, out.f, c->amr.lev.data(), sizeof(int) * m.nb);
    if (!rc) rc = put(c, out.f, c->amr.loc.data(), sizeof(int) * 3 * m.nb);
    if (!rc) rc = put(c, out.f, c->amr.cnt.data(), sizeof(int) * m.nb);
  }
  kmy::DevClock clk;
  if (!rc) rc = kmy::cuda_check(c, cudaMemcpy(&clk, c->clock, sizeof(clk), cudaMemcpyDeviceToHost), "restart clock");
  if (!rc) rc = put(c, out.f, &clk, sizeof(clk));
  if (!rc) rc = put(c, out.f, &c->prm.tp, sizeof(c->prm.tp));
  const size_t n = size_t(m.nb) * m.P, nf = size_t(m.nb) * m.Pf;
  Container &b = c->md["base"];
  if (!rc) rc = save_array(c, out.f, b.cc, c->esz * c->ncc * n);
  if (!rc && c->esz == 4) rc = save_array(c, out.f, b.ener_lo, 4 * n);
  if (!rc) rc = save_array(c, out.f, c->prim, c->esz * kmy::NPRIM * n);
  if (!rc && c->prm.mhd) rc = save_array(c, out.f, b.fc, c->esz * 3 * nf);
  if (!rc && c->prm.mhd) rc = save_array(c, out.f, c->divb, 8 * n);
  if (!rc && std::fflush(out.f) != 0) {
    c->err = "restart: write failed";
    rc = KMY_ERR_STATE;
  }
  return rc;
}

int kmy_load_restart(const char *path, int device, kmy_ctx **out) {
  if (!path || !out) return KMY_ERR_BAD_PARAM;
  *out = nullptr;
  File in;
  in.f = std::fopen(path, "rb");
  if (!in.f) {
    std::fprintf(stderr, "kmy_load_restart: cannot open %s\n", path);
    return KMY_ERR_BAD_PARAM;
  }
  char magic[8];
  Header h{};
  int64_t deck_len = 0;
  if (std::fread(magic, 1, 8, in.f) != 8 || std::memcmp(magic, kMagic, 8) != 0 ||
      std::fread(&h, 1, sizeof(h), in.f) != sizeof(h) || std::fread(&deck_len, 1, 8, in.f) != 8 || deck_len < 0 ||
      deck_len > (int64_t(1) << 30)) {
    std::fprintf(stderr, "kmy_load_restart: %s is not a restart file of this library\n", path);
    return KMY_ERR_STATE;
  }
  std::string deck(size_t(deck_len), '\0');
  if (std::fread(&deck[0], 1, size_t(deck_len), in.f) != size_t(deck_len)) {
    std::fprintf(stderr, "kmy_load_restart: %s is truncated\n", path);
    return KMY_ERR_STATE;
  }
  kmy_ctx *c = nullptr;
  int rc = kmy_create(deck.c_str(), device, &c);
  if (rc) return rc;
  const kmy::MeshDesc &m = c->m;
  if (h.esz != int32_t(c->esz) || h.ncc != c->ncc || h.mhd != (c->prm.mhd ? 1 : 0) || h.ndim != m.ndim ||
      h.P != m.P || h.Pf != m.Pf || h.amr != (c->amr.on ? 1 : 0) || h.nb <= 0 || (!h.amr && h.nb != m.nb)) {
    std::fprintf(stderr, "kmy_load_restart: %s does not match the mesh its deck describes\n", path);
    kmy_destroy(c);
    return KMY_ERR_STATE;
  }
  if (h.amr) {
    kmy::AmrHost &a = c->amr;
    a.lev.resize(h.nb);
    a.loc.resize(size_t(3) * h.nb);
    a.cnt.resize(h.nb);
    rc = get(c, in.f, a.lev.data(), sizeof(int) * h.nb);
    if (!rc) rc = get(c, in.f, a.loc.data(), sizeof(int) * 3 * h.nb);
    if (!rc) rc = get(c, in.f, a.cnt.data(), sizeof(int) * h.nb);
    for (int b = 0; b < h.nb && !rc; b++) {
      bool ok = a.lev[b] >= 0 && a.lev[b] <= a.max_level;
      for (int d = 0; d < 3 && ok; d++) {
        const int lim = d < m.ndim ? (m.nbx[d] << a.lev[b]) : 1;
        ok = a.loc[3 * b + d] >= 0 && a.loc[3 * b + d] < lim;
      }
      if (!ok) {
        c->err = "restart: leaf level or location out of range";
        rc = KMY_ERR_STATE;
      }
    }
    if (!rc) rc = kmy::amr_adopt_leaves(c);
  }
  kmy::DevClock clk;
  if (!rc) rc = get(c, in.f, &clk, sizeof(clk));
  if (!rc) rc = get(c, in.f, &c->prm.tp, sizeof(c->prm.tp));
  if (!rc) rc = kmy::cuda_check(c, cudaMemcpyAsync(c->clock, &clk, sizeof(clk), cudaMemcpyHostToDevice, c->stream),
                                "restart clock");
  const size_t n = size_t(c->m.nb) * c->m.P, nf = size_t(c->m.nb) * c->m.Pf;
  Container &b = c->md["base"];
  b.ghosts = false;
  if (!rc) rc = load_array(c, in.f, b.cc, c->esz * c->ncc * n);
  if (!rc && c->esz == 4) rc = load_array(c, in.f, b.ener_lo, 4 * n);
  if (!rc) rc = load_array(c, in.f, c->prim, c->esz * kmy::NPRIM * n);
  if (!rc && c->prm.mhd) rc = load_array(c, in.f, b.fc, c->esz * 3 * nf);
  if (!rc && c->prm.mhd) rc = load_array(c, in.f, c->divb, 8 * n);
  if (rc) {
    std::fprintf(stderr, "kmy_load_restart: %s\n", c->err.c_str());
    kmy_destroy(c);
    return rc;
  }
  c->prims_valid = h.prims_valid != 0;
  c->prims_interior = h.prims_interior != 0;
  c->path = h.path;
  *out = c;
  return KMY_OK;
}

}  // extern "C"
