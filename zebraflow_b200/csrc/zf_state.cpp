// Exact checkpoints of a context's time-stepping state.
//
// The reference restarts from its CSV snapshots: moments printed with eight
// significant digits and populations rebuilt as feq(D, u) (ZebraflowWT.c:
// 2649-2700, :5253-5295), so a restarted run leaves the trajectory it came
// from.  zf_save_state writes the state the next step reads -- the current
// population buffer in its storage form, BODYFORCE, the stored moments, the
// cells' fp64 positions and velocities, forces, repulsion increments,
// statuses and counters, the nucleus-membrane lists and the iteration count
// (which also seeds the stochastic rounding) -- as raw bytes, and
// zf_load_state puts it back into a context set up with the same lattice,
// storage form, mesh and number of cells, so that a run continued from a
// checkpoint is the run that wrote it.
#include <cstdio>
#include <cstring>
#include <vector>

#include "zf_internal.h"

using namespace zf;

namespace {

constexpr char kMagic[8] = {'Z', 'F', 'S', 'T', 'A', 'T', 'E', '1'};

struct Header {
  int64_t version, nx, ny, nz, storage, ns, n_listed, n_cells, nn, nnn, nuc_cap, nuc_valid;
  zf_status status;
};

struct Blob {
  void* dev;
  size_t bytes;
};

size_t pop_bytes(const zf_ctx* c) {
  const size_t e = (c->p.storage == ZF_STORE_F16 || c->p.storage == ZF_STORE_BF16) ? 2 : 4;
  return (size_t)ZF_Q * (size_t)c->ns * e;
}

// the device buffers of the state, in file order
std::vector<Blob> blobs(zf_ctx* c) {
  std::vector<Blob> b = {{c->d_f[c->cur], pop_bytes(c)},
                         {c->d_force, 3 * (size_t)c->ns * sizeof(float)},
                         {c->d_mom, 4 * (size_t)c->ns * sizeof(float)}};
  if (c->cells_set && c->cells.n_cells > 0) {
    const CellArgs& a = c->cells;
    const size_t nc = (size_t)a.n_cells, m = 3 * nc * a.nn, mn = 3 * nc * a.nnn;
    b.push_back({a.x, m * sizeof(double)});
    b.push_back({a.xn, mn * sizeof(double)});
    b.push_back({a.vel, m * sizeof(double)});
    b.push_back({a.vel_n, mn * sizeof(double)});
    b.push_back({a.ftot, m * sizeof(float)});
    b.push_back({a.ftot_n, mn * sizeof(float)});
    b.push_back({a.wrep, m * sizeof(float)});
    b.push_back({a.wrep_n, mn * sizeof(float)});
    b.push_back({a.status, nc * sizeof(int32_t)});
    b.push_back({a.caps_remove, nc * sizeof(int32_t)});
    b.push_back({a.counters, 4 * sizeof(unsigned long long)});
    if (!c->ib_allocs.empty()) {
      const size_t nnuc = nc * a.nnn;
      b.push_back({c->ib.nuc_list, nnuc * (size_t)c->ib.nuc_cap * sizeof(uint16_t)});
      b.push_back({c->ib.nuc_cnt, nnuc * sizeof(int32_t)});
    }
  }
  return b;
}

Header header_of(zf_ctx* c) {
  Header h{};
  h.version = 1;
  h.nx = c->p.nx;
  h.ny = c->p.ny;
  h.nz = c->p.nz;
  h.storage = c->p.storage;
  h.ns = c->ns;
  h.n_listed = c->n_listed;
  const bool cells = c->cells_set && c->cells.n_cells > 0;
  h.n_cells = cells ? c->cells.n_cells : 0;
  h.nn = cells ? c->cells.nn : 0;
  h.nnn = cells ? c->cells.nnn : 0;
  h.nuc_cap = cells && !c->ib_allocs.empty() ? c->ib.nuc_cap : 0;
  h.nuc_valid = c->nuc_lists_valid;
  h.status = c->status;
  return h;
}

}  // namespace

extern "C" {

int zf_save_state(zf_ctx* c, const char* path) {
  if (!c || !path) return ZF_ERR_ARG;
  if (!c->lattice_set) {
    set_error("zf_save_state: lattice not set");
    return ZF_ERR_STATE;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  if (c->cells_set && c->cells.n_cells > 0 && c->ib_allocs.empty()) {
    const int rc = ib_prepare(c);  // so that the nucleus lists have a home
    if (rc) return rc;
  }
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error("zf_save_state: cannot write %s", path);
    return ZF_ERR_ARG;
  }
  const Header h = header_of(c);
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(&h, sizeof h, 1, f) == 1;
  std::vector<char> host;
  for (const Blob& b : blobs(c)) {
    if (!ok) break;
    host.resize(b.bytes);
    const cudaError_t e = cudaMemcpy(host.data(), b.dev, b.bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      std::fclose(f);
      set_error("zf_save_state: %s", cudaGetErrorString(e));
      return ZF_ERR_CUDA;
    }
    const int64_t n = (int64_t)b.bytes;
    ok = std::fwrite(&n, sizeof n, 1, f) == 1 && std::fwrite(host.data(), 1, b.bytes, f) == b.bytes;
  }
  if (std::fclose(f) != 0) ok = false;
  if (!ok) {
    set_error("zf_save_state: write error on %s", path);
    return ZF_ERR_ARG;
  }
  return ZF_OK;
}

int zf_load_state(zf_ctx* c, const char* path) {
  if (!c || !path) return ZF_ERR_ARG;
  if (!c->lattice_set) {
    set_error("zf_load_state: lattice not set");
    return ZF_ERR_STATE;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  if (c->cells_set && c->cells.n_cells > 0 && c->ib_allocs.empty()) {
    const int rc = ib_prepare(c);
    if (rc) return rc;
  }
  {
    const int rc = cells_copy_wait_host(c);  // the cell buffers are about to be overwritten
    if (rc) return rc;
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("zf_load_state: cannot open %s", path);
    return ZF_ERR_ARG;
  }
  char magic[8];
  Header h{};
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kMagic, 8) != 0 || std::fread(&h, sizeof h, 1, f) != 1) {
    std::fclose(f);
    set_error("zf_load_state: %s is not a state file", path);
    return ZF_ERR_ARG;
  }
  const Header mine = header_of(c);
  if (h.version != 1 || h.nx != mine.nx || h.ny != mine.ny || h.nz != mine.nz || h.storage != mine.storage ||
      h.ns != mine.ns || h.n_listed != mine.n_listed || h.n_cells != mine.n_cells || h.nn != mine.nn ||
      h.nnn != mine.nnn || h.nuc_cap != mine.nuc_cap) {
    std::fclose(f);
    set_error("zf_load_state: %s was written by a context with another lattice, storage form, mesh or "
              "cell count (file: %lldx%lldx%lld, storage %lld, %lld listed, %lld cells)",
              path, (long long)h.nx, (long long)h.ny, (long long)h.nz, (long long)h.storage,
              (long long)h.n_listed, (long long)h.n_cells);
    return ZF_ERR_ARG;
  }
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  std::vector<char> host;
  for (const Blob& b : blobs(c)) {
    int64_t n = 0;
    host.resize(b.bytes);
    if (std::fread(&n, sizeof n, 1, f) != 1 || n != (int64_t)b.bytes || std::fread(host.data(), 1, b.bytes, f) != b.bytes) {
      std::fclose(f);
      set_error("zf_load_state: %s is truncated or does not match this context", path);
      return ZF_ERR_ARG;
    }
    const cudaError_t e = cudaMemcpy(b.dev, host.data(), b.bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      std::fclose(f);
      set_error("zf_load_state: %s", cudaGetErrorString(e));
      return ZF_ERR_CUDA;
    }
  }
  const bool trailing = std::fgetc(f) != EOF;
  std::fclose(f);
  if (trailing) {
    set_error("zf_load_state: %s has trailing data", path);
    return ZF_ERR_ARG;
  }
  c->status = h.status;
  c->nuc_lists_valid = h.nuc_valid != 0;
  c->node_tiles_valid = false;
  return ZF_OK;
}

}  // extern "C"
