// Internal declarations shared by the host setup (zf_host.cpp) and the CUDA
// kernels (zf_lbm.cu, zf_cells.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/zf.h"

// Tile geometry of the sparse lattice: 4x4x4 lattice points, x fastest.
#define ZF_TS 4
#define ZF_TC 64
// Populations are stored tile-major, [tile][19][64]: the 19 planes of one
// tile are contiguous (ZF_PT elements), so the offset of population q inside
// a tile is the constant q*64.  Point slot s = tile*64 + cell.
#define ZF_PT (19 * ZF_TC)
__host__ __device__ __forceinline__ int64_t pop_at(int q, int64_t s) {
  return (s >> 6) * ZF_PT + (int64_t)q * ZF_TC + (s & 63);
}

// Cell codes stored per tile slot (uint8).
enum : uint8_t {
  ZF_CODE_SOLID = 0,      // not listed (reference B_index < 0)
  // 1..9: fluid of that phase (reference B_index 1..9)
  ZF_CODE_WALL = 10,      // listed wall point (reference B_index == 0)
  ZF_CODE_PRESSURE0 = 100 // 101..109: pressure inlet/outlet of reference code 1001..1009
};
// fluid points (collided), and the points the IB coupling treats as fluid
// (reference 0 < B_index < 4998: fluid and pressure inlets/outlets)
__host__ __device__ __forceinline__ bool zf_code_fluid(uint8_t cd) { return cd >= 1 && cd <= 9; }
__host__ __device__ __forceinline__ bool zf_code_pressure(uint8_t cd) {
  return cd > ZF_CODE_PRESSURE0 && cd < ZF_CODE_PRESSURE0 + 10;
}

namespace zf {

// membrane-iteration stages timed by zf_profile (see zf_profile_stages)
constexpr int ZF_PROF_STAGES = 8;
constexpr int ZF_PROF_MARKS = ZF_PROF_STAGES + 1;

void set_error(const char* fmt, ...);

#define ZF_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      ::zf::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),  \
                      __FILE__, __LINE__);                                     \
      return ZF_ERR_CUDA;                                                      \
    }                                                                          \
  } while (0)

// Device-side view of the tiled lattice, passed by value to kernels.
struct LatticeView {
  int ntx, nty, ntz;          // tile grid
  int nx, ny, nz;             // lattice box
  int per_x, per_y, per_z;    // periodic flags
  int64_t ns;                 // slots per population plane (= n_pop_tiles*64)
  const int32_t* tile_map;    // [ntx*nty*ntz] tile id or -1 (all tiles)
  const uint8_t* code;        // [n_all_tiles*64]
};

struct LbmArgs {
  const void* fin;
  void* fout;
  const int32_t* active;      // tiles with >= 1 fluid point
  int n_active;
  const int32_t* nbr;         // [n_pop_tiles][27] neighbour tile ids (-1 none)
  const uint32_t* link;       // [ns] bit q: pull along q bounces back; bit 31: fluid point
  const uint8_t* code;        // [n_pop_tiles*64]
  float* force;               // [3][ns] BODYFORCE (reference units)
  float* mom;                 // [4][ns] D,U,V,W
  float* rho_pre;             // [ns] pre-collision density (wall-equilibrium mode)
  float* u_pre;               // [3][ns] pre-collision velocity (lattices with pressure points)
  int64_t iter_now;           // the iteration this step computes (pressure waveforms)
  double dt_us;               // time step, us (the reference's DT; T_SCALE = DT 1e-6 s)
  int64_t ns;
  float tau;
  float force_dt;             // multiplier of BODYFORCE in the Guo step (reference DT)
  float gx, gy, gz;           // uniform effective force
  float rho_ref, scale, inv_scale;
  double* mass_partial;       // per-block FP64 density sums, or nullptr
  uint32_t step;              // step counter (seeds the stochastic rounding)
  int store_moments, zero_force, tau_from_phase, write_rho_pre, write_u_pre, stochastic;
};

// Device view of the cells (membrane + nucleus meshes shared by every cell).
// Layouts follow the reference: [3][cells][nodes] for vectors, [cells][n]
// for scalars; positions and node velocities are FP64, the rest FP32.
struct CellArgs {
  int n_cells, nn, nt, ne, nnn, nen;
  const int32_t* tri;        // [nt][3]
  const int32_t* edge;       // [ne][6] n1 n2 n3 n4 tri1 tri2
  const uint8_t* area_first; // [ne]
  const float* epar;         // [5][ne] LMAX, Plength, kp, sin(theta0), cos(theta0)
  const float* tri_area_eq;  // [nt]
  const int32_t* edge_n;     // [nen][2]
  const float* epar_n;       // [3][nen] LMAX, Plength, kp
  double* x;                 // [3][nc][nn] um
  double* xn;                // [3][nc][nnn]
  double* vel;               // [3][nc][nn] um/us
  double* vel_n;             // [3][nc][nnn]
  float* ftot;               // [3][nc][nn] N
  float* ftot_n;             // [3][nc][nnn]
  float* wrep;               // [3][nc][nn] velocity increments (NODE_WALLREPUL)
  float* wrep_n;             // [3][nc][nnn]
  float* node_normal;        // [3][nc][nn]
  float* tri_c;              // [3][nc][nt] um
  float* tri_nrm;            // [3][nc][nt]
  float* tri_a;              // [nc][nt] m^2
  float* cell_f;             // [nc][8] area, volume, centroid xyz, F_area_global, F_vol_scalar
  int32_t* status;           // [nc] 1 active, -5000 removed
  int32_t* caps_remove;      // [nc]
  unsigned long long* counters;  // [4] screened terms, cells removed, list overflows, spare
  float kT, kbend, kd, ka, kv;
  float area0, volume0;
  int remove_count;
};

int cells_membrane_launch(zf_ctx* c);
void cells_free(zf_ctx* c);

// Wall mesh on the host (reference WALLNODECOORD, WALLCELLNODE, WALLCELLNORMALS,
// WALL_CENTROID, WALLNODETOCELLNEIGHBORLIST, W_index, Wdistance, Uvoid).
struct VoidPoint {
  int64_t p;   // lattice point (dense index)
  float u[3];  // void velocity
};
struct WallHost {
  int nw = 0, mt = 0, cap = 0;
  std::vector<float> xyz;        // [3][nw]
  std::vector<int32_t> tri;      // [mt][3] 0-based
  std::vector<float> nrm, cen;   // [3][mt]
  std::vector<float> nnrm;       // [3][nw] area-weighted node normals (unit, into the lumen)
  std::vector<int32_t> ntri;     // [nw][cap+1]: count, triangles (0-based)
  std::vector<int32_t> cand_off; // [nw+1] candidates of each node's list ...
  std::vector<float4> cand;      // ... in list order: 3 vertices and the centroid of each
                                 // listed triangle (x, y, z, triangle id as int bits)
  std::vector<float> rad;        // [nw] farthest vertex or centroid of the node's listed
                                 // triangles from the node (um, rounded up)
  std::vector<int32_t> windex;   // [npts] 1-based wall node, 0 none
  std::vector<float> wdist;      // [npts]
  std::vector<VoidPoint> uvoid;  // non-zero void velocities
};
int wall_build(zf_ctx* c, int nw, const float* xyz, int mt, const int32_t* tri1, const float* nrm,
               WallHost& W);

// Device view used by the IB kernels.
struct IbArgs {
  int nx, ny, nz, ntx, nty, ntz;
  int per_z;
  int own_k0, own_k1;           // z planes [own_k0, own_k1) this context owns when the lattice is
                                // one slab of a split one (zf_set_ib_slab): interpolation and
                                // spreading use only those planes, the repulsions run only for
                                // nodes whose lattice index lies there; unbounded otherwise
  int kmin, kmax;               // z range of lattice points the coupling sees: the
                                // reference keeps 3 <= k <= KM-3 (1-based) in its region
                                // of interest; a periodic axis has no limit
  double X0, Y0, Z0, DX;        // um
  float LZ;                     // nz*DX when z is periodic, else 0
  const int32_t* tile_map;      // all tiles
  const uint8_t* code;          // [n_all*64]
  const uint8_t* tile_wall;     // [n_all] tile holds a point with W_index > 0
  const int32_t* windex;        // [n_all*64] 1-based wall node or 0
  const float4* wnode;          // [n_all*64] that wall node's position and bounding
                                // radius (WallHost::rad); w < 0 where W_index is 0
  const float* uvoid;           // [3][n_all*64]
  const float* mom;             // [4][ns] D,U,V,W of population tiles
  float* force;                 // [3][ns] BODYFORCE
  int64_t ns, ns_all;
  // wall mesh
  int nw, mt, wcap;
  const float* wxyz;            // [3][nw]
  const int32_t* wtri;          // [mt][3]
  const float* wnrm;            // [3][mt]
  const float* wnnrm;           // [3][nw] WallHost::nnrm
  const float* wcen;            // [3][mt]
  const int32_t* wntri;         // [nw][wcap+1]
  const float* wrad;            // [nw] WallHost::rad
  // per IB-view point: the wall nodes whose lists can hold the nearest wall
  // triangle of a node with that lattice index (k_wall_rel), as CSR; count
  // -1: too many, the node walks its window
  const int32_t* wrel_cnt;      // [n_all*64]
  const int32_t* wrel_off;      // [n_all*64 + 1]
  const int32_t* wrel;          // 1-based wall node ids
  int32_t* wall_walk;           // [n_cells*(nn+nnn)] nodes queued for the window walk (from the
                                // front) and for the warp scan of their wall-node lists (from the back)
  int32_t* wall_walk_ctr;       // [4] walk: queued count, work counter; lists: queued count, work counter
  int32_t* wall_tri;            // [n_cells*(nn+nnn)] the wall triangle of each node's repulsion, -1 none
  const int32_t* wcand_off;     // [nw+1] WallHost::cand_off
  const float4* wcand;          // WallHost::cand
  // cell list of triangle centroids over population slots (CSR).  Bin keys
  // order the points of a tile with z fastest (bin_key), so the bins of a
  // run of points along z are one contiguous range of entries.
  const int32_t* bin_off;       // [ns+1]
  const int32_t* bin_tri;       // [n_cells*nt] global triangle id = cell*nt + tri
  float4* bin_rec;              // [n_cells*nt][2] per entry, adjacent: centroid xyz and bounding
                                // radius (rec_pack); normal xyz and global triangle id (int bits)
  float4* bin_v;                // [3][n_cells*nt] per entry: vertex xyz (fp32), node id (int bits)
  uint8_t* bin_kk;              // [n_cells*nt] per entry: its key inside the tile (0..63)
  // membrane and nucleus nodes grouped by the lattice tile of their nearest
  // point (tile grid index over all ntx*nty*ntz tiles), rebuilt after positions change
  int64_t ngrid;                // ntx*nty*ntz
  int32_t* node_gt;             // [n_nodes] grid tile of node gid, -1 for removed cells
  int32_t* node_cnt;            // [ngrid+1] counts, then fill cursors
  int32_t* node_off;            // [ngrid+1] first sorted position of each grid tile
  int32_t* node_sorted;         // [n_nodes] node gids grouped by grid tile
  int32_t* tile_list;           // [min(ngrid, n_nodes)] grid tiles that hold nodes
  int32_t* tile_ctr;            // [4] listed tiles, work counters of the tile kernels
  int32_t* node_bsum;           // scan block sums
  // constants
  float vel_scale, gamma_p;
  double force_scale;           // 1/(UNITMASS*LBM_BFORCE_SCALE)
  double dt_stagger;            // DT * SOLVERSTAGGER
  float vmax_remove;
  int nuc_cap;
  uint16_t* nuc_list;           // [nc][nnn][nuc_cap]
  int32_t* nuc_cnt;             // [nc][nnn]
};

int ib_prepare(zf_ctx* c);
void ib_free(zf_ctx* c);
int ib_interp_launch(zf_ctx* c);
int ib_bins_launch(zf_ctx* c);
int ib_nuc_memb_launch(zf_ctx* c, int rebuild);
int ib_rbc_rbc_launch(zf_ctx* c);
int ib_node_tiles_launch(zf_ctx* c);
int ib_kin_buffer_launch(zf_ctx* c, double* buf, int dir);
int lbm_moments_launch(zf_ctx* c);
// adjoint building blocks
int lbm_adj_blocks(zf_ctx* c);
int lbm_adj_launch(zf_ctx* c, const void* f_pre, const float* lam, float* lam_prev, float* gF,
                   double* gw_partial);
// Stencils of a WSS objective's patch nodes over compact points (the distinct
// lattice slots the stencils read): node i owns entries off[i]..off[i+1]-1.
struct PatchStencil {
  int np = 0, nu = 0;
  const int32_t* patch = nullptr;  // [np] wall-node ids
  const int32_t* off = nullptr;    // [np+1]
  const int32_t* idx = nullptr;    // [entries] compact point of each entry
  const float* w = nullptr;        // [entries] Peskin weight
  const int32_t* uslot = nullptr;  // [nu] slot of each compact point
};
int wall_rel_build(zf_ctx* c, std::vector<void*>& own);
int wss_patch_stencil(zf_ctx* c, const float* d_nrm, const int32_t* d_patch, int np, PatchStencil& ps,
                      std::vector<std::pair<void*, size_t>>& bufs);
int wss_patch_launch(zf_ctx* c, const PatchStencil& ps, const float* d_nrm, const float* d_U, double w,
                     double* d_acc);
int wss_patch_adj_launch(zf_ctx* c, const PatchStencil& ps, const float* d_nrm, const float* d_U, double w,
                         float* d_gU);
// flux-split objective over compact points of two sets (set[u] = 0 or 1,
// unit normals n[0..2], n[3..5]): q[0..1] := sum_u U.n_set, then
// acc += w q0/(q0+q1); the adjoint writes gU = w d(q0/(q0+q1))/dU
int flux_objective_launch(zf_ctx* c, const PatchStencil& ps, const uint8_t* d_set, const float* nrm6,
                          const float* d_U, double w, double* d_q, double* d_acc);
int flux_adj_launch(zf_ctx* c, const PatchStencil& ps, const uint8_t* d_set, const float* nrm6,
                    const float* d_U, double w, double* d_q, float* d_gU);
// velocities U[3][nu] of the populations f at the compact points
int lbm_moments_at(zf_ctx* c, const void* f, const PatchStencil& ps, float* d_U);
// lam += seed of gU[3][nu] at the compact points (f: the state the objective
// read); clears gU
int lbm_seed_at(zf_ctx* c, const void* f, const PatchStencil& ps, float* d_gU, float* lam);
int lbm_step_buffers(zf_ctx* c, const void* fin, void* fout, uint32_t step);
// moments D, U, V, W of the populations f into the context's moment planes
int lbm_moments_of(zf_ctx* c, const void* f);
// the adjoint kernels of the cells (zf_adjoint_cells.cu):
// gx += lam^T dF/dx, gxn += lam_n^T dF/dxn, gpar[0..1] += lam^T dF/d(Es, kb)
// for the membrane and nucleus forces at the context's positions
int membrane_vjp_launch(zf_ctx* c, const float* lam, const float* lam_n, float* gx, float* gxn, double* gpar);
// transposed spreading of G (dJ/dBODYFORCE, or null), interpolation and
// position update (lam_x: adjoint of the updated positions, or null) at the
// context's positions: gF/gFn := adjoint of the spread node forces, gx/gxn +=
// position terms, GU[3][ns] += dJ/dU; ftot..wrep_n: the forces the forward spread
int ib_vjp_launch(zf_ctx* c, const float* G, const float* lam_x, const float* lam_xn, float* gx, float* gxn,
                  float* gF, float* gFn, float* GU, float* lam_w, const float* ftot, const float* ftot_n,
                  const float* wrep, const float* wrep_n);
// transposed repulsions at the context's positions: gx/gxn += lam_w^T
// d(wrep)/d(x, xn) of the wall (the triangles the last interpolation chose),
// nucleus-membrane (the current lists) and RBC-RBC repulsions (the current
// cell list); lam_w [3][nc][nn]: the adjoint of the membrane repulsion velocities
int repulsion_vjp_launch(zf_ctx* c, const float* lam_w, float* gx, float* gxn);
// y[0..n) += x[0..n)
int add_launch(zf_ctx* c, float* y, const float* x, int64_t n);
int spread_adj_launch(zf_ctx* c, const float* d_G, float* d_gmem, float* d_gnuc);
int scale_springs_launch(zf_ctx* c, float s);
int wss_launch(zf_ctx* c, const float* d_normals, double pgauge, float* d_wss, float* d_press,
               int32_t* d_valid);
int ib_spread_launch(zf_ctx* c);
int ib_update_launch(zf_ctx* c);
// before a kernel that writes cell positions or statuses: the context's stream
// waits for a pending zf_get_cells_async copy; cells_copy_wait_host waits on
// the host (before cell buffers are freed or replaced)
int cells_write_fence(zf_ctx* c);
int cells_copy_wait_host(zf_ctx* c);

}  // namespace zf

struct zf_ctx {
  zf_params p;
  int device = 0;
  cudaStream_t stream = nullptr;      // stream the context's work is queued on
  cudaStream_t own_stream = nullptr;  // created by zf_create
  // zf_get_cells_async: the copies run on copy_stream after ev_ready (the
  // context's stream); ev_copied marks their end, which the next kernel that
  // writes positions or statuses waits for (cells_write_fence)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_ready = nullptr, ev_copied = nullptr;
  bool copy_pending = false;
  bool lattice_set = false;

  // listed nodes (reference DOMLIST order)
  int64_t n_listed = 0, n_fluid = 0;
  std::vector<int32_t> domlist;   // [n_listed][3]
  std::vector<int32_t> b_index;   // dense copy of the input codes

  // tiles
  int ntx = 0, nty = 0, ntz = 0;
  int64_t n_pop_tiles = 0, n_all_tiles = 0;
  int n_active = 0;
  std::vector<int32_t> h_tile_map;     // host copy
  std::vector<int32_t> h_tile_origin;  // [n_all_tiles][3] tile coords
  int64_t ns = 0;

  int32_t* d_tile_map = nullptr;
  int32_t* d_active = nullptr;
  // z-slab stepping (zf_set_slab): the active tiles of the inner tile layers
  // [0] and of the two face layers next to the halo [1]; halo layers are not
  // stepped
  int32_t* d_active_part[2] = {nullptr, nullptr};
  int n_active_part[2] = {0, 0};
  bool slab_set = false;
  int32_t* d_nbr = nullptr;
  uint32_t* d_link = nullptr;
  uint8_t* d_code = nullptr;
  void* d_f[2] = {nullptr, nullptr};
  int cur = 0;
  float* d_force = nullptr;
  float* d_mom = nullptr;
  float* d_rho_pre = nullptr;
  float* d_u_pre = nullptr;       // [3][ns], only with pressure points
  int64_t n_pressure = 0;         // pressure inlet/outlet points (codes 1001..1009)
  int32_t* d_dom_slot = nullptr;  // [n_listed] slot of listed node l
  float* d_stage = nullptr;       // [19*n_listed] upload/download staging
  int32_t* d_wall_slot = nullptr; // REF mode wall points
  int32_t* d_wall_nbr = nullptr;  // designated neighbour slot (-1 none)
  int n_wall = 0;
  double* d_red = nullptr;        // reduction scratch
  int red_cap = 0;
  // listed points of single lattice planes z = k, in (x, y) order, for the
  // z-slab halo exchange (zf_plane_pack / zf_plane_unpack)
  struct PlaneSlots {
    int k, n;
    int32_t* d_slots;
  };
  std::vector<PlaneSlots> planes;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  zf_status status{};
  int64_t device_bytes = 0;

  // membrane mesh and cells
  bool mesh_set = false, cells_set = false;
  void* mesh_host = nullptr;       // zf::MeshHost*
  zf::CellArgs cells{};            // device pointers + sizes
  std::vector<void*> cell_allocs;  // device buffers owned for the cells
  std::vector<void*> mesh_allocs;  // device buffers owned for the mesh

  // wall mesh and the IB view of the lattice
  bool wall_set = false;
  zf::IbArgs ib{};
  std::vector<void*> wall_allocs;  // wall + aux-tile buffers
  std::vector<void*> ib_allocs;    // cell list + nucleus lists (sized with the cells)
  bool nuc_lists_valid = false;    // nucleus-membrane lists built since the cells were set
  bool node_tiles_valid = false;   // node-tile lists match the current positions
  int tile_blocks = 0;             // persistent grid of the tile kernels

  // adjoint: whether its forward moves the cells (zf_adjoint_cells), and the
  // gradient of the last such adjoint with respect to the starting positions
  bool adj_move_cells = false;

  // the IB slab of a split lattice (zf_set_ib_slab): owned planes, and the
  // period of z positions (0: none)
  bool ib_slab = false;
  int ib_k0 = 0, ib_k1 = 0;
  double ib_lz = 0.0;
  std::vector<float> adj_gx, adj_gxn;  // [3][nc][nn], [3][nc][nnn]

  // instrumentation: kernel launches, and optional event pairs around the LBM
  // kernel and the membrane block of zf_step
  int64_t launches = 0;
  bool profiling = false;
  std::vector<cudaEvent_t> prof_ev;  // [2*cap] LBM run pairs, then ZF_PROF_MARKS per membrane block
  int prof_cap = 0, prof_lbm = 0, prof_mem = 0;  // event pairs: LBM runs, membrane blocks
  bool prof_open = false;                          // an LBM run is being timed
  int prof_open_n = 0;                             // its launches so far
  std::vector<int> prof_run_n;                     // launches of each timed LBM run
};

namespace zf {
int lbm_launch(zf_ctx* c, int store_moments, int zero_force, double* mass_out = nullptr);
int lbm_launch_part(zf_ctx* c, int part, int finish, int store_moments = 0, int zero_force = 0);
int ensure_red(zf_ctx* c, int n);
int lbm_step_mass_noalloc(zf_ctx* c, int store_moments, int zero_force, double* mass_out);
int lbm_upload_populations(zf_ctx* c, const float* f);
int lbm_plane_slots(zf_ctx* c, int k, zf_ctx::PlaneSlots* out);
int lbm_plane_copy(zf_ctx* c, int k, int dir, void* buf, bool pack);
int lbm_download_populations(zf_ctx* c, float* f);
int lbm_init_equilibrium(zf_ctx* c);
int lbm_scatter_listed(zf_ctx* c, const float* h, int planes, float* d_dst);
int lbm_gather_listed(zf_ctx* c, const float* d_src, int planes, float* h);
int lbm_mass(zf_ctx* c, int include_walls, double* out);
int dev_alloc(zf_ctx* c, void** p, size_t bytes);
}  // namespace zf
