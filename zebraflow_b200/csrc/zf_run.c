/*
 * zf_run — the time loop of ZebraflowWT.c's main() (:5646-12412) as a C host
 * program over the C ABI of libzf.so (include/zf.h).
 *
 * The reference's main() reads its vessel, meshes and cells from files and
 * then runs, every iteration, the LBM blocks and, every SOLVERSTAGGER-th
 * iteration, the membrane, IB coupling, repulsion and position-update blocks.
 * This driver builds the inputs of a synthetic workload with the library's
 * generators (a straight tube or a periodic Y-bifurcation, its wall mesh,
 * icosphere membranes and nuclei placed from a seed), runs the loop through
 * zf_step in whole cycles of SOLVERSTAGGER iterations, reports throughput
 * from CUDA events, and writes the final state (node positions, cell status,
 * wall shear stress, fluid moments) as a binary dump (--out).  With
 * --output-every N it writes, at iteration 0 and every N iterations, the
 * files the reference's OUTPUT() writes (FLUIDdomain, AllCellMemb,
 * AllCellNucleus, AllNucEdgeMesh, VolumeAreaHistory; ZebraflowWT.c:282-509)
 * and the post-processor's Wallpressure VTK file (PostProWSSandPressure.c:
 * 375-433) into --output-dir.  --save-state / --load-state write and read an
 * exact checkpoint (zf_save_state) at the end / start of the run.
 *
 * usage: zf_run [--tube NX NY NZ R | --bifurcation NX NY NZ RP RD HALF_ANGLE]
 *               [--cells N] [--seed S] [--steps N] [--stagger S] [--tau T]
 *               [--g G] [--storage f32|f16|bf16|f32dev] [--device D]
 *               [--out FILE] [--output-every N] [--output-dir DIR]
 *               [--save-state FILE] [--load-state FILE]
 * Defaults: the 48x48x128 tube of radius 20 with 8 cells, 1000 iterations.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "zf.h"

#define AX_X 3.5 /* membrane semi-axes, um (7, 4.5, 2 lattice units) */
#define AX_Y 2.25
#define AX_Z 1.0
#define AXN_X 1.25 /* nucleus semi-axes, um (2.5, 1.8, 1.2 lattice units) */
#define AXN_Y 0.9
#define AXN_Z 0.6
#define DX_UM 0.5
#define MARGIN_UM 0.4 /* placement margin around each cell's ellipsoid */

static int check(int rc, const char* what) {
  if (rc != ZF_OK) {
    fprintf(stderr, "zf_run: %s failed (%d): %s\n", what, rc, zf_last_error());
    exit(1);
  }
  return rc;
}

static void* xmalloc(size_t n) {
  void* p = malloc(n ? n : 1);
  if (!p) {
    fprintf(stderr, "zf_run: out of host memory (%zu bytes)\n", n);
    exit(1);
  }
  return p;
}

static int cmp_edge(const void* a, const void* b) {
  const int32_t* x = (const int32_t*)a;
  const int32_t* y = (const int32_t*)b;
  if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
  return x[1] < y[1] ? -1 : (x[1] > y[1]);
}

/* unique edges of a triangle mesh, sorted by (min, max) node: [n][2] 1-based */
static int32_t* mesh_edges(const int32_t* tri, int n_tri, int* n_edge) {
  int32_t* e = (int32_t*)xmalloc(sizeof(int32_t) * 6 * (size_t)n_tri);
  for (int t = 0; t < n_tri; ++t)
    for (int v = 0; v < 3; ++v) {
      const int32_t a = tri[3 * t + v], b = tri[3 * t + (v + 1) % 3];
      e[2 * (3 * t + v)] = a < b ? a : b;
      e[2 * (3 * t + v) + 1] = a < b ? b : a;
    }
  qsort(e, 3 * (size_t)n_tri, 2 * sizeof(int32_t), cmp_edge);
  int n = 0;
  for (int i = 0; i < 3 * n_tri; ++i)
    if (n == 0 || e[2 * i] != e[2 * (n - 1)] || e[2 * i + 1] != e[2 * (n - 1) + 1]) {
      e[2 * n] = e[2 * i];
      e[2 * n + 1] = e[2 * i + 1];
      ++n;
    }
  *n_edge = n;
  return e;
}

typedef struct {
  int bifurcation;
  int nx, ny, nz;
  double R, Rp, Rd, half_angle;
  int cells;
  uint64_t seed;
  int steps, stagger;
  float tau, g;
  int storage, device;
  const char* out;
  int output_every;
  const char* output_dir;
  const char* save_state;
  const char* load_state;
} opts;

static void usage(void) {
  fprintf(stderr,
          "usage: zf_run [--tube NX NY NZ R | --bifurcation NX NY NZ RP RD HALF_ANGLE] [--cells N]\n"
          "              [--seed S] [--steps N] [--stagger S] [--tau T] [--g G]\n"
          "              [--storage f32|f16|bf16|f32dev] [--device D] [--out FILE]\n"
          "              [--output-every N] [--output-dir DIR] [--save-state FILE] [--load-state FILE]\n");
  exit(2);
}

static opts parse(int argc, char** argv) {
  opts o = {0,    48,   48, 128, 20.0, 0, 0, 20.0, 8, 1234, 1000, 50, 0.9f, 1e-6f, ZF_STORE_F32, 0, NULL, 0,
            "SimulationOutputData", NULL, NULL};
  for (int i = 1; i < argc; ++i) {
    const char* a = argv[i];
#define NEED(k) \
  if (i + (k) >= argc) usage();
    if (!strcmp(a, "--tube")) {
      NEED(4);
      o.bifurcation = 0;
      o.nx = atoi(argv[++i]);
      o.ny = atoi(argv[++i]);
      o.nz = atoi(argv[++i]);
      o.R = atof(argv[++i]);
    } else if (!strcmp(a, "--bifurcation")) {
      NEED(6);
      o.bifurcation = 1;
      o.nx = atoi(argv[++i]);
      o.ny = atoi(argv[++i]);
      o.nz = atoi(argv[++i]);
      o.Rp = atof(argv[++i]);
      o.Rd = atof(argv[++i]);
      o.half_angle = atof(argv[++i]);
    } else if (!strcmp(a, "--cells")) {
      NEED(1);
      o.cells = atoi(argv[++i]);
    } else if (!strcmp(a, "--seed")) {
      NEED(1);
      o.seed = strtoull(argv[++i], NULL, 10);
    } else if (!strcmp(a, "--steps")) {
      NEED(1);
      o.steps = atoi(argv[++i]);
    } else if (!strcmp(a, "--stagger")) {
      NEED(1);
      o.stagger = atoi(argv[++i]);
    } else if (!strcmp(a, "--tau")) {
      NEED(1);
      o.tau = (float)atof(argv[++i]);
    } else if (!strcmp(a, "--g")) {
      NEED(1);
      o.g = (float)atof(argv[++i]);
    } else if (!strcmp(a, "--storage")) {
      NEED(1);
      const char* s = argv[++i];
      if (!strcmp(s, "f32")) o.storage = ZF_STORE_F32;
      else if (!strcmp(s, "f16")) o.storage = ZF_STORE_F16;
      else if (!strcmp(s, "bf16")) o.storage = ZF_STORE_BF16;
      else if (!strcmp(s, "f32dev")) o.storage = ZF_STORE_F32_DEV;
      else usage();
    } else if (!strcmp(a, "--device")) {
      NEED(1);
      o.device = atoi(argv[++i]);
    } else if (!strcmp(a, "--out")) {
      NEED(1);
      o.out = argv[++i];
    } else if (!strcmp(a, "--output-every")) {
      NEED(1);
      o.output_every = atoi(argv[++i]);
    } else if (!strcmp(a, "--output-dir")) {
      NEED(1);
      o.output_dir = argv[++i];
    } else if (!strcmp(a, "--save-state")) {
      NEED(1);
      o.save_state = argv[++i];
    } else if (!strcmp(a, "--load-state")) {
      NEED(1);
      o.load_state = argv[++i];
    } else {
      usage();
    }
#undef NEED
  }
  if (o.nx <= 0 || o.ny <= 0 || o.nz <= 0 || o.cells < 0 || o.steps < 0 || o.stagger <= 0 || o.output_every < 0)
    usage();
  return o;
}

/* wall mesh of the vessel: sizes first, then the arrays */
static void wall_mesh(const opts* o, const double* origin, int* nw, int* mt, float** xyz, int32_t** tri,
                      float** nrm) {
  const double c = 0.5 * (o->nx - 1);
  int nseg = (int)lround(2 * 3.14159265358979 * o->R); /* one segment per lattice unit of circumference */
  if (nseg < 12) nseg = 12;
  for (int pass = 0; pass < 2; ++pass) {
    float* X = pass ? *xyz : NULL;
    int32_t* T = pass ? *tri : NULL;
    float* N = pass ? *nrm : NULL;
    if (o->bifurcation)
      check(zf_gen_wall_bifurcation(o->nx, o->ny, o->nz, o->Rp, o->Rd, o->half_angle, origin, DX_UM, nw, mt, X,
                                    T, N, pass ? *nw : 0, pass ? *mt : 0),
            "zf_gen_wall_bifurcation");
    else
      check(zf_gen_wall_tube(c, 0.5 * (o->ny - 1), o->R, o->nz, 1.0, nseg, origin, DX_UM, nw, mt, X, T, N,
                             pass ? *nw : 0, pass ? *mt : 0),
            "zf_gen_wall_tube");
    if (!pass) {
      *xyz = (float*)xmalloc(sizeof(float) * 3 * (size_t)*nw);
      *tri = (int32_t*)xmalloc(sizeof(int32_t) * 3 * (size_t)*mt);
      *nrm = (float*)xmalloc(sizeof(float) * 3 * (size_t)*mt);
    }
  }
}

/* the reference's output file name: DIR/NAME-<iteration, 9 digits>.EXT (:304-337) */
static const char* out_name(char* buf, size_t n, const char* dir, const char* name, long long it, const char* ext) {
  snprintf(buf, n, "%s/%s-%09lld.%s", dir, name, it, ext);
  return buf;
}

typedef struct {
  const opts* o;
  zf_ctx* ctx;
  const int32_t* b;
  int placed, nn, nnn, nw, mt, n_edge_n;
  const float* wxyz;
  const int32_t* wtri;
  const int32_t* edge_n;
} run_t;

/* OUTPUT() of the reference (ZebraflowWT.c:282-509) and the post-processor's
 * wall file, for the current state */
static void write_outputs(const run_t* r) {
  const opts* o = r->o;
  zf_ctx* ctx = r->ctx;
  char path[4096];
  int64_t it = 0, n = 0, nf = 0;
  check(zf_iteration(ctx, &it), "zf_iteration");
  check(zf_num_listed(ctx, &n, &nf), "zf_num_listed");
  const size_t npts = (size_t)o->nx * o->ny * o->nz;
  float* mom = (float*)xmalloc(sizeof(float) * 4 * (size_t)n);
  float* bf = (float*)xmalloc(sizeof(float) * 3 * (size_t)n);
  int32_t* en = (int32_t*)xmalloc(sizeof(int32_t) * (size_t)n);
  int32_t* wi = (int32_t*)xmalloc(sizeof(int32_t) * npts);
  check(zf_lbm_moments(ctx), "zf_lbm_moments");
  check(zf_download_moments(ctx, mom, mom + n, mom + 2 * n, mom + 3 * n), "zf_download_moments");
  check(zf_download_bodyforce(ctx, bf), "zf_download_bodyforce");
  check(zf_get_cell_list_counts(ctx, en), "zf_get_cell_list_counts");
  check(zf_get_wall_index(ctx, wi, NULL), "zf_get_wall_index");
  const double origin[3] = {0.0, 0.0, 0.0};
  check(zf_write_fluid_csv(out_name(path, sizeof path, o->output_dir, "FLUIDdomain", it, "csv"), o->nx, o->ny,
                           o->nz, origin, DX_UM, r->b, mom, mom + n, mom + 2 * n, mom + 3 * n, bf, en, wi),
        "zf_write_fluid_csv");
  if (r->placed > 0) {
    const size_t nc = (size_t)r->placed, m = 3 * nc * r->nn, mn = 3 * nc * r->nnn;
    double *x = (double*)xmalloc(sizeof(double) * m), *xn = (double*)xmalloc(sizeof(double) * mn);
    double *v = (double*)xmalloc(sizeof(double) * m), *vn = (double*)xmalloc(sizeof(double) * mn);
    float *wr = (float*)xmalloc(sizeof(float) * m), *wrn = (float*)xmalloc(sizeof(float) * mn);
    float *ft = (float*)xmalloc(sizeof(float) * m), *ftn = (float*)xmalloc(sizeof(float) * mn);
    float* cf = (float*)xmalloc(sizeof(float) * 8 * nc);
    int32_t* st = (int32_t*)xmalloc(sizeof(int32_t) * nc);
    int32_t ne = 0;
    double a0 = 0, v0 = 0;
    check(zf_mesh_info(ctx, &ne, &a0, &v0), "zf_mesh_info");
    float* epar = (float*)xmalloc(sizeof(float) * 5 * (size_t)ne);
    float* epar_n = (float*)xmalloc(sizeof(float) * 3 * (size_t)r->n_edge_n);
    check(zf_get_cells(ctx, x, xn, st), "zf_get_cells");
    check(zf_get_cell_kinematics(ctx, v, vn, wr, wrn), "zf_get_cell_kinematics");
    check(zf_get_cell_forces(ctx, ft, ftn), "zf_get_cell_forces");
    check(zf_get_cell_geometry(ctx, NULL, NULL, NULL, NULL, cf), "zf_get_cell_geometry");
    check(zf_get_edge_params(ctx, epar, epar_n, NULL), "zf_get_edge_params");
    check(zf_write_membrane_csv(out_name(path, sizeof path, o->output_dir, "AllCellMemb", it, "csv"), r->placed,
                                r->nn, NULL, st, x, v, NULL, wr, NULL, NULL, ft, NULL, NULL),
          "zf_write_membrane_csv");
    check(zf_write_nucleus_csv(out_name(path, sizeof path, o->output_dir, "AllCellNucleus", it, "csv"), r->placed,
                               r->nnn, NULL, st, xn, vn, ftn, NULL, NULL),
          "zf_write_nucleus_csv");
    check(zf_write_nucleus_edges_csv(out_name(path, sizeof path, o->output_dir, "AllNucEdgeMesh", it, "csv"),
                                     r->placed, r->nnn, r->n_edge_n, NULL, st, xn, r->edge_n, epar_n),
          "zf_write_nucleus_edges_csv");
    snprintf(path, sizeof path, "%s/VolumeAreaHistory.dat", o->output_dir);
    check(zf_append_volume_area(path, it, r->placed, NULL, st, cf, NULL), "zf_append_volume_area");
    free(x), free(xn), free(v), free(vn), free(wr), free(wrn), free(ft), free(ftn), free(cf), free(st);
    free(epar), free(epar_n);
  }
  float* wss = (float*)xmalloc(sizeof(float) * 3 * (size_t)r->nw);
  float* press = (float*)xmalloc(sizeof(float) * (size_t)r->nw);
  int32_t* valid = (int32_t*)xmalloc(sizeof(int32_t) * (size_t)r->nw);
  check(zf_wss(ctx, NULL, 120.0, wss, press, valid), "zf_wss");
  check(zf_write_wall_vtk(out_name(path, sizeof path, o->output_dir, "Wallpressure", it, "vtk"), r->nw, r->wxyz,
                          r->mt, r->wtri, press, wss, valid),
        "zf_write_wall_vtk");
  free(mom), free(bf), free(en), free(wi), free(wss), free(press), free(valid);
}

int main(int argc, char** argv) {
  const opts o = parse(argc, argv);
  const double origin[3] = {0.0, 0.0, 0.0};
  const size_t npts = (size_t)o.nx * o.ny * o.nz;

  /* vessel (the reference reads FLUIDdomainBindex.csv, ZebraflowWT.c:2574-2619) */
  int32_t* b = (int32_t*)xmalloc(sizeof(int32_t) * npts);
  if (o.bifurcation)
    check(zf_gen_bifurcation(o.nx, o.ny, o.nz, o.Rp, o.Rd, o.half_angle, b, NULL), "zf_gen_bifurcation");
  else
    check(zf_gen_tube(o.nx, o.ny, o.nz, 0.5 * (o.nx - 1), 0.5 * (o.ny - 1), o.R, 1, b), "zf_gen_tube");
  int64_t n_fluid = 0;
  for (size_t p = 0; p < npts; ++p) n_fluid += b[p] > 0;

  zf_params P;
  zf_params_default(&P);
  P.nx = o.nx;
  P.ny = o.ny;
  P.nz = o.nz;
  for (int d = 0; d < 3; ++d) P.origin[d] = origin[d];
  P.dx = DX_UM;
  P.tau = o.tau;
  P.tau_from_phase = 0;
  P.wall_mode = ZF_WALL_HALFWAY_BB;
  P.periodic[0] = P.periodic[1] = 0;
  P.periodic[2] = 1;
  P.g[0] = P.g[1] = 0.f;
  P.g[2] = o.g;
  P.storage = o.storage;
  P.stagger = o.stagger;
  P.area0 = 0.0; /* rest area and volume from the rest mesh */
  P.volume0 = 0.0;

  zf_ctx* ctx = zf_create(&P, o.device);
  if (!ctx) {
    fprintf(stderr, "zf_run: zf_create failed: %s\n", zf_last_error());
    return 1;
  }
  check(zf_set_lattice(ctx, b), "zf_set_lattice");

  /* wall mesh (the reference reads it at ZebraflowWT.c:3715-3897) */
  int nw = 0, mt = 0;
  float *wxyz = NULL, *wnrm = NULL;
  int32_t* wtri = NULL;
  wall_mesh(&o, origin, &nw, &mt, &wxyz, &wtri, &wnrm);
  check(zf_set_wall(ctx, nw, wxyz, mt, wtri, wnrm), "zf_set_wall");

  /* membrane and nucleus meshes (the reference reads them at :1601-1922) */
  /* icosphere levels 3 (membrane) and 2 (nucleus): 10 4^L + 2 nodes, 20 4^L triangles */
  const int nn = 10 * 64 + 2, nt = 20 * 64, nnn = 10 * 16 + 2, ntn = 20 * 16;
  double* rest = (double*)xmalloc(sizeof(double) * 3 * nn);
  double* rest_n = (double*)xmalloc(sizeof(double) * 3 * nnn);
  int32_t* tri = (int32_t*)xmalloc(sizeof(int32_t) * 3 * nt);
  int32_t* tri_n = (int32_t*)xmalloc(sizeof(int32_t) * 3 * ntn);
  check(zf_gen_icosphere(3, rest, tri), "zf_gen_icosphere");
  check(zf_gen_icosphere(2, rest_n, tri_n), "zf_gen_icosphere");
  const double ax[3] = {AX_X, AX_Y, AX_Z}, axn[3] = {AXN_X, AXN_Y, AXN_Z};
  for (int n = 0; n < nn; ++n)
    for (int d = 0; d < 3; ++d) rest[3 * n + d] *= ax[d];
  for (int n = 0; n < nnn; ++n)
    for (int d = 0; d < 3; ++d) rest_n[3 * n + d] *= axn[d];
  int n_edge_n = 0;
  int32_t* edge_n = mesh_edges(tri_n, ntn, &n_edge_n);
  check(zf_set_mesh(ctx, nn, nt, tri, rest, nnn, n_edge_n, edge_n, rest_n), "zf_set_mesh");

  /* cells (the reference reads AllCellMembStart / AllCellNucStart, :5297-5637) */
  int placed = 0;
  double* x = (double*)xmalloc(sizeof(double) * 3 * (size_t)o.cells * nn);
  double* xn = (double*)xmalloc(sizeof(double) * 3 * (size_t)o.cells * nnn);
  if (o.cells > 0) {
    check(zf_gen_cells(b, o.nx, o.ny, o.nz, origin, DX_UM, 1, o.cells, nn, rest, nnn, rest_n, ax, MARGIN_UM, 0.0,
                       o.seed, x, xn, &placed),
          "zf_gen_cells");
    /* compact [3][o.cells][n] to [3][placed][n] */
    for (int d = 1; d < 3; ++d) {
      memmove(x + (size_t)d * placed * nn, x + (size_t)d * o.cells * nn, sizeof(double) * (size_t)placed * nn);
      memmove(xn + (size_t)d * placed * nnn, xn + (size_t)d * o.cells * nnn, sizeof(double) * (size_t)placed * nnn);
    }
    if (placed > 0) check(zf_set_cells(ctx, placed, x, xn), "zf_set_cells");
  }

  if (o.load_state) check(zf_load_state(ctx, o.load_state), "zf_load_state");
  const run_t run = {&o, ctx, b, placed, nn, nnn, nw, mt, n_edge_n, wxyz, wtri, edge_n};
  int64_t it0 = 0;
  check(zf_iteration(ctx, &it0), "zf_iteration");
  if (o.output_every > 0 && it0 % o.output_every == 0) write_outputs(&run);

  /* the time loop in whole cycles of `stagger` iterations (and up to each
     output iteration); outputs are written outside the timed steps */
  float ms = 0.f, part = 0.f;
  int done = 0;
  while (done < o.steps) {
    const int64_t it = it0 + done;
    int n = o.stagger - (int)(it % o.stagger);
    if (o.output_every > 0) {
      const int to_out = o.output_every - (int)(it % o.output_every);
      if (to_out < n) n = to_out;
    }
    if (n > o.steps - done) n = o.steps - done;
    check(zf_step_timed(ctx, n, &part), "zf_step_timed");
    ms += part;
    done += n;
    if (o.output_every > 0 && (it0 + done) % o.output_every == 0) write_outputs(&run);
  }
  if (o.save_state) check(zf_save_state(ctx, o.save_state), "zf_save_state");
  zf_status st;
  check(zf_get_status(ctx, &st), "zf_get_status");
  const int64_t blocks = placed > 0 ? st.iter / o.stagger - it0 / o.stagger : 0;
  const double s = ms * 1e-3;
  printf("zf_run: %d iterations, %lld fluid points, %d cells (%lld removed), %lld membrane blocks, "
         "%.3f ms device time, %.1f MLUPS, %.4g membrane-node updates/s\n",
         o.steps, (long long)n_fluid, placed, (long long)st.cells_removed, (long long)blocks, ms,
         s > 0 ? (double)n_fluid * o.steps / s / 1e6 : 0.0,
         s > 0 ? (double)placed * (nn + nnn) * blocks / s : 0.0);

  /* final state */
  int32_t* status = (int32_t*)xmalloc(sizeof(int32_t) * (placed ? placed : 1));
  if (placed > 0) check(zf_get_cells(ctx, x, xn, status), "zf_get_cells");
  float* wss = (float*)xmalloc(sizeof(float) * 3 * (size_t)nw);
  float* press = (float*)xmalloc(sizeof(float) * (size_t)nw);
  int32_t* valid = (int32_t*)xmalloc(sizeof(int32_t) * (size_t)nw);
  check(zf_wss(ctx, NULL, 120.0, wss, press, valid), "zf_wss");
  int64_t n_listed = 0, nf = 0;
  check(zf_num_listed(ctx, &n_listed, &nf), "zf_num_listed");
  float* mom = (float*)xmalloc(sizeof(float) * 4 * (size_t)n_listed);
  check(zf_download_moments(ctx, mom, mom + n_listed, mom + 2 * n_listed, mom + 3 * n_listed),
        "zf_download_moments");

  if (o.out) {
    /* binary dump: magic, sizes, positions, status, WSS, moments */
    FILE* f = fopen(o.out, "wb");
    if (!f) {
      fprintf(stderr, "zf_run: cannot write %s\n", o.out);
      return 1;
    }
    const int32_t hdr[4] = {placed, nn, nnn, nw};
    const int64_t hdr2[2] = {st.iter, n_listed};
    fwrite("ZFRUN001", 1, 8, f);
    fwrite(hdr, sizeof hdr, 1, f);
    fwrite(hdr2, sizeof hdr2, 1, f);
    fwrite(x, sizeof(double), 3 * (size_t)placed * nn, f);
    fwrite(xn, sizeof(double), 3 * (size_t)placed * nnn, f);
    fwrite(status, sizeof(int32_t), (size_t)placed, f);
    fwrite(wss, sizeof(float), 3 * (size_t)nw, f);
    fwrite(mom, sizeof(float), 4 * (size_t)n_listed, f);
    if (fclose(f)) {
      fprintf(stderr, "zf_run: write error on %s\n", o.out);
      return 1;
    }
  }
  zf_destroy(ctx);
  free(b), free(wxyz), free(wtri), free(wnrm), free(rest), free(rest_n), free(tri), free(tri_n), free(edge_n);
  free(x), free(xn), free(status), free(wss), free(press), free(valid), free(mom);
  return 0;
}
