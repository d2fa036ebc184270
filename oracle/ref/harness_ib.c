/*
 * ORACLE — test infrastructure only.  Runs the reference's own membrane
 * iteration, IB coupling and cell interactions included, on a scene read from
 * a file (lattice sub-box, fluid velocity, wall mesh with its lattice index,
 * cells; written by tests/golden/make_ref_golden.py from tests/golden/ib_scene.py)
 * and writes the state after every stage.
 *
 * Linked against ZebraflowWT.c compiled where it lies (`main` renamed) and
 * passed through oracle/ref/expose_omp.py (OpenMP regions of main() callable
 * as zf_ref_omp_L<line of their pragma>).  Set-up: the reference's own
 * CGSM_ZFISHRBC_DATA_GEN, the calibration loop of main() (ZebraflowWT.c:
 * 2336-2346) and LBM_DOM_SETUP (:1481-1502); the rest areas from a CGSM_AREA
 * pass over the undeformed mesh (the formula main() uses at :2387-2460); the
 * lattice coordinates X, Y, Z as main() sets them (:2509-2511); the wall
 * triangle lists and centroids as main() builds them (:3899-3932, :4650-4658).
 * The lattice wall index W_index and void velocity Uvoid come from the scene
 * (the oracle's restatement of :3715-3822 and :4788-4852).  One membrane
 * iteration, in main()'s order, each region called through GOMP_parallel:
 *   zf_ref_omp_L5659   Eulerian triangle lists cleared        :5659-5667
 *   zf_ref_omp_L5706   CGSM_NODAL_FORCE_ZERO                  :5706-5745 (shares `i`)
 *   zf_ref_omp_L5749   CGSM_AREA + Eulerian triangle lists    :5749-6096
 *   zf_ref_omp_L6718   cell centroid, area                    :6718-6796
 *   zf_ref_omp_L6801   CGSM_LOCAL_FORCES                      :6801-7505 (shares `node`)
 *   zf_ref_omp_L7513   CGSM_VOLUME_CALC                       :7513-7535
 *   zf_ref_omp_L8694   IB interpolation + wall repulsion      :8694-9510
 *   zf_ref_omp_L9520   nucleus-membrane repulsion             :9520-9903
 *   zf_ref_omp_L9915   RBC-RBC repulsion (region-of-interest) :9915-10197
 *   zf_ref_omp_L10740  IB spreading (region-of-interest)      :10740-11172
 *   zf_ref_omp_L11923  position update (region-of-interest)   :11923-12189
 * The LBM regions between them are left out (the fluid velocity is the
 * scene's) and so are the parent-domain regions (no parent cells).  Cells are
 * region-of-interest cells 345.. with CellStatus 1.  Every cell region runs on
 * one thread, so that the float sums it accumulates into shared arrays
 * (spreading, pairwise repulsion) come out the same on every run.
 *
 * With a step count in the scene header the harness runs that many iterations
 * of main()'s time loop instead, from the scene's populations: every iteration
 * the LBM blocks (:6101-6145, :6292-6433, :6601-6626, after LBM_BC_SETUP), every
 * 50th also the cell blocks above around them in main()'s order, and writes the
 * final populations, body force and node positions.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#define IM_ 249
#define JM_ 547
#define KM_ 723
#define NL 8500000
#define CAPSM 3000
#define NODEM 504
#define TRIM 1004
#define NODEM_N 121
#define NODEW 1107042
#define CELLW 2212824
#define EULMAX 800

extern int iter, iter_local, simfailure, RBCSOLVERFLAG;
extern float relaxfactor, relaxfactor2, ZM_1, ZM_2, ZM_3, XM, YM, ZM;
extern int B_index[IM_ + 1][JM_ + 1][KM_ + 1], W_index[IM_ + 1][JM_ + 1][KM_ + 1];
extern int DOMID[IM_ + 1][JM_ + 1][KM_ + 1], DOMLIST[NL][3], DOMMAX;
extern float X[IM_ + 1][JM_ + 1][KM_ + 1], Y[IM_ + 1][JM_ + 1][KM_ + 1], Z[IM_ + 1][JM_ + 1][KM_ + 1];
extern float Uvoid[IM_ + 1][JM_ + 1][KM_ + 1], Vvoid[IM_ + 1][JM_ + 1][KM_ + 1],
    Wvoid[IM_ + 1][JM_ + 1][KM_ + 1];
extern float U[NL], V[NL], W[NL], D[NL], BODYFORCE[3][NL];
extern float F[20][NL], F_OLD[20][NL];
extern float Xlattice[3][20], UC[20], VC[20], WC[20], Wcoeff[20];
extern float WALLNODECOORD[3][NODEW + 1], WALLCELLNORMALS[3][CELLW + 1], WALL_CENTROID[3][CELLW + 1];
extern int WALLCELLNODE[3][CELLW + 1], WALLNODETOCELLNEIGHBORLIST[12 + 1][NODEW + 1];
extern double NODECOORD[3][CAPSM + 1][NODEM + 1], NODECOORD_N[3][CAPSM + 1][NODEM_N + 1];
extern double NODE_VEL[3][CAPSM + 1][NODEM + 1], NODE_VEL_N[3][CAPSM + 1][NODEM_N + 1];
extern float F_Total[3][CAPSM + 1][NODEM + 1], F_Total_N[3][CAPSM + 1][NODEM_N + 1];
extern float NODE_WALLREPUL[3][CAPSM + 1][NODEM + 1], NODE_WALLREPUL_N[3][CAPSM + 1][NODEM_N + 1];
extern float NODE_AREA[CAPSM + 1][NODEM + 1], NODE_AREA0[NODEM + 1];
extern float TRI_AREA[CAPSM + 1][TRIM + 1], TRI_AREA_eq[TRIM + 1];
extern int CellStatus[CAPSM + 1], REGRESSFLAG[CAPSM + 1], NucMembUpdate[CAPSM + 1];

void CGSM_ZFISHRBC_DATA_GEN(void);
void CGSM_FILAMENT_PARAMETERS(void);
void CGSM_EQUILIBRIUM_METRICS(void);
void LBM_DOM_SETUP(void);
void LBM_BC_SETUP(void);
void GOMP_parallel(void (*fn)(void*), void* data, unsigned num_threads, unsigned flags);
void zf_ref_omp_L5659(void*);
void zf_ref_omp_L5706(void*);
void zf_ref_omp_L5749(void*);
void zf_ref_omp_L6101(void*);
void zf_ref_omp_L6292(void*);
void zf_ref_omp_L6601(void*);
void zf_ref_omp_L6718(void*);
void zf_ref_omp_L6801(void*);
void zf_ref_omp_L7513(void*);
void zf_ref_omp_L8694(void*);
void zf_ref_omp_L9520(void*);
void zf_ref_omp_L9915(void*);
void zf_ref_omp_L10740(void*);
void zf_ref_omp_L11923(void*);

static FILE* fo;
static void put(const void* p, size_t bytes) {
  if (fwrite(p, 1, bytes, fo) != bytes) exit(2);
}
static void get(FILE* f, void* p, size_t bytes) {
  if (fread(p, 1, bytes, f) != bytes) {
    fprintf(stderr, "short scene file\n");
    exit(3);
  }
}

static int nc;
#define C0 345
static void put_nodes_d(double (*a)[CAPSM + 1][NODEM + 1]) {
  for (int x = 0; x < 3; ++x)
    for (int c = 0; c < nc; ++c) put(&a[x][C0 + c][1], 8 * NODEM);
}
static void put_nuc_d(double (*a)[CAPSM + 1][NODEM_N + 1]) {
  for (int x = 0; x < 3; ++x)
    for (int c = 0; c < nc; ++c) put(&a[x][C0 + c][1], 8 * NODEM_N);
}
static void put_nodes_f(float (*a)[CAPSM + 1][NODEM + 1]) {
  for (int x = 0; x < 3; ++x)
    for (int c = 0; c < nc; ++c) put(&a[x][C0 + c][1], 4 * NODEM);
}
static void put_nuc_f(float (*a)[CAPSM + 1][NODEM_N + 1]) {
  for (int x = 0; x < 3; ++x)
    for (int c = 0; c < nc; ++c) put(&a[x][C0 + c][1], 4 * NODEM_N);
}

static void forces(int geometry_only) {
  int i_shared = 0;
  struct { int* i; } d4 = {&i_shared};
  struct { int node; } d19 = {0};
  GOMP_parallel(zf_ref_omp_L5659, NULL, 1, 0);
  GOMP_parallel(zf_ref_omp_L5706, &d4, 1, 0);
  GOMP_parallel(zf_ref_omp_L5749, NULL, 1, 0);
  if (geometry_only) return;
  GOMP_parallel(zf_ref_omp_L6718, NULL, 1, 0);
  GOMP_parallel(zf_ref_omp_L6801, &d19, 1, 0);
  GOMP_parallel(zf_ref_omp_L7513, NULL, 1, 0);
}

int main(int argc, char** argv) {
  if (argc < 3) return 1;
  FILE* fs = fopen(argv[1], "rb");
  if (!fs) return 1;
  int hdr[12];
  get(fs, hdr, sizeof hdr);
  const int I0 = hdr[0], J0 = hdr[1], K0 = hdr[2], nx = hdr[3], ny = hdr[4], nz = hdr[5];
  const int nw = hdr[6], mt = hdr[7], n_listed = hdr[10], n_steps = hdr[11];
  nc = hdr[8];
  const size_t npts = (size_t)nx * ny * nz;
  int32_t* b = malloc(npts * 4);
  int32_t* wi = malloc(npts * 4);
  float* uv = malloc(3 * npts * 4);
  float* vel = malloc(3 * (size_t)n_listed * 4);
  float *wxyz = malloc(3 * (size_t)nw * 4), *wnrm = malloc(3 * (size_t)mt * 4);
  int32_t* wtri = malloc(3 * (size_t)mt * 4);
  double *cx = malloc(3 * (size_t)nc * NODEM * 8), *cxn = malloc(3 * (size_t)nc * NODEM_N * 8);
  get(fs, b, npts * 4);
  get(fs, vel, 3 * (size_t)n_listed * 4);
  get(fs, wi, npts * 4);
  get(fs, uv, 3 * npts * 4);
  get(fs, wxyz, 3 * (size_t)nw * 4);
  get(fs, wtri, 3 * (size_t)mt * 4);
  get(fs, wnrm, 3 * (size_t)mt * 4);
  get(fs, cx, 3 * (size_t)nc * NODEM * 8);
  get(fs, cxn, 3 * (size_t)nc * NODEM_N * 8);
  float* f0 = NULL;
  if (n_steps > 0) {
    f0 = malloc(19 * (size_t)n_listed * 4);
    get(fs, f0, 19 * (size_t)n_listed * 4);
  }
  fclose(fs);
  if (nc < 1 || C0 + nc - 1 > CAPSM || nw > NODEW || mt > CELLW) return 4;

  /* membrane mesh and calibration (:2336-2346) */
  CGSM_ZFISHRBC_DATA_GEN();
  iter_local = 0;
  do {
    iter_local = iter_local + 1;
    CGSM_FILAMENT_PARAMETERS();
    CGSM_EQUILIBRIUM_METRICS();
  } while (iter_local <= 50);
  XM = -1.f + (IM_ - 1) * 0.5f;
  YM = 29.f + (JM_ - 1) * 0.5f;
  ZM = -27.f + (KM_ - 1) * 0.5f;
  ZM_1 = -86.f + (121 - 1) * 0.5f;
  ZM_2 = 332.5f + (121 - 1) * 0.5f;
  ZM_3 = 332.5f + (121 - 1) * 0.5f;
  relaxfactor = relaxfactor2 = 1.f;
  for (int c = 1; c <= CAPSM; ++c) {
    CellStatus[c] = -5000;
    REGRESSFLAG[c] = 0;
  }

  /* lattice: everything unlisted except the scene's sub-box */
  for (int i = 1; i <= IM_; ++i)
    for (int j = 1; j <= JM_; ++j)
      for (int k = 1; k <= KM_; ++k) {
        B_index[i][j][k] = -1;
        W_index[i][j][k] = 0;
      }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const size_t p = ((size_t)i * ny + j) * nz + k;
        const int I = I0 + i + 1, J = J0 + j + 1, K = K0 + k + 1;
        B_index[I][J][K] = b[p];
        W_index[I][J][K] = wi[p];
        Uvoid[I][J][K] = uv[p];
        Vvoid[I][J][K] = uv[npts + p];
        Wvoid[I][J][K] = uv[2 * npts + p];
        X[I][J][K] = -1. + (I - 1) * 0.5;
        Y[I][J][K] = 29. + (J - 1) * 0.5;
        Z[I][J][K] = -27. + (K - 1) * 0.5;
      }
  LBM_DOM_SETUP();
  if (DOMMAX != n_listed) return 5;
  for (int l = 1; l <= DOMMAX; ++l) {
    U[l] = vel[l - 1];
    V[l] = vel[n_listed + l - 1];
    W[l] = vel[2 * (size_t)n_listed + l - 1];
    D[l] = 1.f;
    BODYFORCE[0][l] = BODYFORCE[1][l] = BODYFORCE[2][l] = 0.f;
  }

  /* wall mesh, its node -> triangle lists (:3899-3932) and centroids (:4650-4658) */
  for (int m = 1; m <= nw; ++m)
    for (int a = 0; a < 3; ++a) WALLNODECOORD[a][m] = wxyz[(size_t)a * nw + m - 1];
  for (int m = 1; m <= nw; ++m)
    for (int q = 0; q <= 12; ++q) WALLNODETOCELLNEIGHBORLIST[q][m] = 0;
  for (int t = 1; t <= mt; ++t) {
    for (int a = 0; a < 3; ++a) {
      WALLCELLNODE[a][t] = wtri[(size_t)a * mt + t - 1];
      WALLCELLNORMALS[a][t] = wnrm[(size_t)a * mt + t - 1];
    }
    for (int a = 0; a < 3; ++a) {
      const int n = WALLCELLNODE[a][t];
      const int cnt = ++WALLNODETOCELLNEIGHBORLIST[0][n];
      if (cnt > 12) return 6;
      WALLNODETOCELLNEIGHBORLIST[cnt][n] = t;
    }
    float p1[3], p2[3], p3[3];
    for (int a = 0; a < 3; ++a) {
      p1[a] = WALLNODECOORD[a][WALLCELLNODE[0][t]];
      p2[a] = WALLNODECOORD[a][WALLCELLNODE[1][t]];
      p3[a] = WALLNODECOORD[a][WALLCELLNODE[2][t]];
    }
    for (int a = 0; a < 3; ++a) WALL_CENTROID[a][t] = (p1[a] + p2[a] + p3[a]) / 3.;
  }

  /* rest areas: a CGSM_AREA pass over an undeformed copy of the rest mesh,
     placed outside the sub-box */
  RBCSOLVERFLAG = 1;
  iter = 50;
  for (int a = 0; a < 3; ++a) {
    for (int n = 1; n <= NODEM; ++n) NODECOORD[a][C0][n] = NODECOORD[a][1][n];
    for (int n = 1; n <= NODEM_N; ++n) NODECOORD_N[a][C0][n] = NODECOORD_N[a][1][n];
  }
  CellStatus[C0] = 1;
  forces(1);
  for (int t = 1; t <= TRIM; ++t) TRI_AREA_eq[t] = TRI_AREA[C0][t];
  for (int n = 1; n <= NODEM; ++n) NODE_AREA0[n] = NODE_AREA[C0][n];

  /* the scene's cells */
  for (int c = 0; c < nc; ++c) {
    for (int a = 0; a < 3; ++a) {
      for (int n = 1; n <= NODEM; ++n)
        NODECOORD[a][C0 + c][n] = cx[((size_t)a * nc + c) * NODEM + n - 1];
      for (int n = 1; n <= NODEM_N; ++n)
        NODECOORD_N[a][C0 + c][n] = cxn[((size_t)a * nc + c) * NODEM_N + n - 1];
    }
    CellStatus[C0 + c] = 1;
    NucMembUpdate[C0 + c] = 0;
  }
  iter = hdr[9];
  simfailure = 0;

  fo = fopen(argv[2], "wb");
  if (!fo) return 1;
  if (n_steps > 0) {
    /* lattice constants as main() sets them (:2471-2503), boundary list,
       the scene's populations, no body force */
    static const int E[19][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},
                                 {0, 0, -1}, {1, 1, 0},  {-1, -1, 0}, {-1, 1, 0}, {1, -1, 0},
                                 {1, 0, 1},  {-1, 0, -1}, {-1, 0, 1}, {1, 0, -1}, {0, 1, 1},
                                 {0, -1, -1}, {0, -1, 1}, {0, 1, -1}, {0, 0, 0}};
    for (int c = 1; c <= 19; ++c) {
      for (int a = 0; a < 3; ++a) Xlattice[a][c] = (float)E[c - 1][a];
      UC[c] = Xlattice[0][c];
      VC[c] = Xlattice[1][c];
      WC[c] = Xlattice[2][c];
      Wcoeff[c] = c <= 6 ? 1.f / 18.f : (c <= 18 ? 1.f / 36.f : 1.f / 3.f);
    }
    LBM_BC_SETUP();
    for (int l = 1; l <= DOMMAX; ++l)
      for (int c = 1; c <= 19; ++c) F[c][l] = F_OLD[c][l] = f0[(size_t)(c - 1) * n_listed + l - 1];
    int i_shared = 0;
    struct { int* i; } d4 = {&i_shared};
    struct { int node; } d19 = {0};
    for (int s = 1; s <= n_steps; ++s) {
      iter = s;
      RBCSOLVERFLAG = s % 50 == 0;
      if (RBCSOLVERFLAG) {
        GOMP_parallel(zf_ref_omp_L5659, NULL, 1, 0);
        GOMP_parallel(zf_ref_omp_L5706, &d4, 1, 0);
        GOMP_parallel(zf_ref_omp_L5749, NULL, 1, 0);
      }
      GOMP_parallel(zf_ref_omp_L6101, NULL, 0, 0);
      GOMP_parallel(zf_ref_omp_L6292, NULL, 0, 0);
      GOMP_parallel(zf_ref_omp_L6601, NULL, 0, 0);
      if (RBCSOLVERFLAG) {
        GOMP_parallel(zf_ref_omp_L6718, NULL, 1, 0);
        GOMP_parallel(zf_ref_omp_L6801, &d19, 1, 0);
        GOMP_parallel(zf_ref_omp_L7513, NULL, 1, 0);
        GOMP_parallel(zf_ref_omp_L8694, NULL, 1, 0);
        GOMP_parallel(zf_ref_omp_L9520, NULL, 1, 0);
        GOMP_parallel(zf_ref_omp_L9915, NULL, 1, 0);
        GOMP_parallel(zf_ref_omp_L10740, NULL, 1, 0);
        GOMP_parallel(zf_ref_omp_L11923, NULL, 1, 0);
      }
    }
    for (int c = 1; c <= 19; ++c) put(&F_OLD[c][1], 4 * (size_t)DOMMAX);
    for (int a = 0; a < 3; ++a) put(&BODYFORCE[a][1], 4 * (size_t)DOMMAX);
    put_nodes_d(NODECOORD);
    put_nuc_d(NODECOORD_N);
    for (int c = 0; c < nc; ++c) put(&CellStatus[C0 + c], 4);
    put(&simfailure, 4);
    fclose(fo);
    return 0;
  }
  forces(0);
  put_nodes_f(F_Total);
  put_nuc_f(F_Total_N);
  GOMP_parallel(zf_ref_omp_L8694, NULL, 1, 0);
  put_nodes_d(NODE_VEL);
  put_nuc_d(NODE_VEL_N);
  put_nodes_f(NODE_WALLREPUL);
  put_nuc_f(NODE_WALLREPUL_N);
  GOMP_parallel(zf_ref_omp_L9520, NULL, 1, 0);
  put_nodes_f(NODE_WALLREPUL);
  put_nuc_f(NODE_WALLREPUL_N);
  GOMP_parallel(zf_ref_omp_L9915, NULL, 1, 0);
  put_nodes_f(NODE_WALLREPUL);
  put_nuc_f(NODE_WALLREPUL_N);
  GOMP_parallel(zf_ref_omp_L10740, NULL, 1, 0);
  for (int a = 0; a < 3; ++a) put(&BODYFORCE[a][1], 4 * (size_t)DOMMAX);
  put_nodes_d(NODE_VEL);
  put_nuc_d(NODE_VEL_N);
  GOMP_parallel(zf_ref_omp_L11923, NULL, 1, 0);
  put_nodes_d(NODECOORD);
  put_nuc_d(NODECOORD_N);
  for (int c = 0; c < nc; ++c) put(&CellStatus[C0 + c], 4);
  put(&simfailure, 4);
  fclose(fo);
  return 0;
}
