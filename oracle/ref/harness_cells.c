/*
 * ORACLE — test infrastructure only.  Runs the reference's own membrane step
 * (forces of four deformed RBCs with nuclei, one screened, one removed) and
 * writes inputs and outputs to a binary file that the oracle tests compare
 * with the CPU restatement.
 *
 * Linked against ZebraflowWT.c compiled where it lies (`main` renamed) and
 * passed through oracle/ref/expose_omp.py (OpenMP regions of main() callable as
 * zf_ref_omp_L<line of their pragma>).  Set-up: the reference's own
 * CGSM_ZFISHRBC_DATA_GEN and the CGSM_FILAMENT_PARAMETERS /
 * CGSM_EQUILIBRIUM_METRICS loop of main() (ZebraflowWT.c:2336-2346) on the
 * shipped meshes; the rest triangle areas TRI_AREA_eq are those of the rest
 * mesh (main() computes them at :2387-2460 with the same formula as CGSM_AREA,
 * so the harness takes them from a CGSM_AREA pass over an undeformed copy).
 * Membrane step, in main()'s order, each region called through GOMP_parallel:
 *   zf_ref_omp_L5706  CGSM_NODAL_FORCE_ZERO         :5706-5745 (shares `i`)
 *   zf_ref_omp_L5749  CGSM_AREA (+ sliver push)     :5749-6096
 *   zf_ref_omp_L6718  cell centroid, area           :6718-6796
 *   zf_ref_omp_L6801  CGSM_LOCAL_FORCES             :6801-7505 (shares `node`)
 *   zf_ref_omp_L7513  CGSM_VOLUME_CALC              :7513-7535
 * The shared locals are passed as main() passes them (the object's debug info
 * gives the layouts: a pointer to `i`, the value of `node`); the region that
 * shares `i` between its threads runs on one thread.  The cells are region-of-
 * interest cells (numbers above 344, CellStatus 1) on an empty lattice, so the
 * cell-list insert of CGSM_AREA finds no lattice point and adds nothing.
 * Declarations name the reference's globals with its sizes (ZebraflowWT.c:
 * 85-122, :171-172, :220-248, :260-272).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define IM_ 249
#define JM_ 547
#define KM_ 723
#define CAPSM 3000
#define NODEM 504
#define TRIM 1004
#define NODEM_N 121

extern int iter, iter_local, simfailure, RBCSOLVERFLAG;
extern float relaxfactor, relaxfactor2, ZM_1, ZM_2, ZM_3, XM, YM, ZM;
extern int B_index[IM_ + 1][JM_ + 1][KM_ + 1];
extern double NODECOORD[3][CAPSM + 1][NODEM + 1], NODECOORD_N[3][CAPSM + 1][NODEM_N + 1];
extern float F_Total[3][CAPSM + 1][NODEM + 1], F_Total_N[3][CAPSM + 1][NODEM_N + 1];
extern float NODE_AREA[CAPSM + 1][NODEM + 1], NODE_AREA0[NODEM + 1];
extern float TRI_AREA[CAPSM + 1][TRIM + 1], TRI_AREA_eq[TRIM + 1];
extern float TRI_NORMAL[3][CAPSM + 1][TRIM + 1], TRI_CENTROID[3][CAPSM + 1][TRIM + 1];
extern float NODE_NORMAL[3][CAPSM + 1][NODEM + 1];
extern float CAPS_CENTROID[3][CAPSM + 1], CAPS_AREA[CAPSM + 1], CAPS_VOL[CAPSM + 1];
extern float F_AREA_GLOBAL[CAPSM + 1], F_VOLUME_SCALAR[CAPSM + 1];
extern int CellStatus[CAPSM + 1], CAPS_REMOVE[CAPSM + 1];

void CGSM_ZFISHRBC_DATA_GEN(void);
void CGSM_FILAMENT_PARAMETERS(void);
void CGSM_EQUILIBRIUM_METRICS(void);
void GOMP_parallel(void (*fn)(void*), void* data, unsigned num_threads, unsigned flags);
void zf_ref_omp_L5706(void*);
void zf_ref_omp_L5749(void*);
void zf_ref_omp_L6718(void*);
void zf_ref_omp_L6801(void*);
void zf_ref_omp_L7513(void*);

#define NCELL 4
static const int CELL[NCELL] = {345, 346, 347, 348};

static uint64_t rng = 0x2545F4914F6CDD1Dull;
static double u01(void) {
  rng ^= rng << 13;
  rng ^= rng >> 7;
  rng ^= rng << 17;
  return (double)(rng >> 11) * (1.0 / 9007199254740992.0);
}
static double nrm(void) { return sqrt(-2.0 * log(u01() + 1e-300)) * cos(6.283185307179586 * u01()); }

static void put(FILE* f, const void* p, size_t bytes) {
  if (fwrite(p, 1, bytes, f) != bytes) exit(2);
}

/* one membrane step of the cells whose CellStatus is above -5000 (geometry
   only: force reset and CGSM_AREA) */
static void membrane_step(int geometry_only) {
  int i_shared = 0;
  struct { int* i; } d4 = {&i_shared};
  struct { int node; } d19 = {0};
  RBCSOLVERFLAG = 1;
  GOMP_parallel(zf_ref_omp_L5706, &d4, 1, 0);
  GOMP_parallel(zf_ref_omp_L5749, NULL, 0, 0);
  if (geometry_only) return;
  GOMP_parallel(zf_ref_omp_L6718, NULL, 0, 0);
  /* one thread: the block counts screened forces into the shared simfailure
     without atomics */
  GOMP_parallel(zf_ref_omp_L6801, &d19, 1, 0);
  GOMP_parallel(zf_ref_omp_L7513, NULL, 0, 0);
}

int main(int argc, char** argv) {
  const char* out = argc > 1 ? argv[1] : "ref_cells.bin";
  /* membrane mesh and its calibration, as main() runs them (:2336-2346) */
  CGSM_ZFISHRBC_DATA_GEN();
  iter_local = 0;
  do {
    iter_local = iter_local + 1;
    CGSM_FILAMENT_PARAMETERS();
    CGSM_EQUILIBRIUM_METRICS();
  } while (iter_local <= 50);

  /* the box bounds main() and the parent set-up compute (:762-764, :2523-2525) */
  XM = -1.f + (IM_ - 1) * 0.5f;
  YM = 29.f + (JM_ - 1) * 0.5f;
  ZM = -27.f + (KM_ - 1) * 0.5f;
  ZM_1 = -86.f + (121 - 1) * 0.5f;
  ZM_2 = 332.5f + (121 - 1) * 0.5f;
  ZM_3 = 332.5f + (121 - 1) * 0.5f;
  relaxfactor = relaxfactor2 = 1.f;
  iter = 50;
  for (int i = 1; i <= IM_; ++i)
    for (int j = 1; j <= JM_; ++j)
      for (int k = 1; k <= KM_; ++k) B_index[i][j][k] = -1;
  for (int c = 1; c <= CAPSM; ++c) CellStatus[c] = -5000;

  /* rest areas: a CGSM_AREA pass over an undeformed copy of the rest mesh */
  const int c0 = CELL[0];
  for (int a = 0; a < 3; ++a) {
    for (int n = 1; n <= NODEM; ++n) NODECOORD[a][c0][n] = NODECOORD[a][1][n];
    for (int n = 1; n <= NODEM_N; ++n) NODECOORD_N[a][c0][n] = NODECOORD_N[a][1][n];
  }
  CellStatus[c0] = 1;
  membrane_step(1);
  for (int t = 1; t <= TRIM; ++t) TRI_AREA_eq[t] = TRI_AREA[c0][t];
  for (int n = 1; n <= NODEM; ++n) NODE_AREA0[n] = NODE_AREA[c0][n];

  /* four deformed cells: rest mesh stretched, moved into the box, with node
     noise 0.03 um (nucleus 0.02 um); the last two with noise large enough
     that force screening acts (0.3 um) and that the cell is removed (1 um) */
  const double stretch[NCELL][3] = {{1.06, 0.97, 1.0}, {0.98, 1.03, 1.05}, {1.0, 1.0, 1.0},
                                    {1.0, 1.0, 1.0}};
  const double shift[NCELL][3] = {{60.0, 150.0, 150.0}, {75.0, 160.0, 170.0},
                                  {90.0, 150.0, 150.0}, {105.0, 160.0, 170.0}};
  const double noise[NCELL] = {0.03, 0.03, 0.3, 1.0};
  for (int s = 0; s < NCELL; ++s) {
    const int c = CELL[s];
    for (int n = 1; n <= NODEM; ++n)
      for (int a = 0; a < 3; ++a)
        NODECOORD[a][c][n] = NODECOORD[a][1][n] * stretch[s][a] + shift[s][a] + noise[s] * nrm();
    for (int n = 1; n <= NODEM_N; ++n)
      for (int a = 0; a < 3; ++a)
        NODECOORD_N[a][c][n] = NODECOORD_N[a][1][n] * stretch[s][a] + shift[s][a] + 0.02 * nrm();
    CellStatus[c] = 1;
  }
  /* the input coordinates (a removed cell's are overwritten by the step) */
  static double x_in[NCELL][3][NODEM + 1], xn_in[NCELL][3][NODEM_N + 1];
  for (int s = 0; s < NCELL; ++s)
    for (int a = 0; a < 3; ++a) {
      for (int n = 1; n <= NODEM; ++n) x_in[s][a][n] = NODECOORD[a][CELL[s]][n];
      for (int n = 1; n <= NODEM_N; ++n) xn_in[s][a][n] = NODECOORD_N[a][CELL[s]][n];
    }
  simfailure = 0;
  printf("membrane step of the deformed cells\n");
  fflush(stdout);
  membrane_step(0);

  FILE* f = fopen(out, "wb");
  if (!f) return 1;
  int dims[4] = {NCELL, NODEM, NODEM_N, TRIM};
  put(f, dims, sizeof dims);
  put(f, &TRI_AREA_eq[1], 4 * TRIM);
  for (int s = 0; s < NCELL; ++s) {
    const int c = CELL[s];
    for (int a = 0; a < 3; ++a) put(f, &x_in[s][a][1], 8 * NODEM);
    for (int a = 0; a < 3; ++a) put(f, &xn_in[s][a][1], 8 * NODEM_N);
    for (int a = 0; a < 3; ++a) put(f, &F_Total[a][c][1], 4 * NODEM);
    for (int a = 0; a < 3; ++a) put(f, &F_Total_N[a][c][1], 4 * NODEM_N);
    put(f, &TRI_AREA[c][1], 4 * TRIM);
    for (int a = 0; a < 3; ++a) put(f, &TRI_NORMAL[a][c][1], 4 * TRIM);
    for (int a = 0; a < 3; ++a) put(f, &TRI_CENTROID[a][c][1], 4 * TRIM);
    for (int a = 0; a < 3; ++a) put(f, &NODE_NORMAL[a][c][1], 4 * NODEM);
    float cellf[7] = {CAPS_AREA[c], CAPS_VOL[c], CAPS_CENTROID[0][c], CAPS_CENTROID[1][c],
                      CAPS_CENTROID[2][c], F_AREA_GLOBAL[c], F_VOLUME_SCALAR[c]};
    put(f, cellf, sizeof cellf);
    int st[2] = {CellStatus[c], CAPS_REMOVE[c]};
    put(f, st, sizeof st);
  }
  put(f, &simfailure, 4);
  fclose(f);
  return 0;
}
