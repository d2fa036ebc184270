/*
 * ORACLE — test infrastructure only.  Runs the reference's own OUTPUT()
 * (ZebraflowWT.c:282-509) on a small lattice and two cells filled with seeded
 * values, so that the tests can hold this library's writers of the same
 * files (zebraflow_b200/csrc/zf_io.cpp) to the reference's bytes.
 *
 * Linked against ZebraflowWT.c compiled where it lies (`main` renamed).  The
 * set-up is the reference's LBM_DOM_SETUP on a capped tube; the parent
 * domains are left empty (B_index_1..3 = -1) and every cell slot but two is
 * removed (CellStatus -5000), as main() initialises them (:2505-2570,
 * :5297-5325).  OUTPUT() writes into SimulationOutputData/ under the current
 * directory; the inputs it was given go to the binary file named by argv[1]:
 *   int32 n, int32 dims[3] (the box written below, 1-based lower corner in
 *   dims[3..5]), then per listed point (i, j, k 1-based, B_index, EulNeigh,
 *   W_index) and D, U, V, W, BODYFORCE[3] as float planes; the two cells'
 *   ids and every membrane / nucleus array OUTPUT() prints.
 * Declarations name the reference's globals with its sizes (ZebraflowWT.c:81-276).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/stat.h>

#define IM_ 249
#define JM_ 547
#define KM_ 723
#define IM_1 69
#define JM_1 56
#define KM_1 121
#define IM_2 64
#define JM_2 60
#define KM_2 121
#define IM_3 42
#define JM_3 27
#define KM_3 121
#define NL 8500000
#define CAPS 3000
#define NODEM 504
#define NODEM_N 121
#define EDGEM_N 544
#define EULMAX 800

extern int iter;
extern float X[IM_ + 1][JM_ + 1][KM_ + 1], Y[IM_ + 1][JM_ + 1][KM_ + 1], Z[IM_ + 1][JM_ + 1][KM_ + 1];
extern int B_index[IM_ + 1][JM_ + 1][KM_ + 1], W_index[IM_ + 1][JM_ + 1][KM_ + 1];
extern int B_index_1[IM_1 + 1][JM_1 + 1][KM_1 + 1], B_index_2[IM_2 + 1][JM_2 + 1][KM_2 + 1],
    B_index_3[IM_3 + 1][JM_3 + 1][KM_3 + 1];
extern int DOMID[IM_ + 1][JM_ + 1][KM_ + 1], DOMLIST[NL][3], DOMMAX;
extern float U[NL], V[NL], W[NL], D[NL], BODYFORCE[3][NL];
extern int EulNeigh[EULMAX + 1][NL];
extern int CellStatus[CAPS + 1], REGRESSFLAG[CAPS + 1];
extern double NODECOORD[3][CAPS + 1][NODEM + 1], NODE_VEL[3][CAPS + 1][NODEM + 1];
extern int NODE_WALLNEIGH[CAPS + 1][NODEM + 1], MembOut_NeighFlag[CAPS + 1][NODEM + 1];
extern float NODE_WALLREPUL[3][CAPS + 1][NODEM + 1], NODE_AREA[CAPS + 1][NODEM + 1], NODE_AREA0[NODEM + 1];
extern float F_Total[3][CAPS + 1][NODEM + 1], F_VOLUME[3][CAPS + 1][NODEM + 1];
extern double NODECOORD_N[3][CAPS + 1][NODEM_N + 1], NODE_VEL_N[3][CAPS + 1][NODEM_N + 1];
extern float F_Total_N[3][CAPS + 1][NODEM_N + 1];
extern int NUC_Neigh[CAPS + 1][NODEM_N + 1], NUC_NeighFlag[CAPS + 1][NODEM_N + 1];
extern float LMAX_N[EDGEM_N + 1];
extern int EDGENODE_LIST_N[EDGEM_N + 1][3];
extern float CAPS_VOL[CAPS + 1], CAPS_AREA[CAPS + 1], CAPS_CENTROID[3][CAPS + 1];

void LBM_DOM_SETUP(void);
void OUTPUT(void);

static uint64_t rng = 0x2545F4914F6CDD1Dull;
static double u01(void) {
  rng ^= rng << 13;
  rng ^= rng >> 7;
  rng ^= rng << 17;
  return (double)(rng >> 11) * (1.0 / 9007199254740992.0);
}
static double sym(double a) { return a * (2.0 * u01() - 1.0); }

static void put(FILE* f, const void* p, size_t bytes) {
  if (fwrite(p, 1, bytes, f) != bytes) exit(2);
}

/* the box holding the lattice: i, j in [CI-6, CI+6], k in [1, 26] */
#define CI 20
#define CJ 30
#define KB 26

static const int CELLS[2] = {3, 9};

int main(int argc, char** argv) {
  const char* out = argc > 1 ? argv[1] : "ref_output_inputs.bin";
  for (int i = 1; i <= IM_; ++i)
    for (int j = 1; j <= JM_; ++j)
      for (int k = 1; k <= KM_; ++k) B_index[i][j][k] = -1;
  for (int i = 1; i <= IM_1; ++i)
    for (int j = 1; j <= JM_1; ++j)
      for (int k = 1; k <= KM_1; ++k) B_index_1[i][j][k] = -1;
  for (int i = 1; i <= IM_2; ++i)
    for (int j = 1; j <= JM_2; ++j)
      for (int k = 1; k <= KM_2; ++k) B_index_2[i][j][k] = -1;
  for (int i = 1; i <= IM_3; ++i)
    for (int j = 1; j <= JM_3; ++j)
      for (int k = 1; k <= KM_3; ++k) B_index_3[i][j][k] = -1;
  /* a tube of radius 4 along k with wall points around it and a phase-5 core */
  for (int i = CI - 6; i <= CI + 6; ++i)
    for (int j = CJ - 6; j <= CJ + 6; ++j)
      for (int k = 1; k <= KB; ++k) {
        X[i][j][k] = -1. + (i - 1) * 0.5; /* ZebraflowWT.c:2511-2513 */
        Y[i][j][k] = 29. + (j - 1) * 0.5;
        Z[i][j][k] = -27. + (k - 1) * 0.5;
        const int r2 = (i - CI) * (i - CI) + (j - CJ) * (j - CJ);
        if (k >= 3 && k <= KB - 2) B_index[i][j][k] = r2 < 16 ? (r2 < 4 ? 5 : 1) : (r2 < 30 ? 0 : -1);
        W_index[i][j][k] = B_index[i][j][k] == 0 ? 1 + (int)(u01() * 5000) : 0;
      }
  LBM_DOM_SETUP();
  for (int l = 1; l <= DOMMAX; ++l) {
    D[l] = (float)(1.0 + sym(0.05));
    U[l] = (float)sym(2e-3);
    V[l] = (float)sym(2e-3);
    W[l] = (float)sym(2e-3);
    for (int a = 0; a < 3; ++a) BODYFORCE[a][l] = (float)sym(1e-4);
    EulNeigh[0][l] = (int)(u01() * 6);
  }
  /* cells: every slot removed but two */
  for (int c = 1; c <= CAPS; ++c) CellStatus[c] = -5000;
  for (int n = 1; n <= NODEM; ++n) NODE_AREA0[n] = (float)(1e-13 * (1.0 + u01()));
  for (int e = 1; e <= EDGEM_N; ++e) {
    EDGENODE_LIST_N[e][1] = 1 + (int)(u01() * NODEM_N);
    EDGENODE_LIST_N[e][2] = 1 + (int)(u01() * NODEM_N);
    LMAX_N[e] = (float)(1e-6 * (0.5 + u01()));
  }
  for (int s = 0; s < 2; ++s) {
    const int c = CELLS[s];
    CellStatus[c] = s ? 2 : 1;
    REGRESSFLAG[c] = s ? -200 : 0;
    CAPS_VOL[c] = (float)(9.7e-17 * (1.0 + sym(0.1)));
    CAPS_AREA[c] = (float)(1.45e-10 * (1.0 + sym(0.1)));
    for (int a = 0; a < 3; ++a) CAPS_CENTROID[a][c] = (float)(20.0 + sym(15.0));
    for (int n = 1; n <= NODEM; ++n) {
      for (int a = 0; a < 3; ++a) {
        NODECOORD[a][c][n] = 20.0 + sym(15.0);
        NODE_VEL[a][c][n] = sym(1e-3);
        NODE_WALLREPUL[a][c][n] = (float)sym(1e-5);
        F_Total[a][c][n] = (float)sym(1e-12);
        F_VOLUME[a][c][n] = (float)sym(1e-13);
      }
      NODE_WALLNEIGH[c][n] = (int)(u01() * 60000);
      NODE_AREA[c][n] = (float)(NODE_AREA0[n] * (1.0 + sym(0.2)));
      MembOut_NeighFlag[c][n] = (int)(u01() * 3) - 1;
    }
    for (int n = 1; n <= NODEM_N; ++n) {
      for (int a = 0; a < 3; ++a) {
        NODECOORD_N[a][c][n] = 20.0 + sym(15.0);
        NODE_VEL_N[a][c][n] = sym(1e-3);
        F_Total_N[a][c][n] = (float)sym(1e-12);
      }
      NUC_Neigh[c][n] = (int)(u01() * 1004);
      NUC_NeighFlag[c][n] = (int)(u01() * 3) - 1;
    }
  }
  iter = 0;
  mkdir("SimulationOutputData", 0755);
  OUTPUT();

  FILE* f = fopen(out, "wb");
  if (!f) return 1;
  const int hdr[7] = {DOMMAX, 13, 13, KB, CI - 6, CJ - 6, 1};
  put(f, hdr, sizeof hdr);
  for (int l = 1; l <= DOMMAX; ++l) {
    const int i = DOMLIST[l][0], j = DOMLIST[l][1], k = DOMLIST[l][2];
    const int rec[6] = {i, j, k, B_index[i][j][k], EulNeigh[0][l], W_index[i][j][k]};
    put(f, rec, sizeof rec);
  }
  put(f, &D[1], sizeof(float) * (size_t)DOMMAX);
  put(f, &U[1], sizeof(float) * (size_t)DOMMAX);
  put(f, &V[1], sizeof(float) * (size_t)DOMMAX);
  put(f, &W[1], sizeof(float) * (size_t)DOMMAX);
  for (int a = 0; a < 3; ++a) put(f, &BODYFORCE[a][1], sizeof(float) * (size_t)DOMMAX);
  put(f, &NODE_AREA0[1], sizeof(float) * NODEM);
  for (int e = 1; e <= EDGEM_N; ++e) put(f, &EDGENODE_LIST_N[e][1], 2 * sizeof(int));
  put(f, &LMAX_N[1], sizeof(float) * EDGEM_N);
  for (int s = 0; s < 2; ++s) {
    const int c = CELLS[s];
    const int ch[3] = {c, CellStatus[c], REGRESSFLAG[c]};
    put(f, ch, sizeof ch);
    const float cf[5] = {CAPS_AREA[c], CAPS_VOL[c], CAPS_CENTROID[0][c], CAPS_CENTROID[1][c], CAPS_CENTROID[2][c]};
    put(f, cf, sizeof cf);
    for (int a = 0; a < 3; ++a) put(f, &NODECOORD[a][c][1], sizeof(double) * NODEM);
    for (int a = 0; a < 3; ++a) put(f, &NODE_VEL[a][c][1], sizeof(double) * NODEM);
    put(f, &NODE_WALLNEIGH[c][1], sizeof(int) * NODEM);
    for (int a = 0; a < 3; ++a) put(f, &NODE_WALLREPUL[a][c][1], sizeof(float) * NODEM);
    put(f, &NODE_AREA[c][1], sizeof(float) * NODEM);
    for (int a = 0; a < 3; ++a) put(f, &F_Total[a][c][1], sizeof(float) * NODEM);
    for (int a = 0; a < 3; ++a) put(f, &F_VOLUME[a][c][1], sizeof(float) * NODEM);
    put(f, &MembOut_NeighFlag[c][1], sizeof(int) * NODEM);
    for (int a = 0; a < 3; ++a) put(f, &NODECOORD_N[a][c][1], sizeof(double) * NODEM_N);
    for (int a = 0; a < 3; ++a) put(f, &NODE_VEL_N[a][c][1], sizeof(double) * NODEM_N);
    for (int a = 0; a < 3; ++a) put(f, &F_Total_N[a][c][1], sizeof(float) * NODEM_N);
    put(f, &NUC_Neigh[c][1], sizeof(int) * NODEM_N);
    put(f, &NUC_NeighFlag[c][1], sizeof(int) * NODEM_N);
  }
  fclose(f);
  return 0;
}
