/*
 * ORACLE — test infrastructure only.  Links against the reference's own
 * ZebraflowWT.c (compiled where it lies, `main` renamed, by oracle/ref/Makefile)
 * and runs its set-up functions on the shipped RBC/nucleus meshes and on a
 * small synthetic lattice, writing their outputs to a binary file that the
 * oracle tests compare with the CPU restatement:
 *   CGSM_ZFISHRBC_DATA_GEN        ZebraflowWT.c:1592-1925 (edge/rhombus list)
 *   CGSM_FILAMENT_PARAMETERS x51  :1930-2053 with the loop of :2336-2346
 *   CGSM_EQUILIBRIUM_METRICS      :2056-2223
 *   LBM_DOM_SETUP, LBM_BC_SETUP   :1481-1589 (listed order, designated neighbours)
 * The declarations below name the reference's globals with the sizes of its
 * compile-time constants (ZebraflowWT.c:81-122, :171-276).
 */
#include <stdio.h>
#include <stdlib.h>

#define IM_ 249
#define JM_ 547
#define KM_ 723
#define NODEM 504
#define EDGEM 1506
#define TRIM 1004
#define NODEM_N 121
#define EDGEM_N 544
#define CAPSM 3000

extern int iter, iter_local;
extern int EDGENODE_LIST[EDGEM + 1][6 + 1];
extern int EDGENODE_LIST_N[EDGEM_N + 1][2 + 1];
extern float LMAX[EDGEM + 1], Plength[EDGEM + 1], kp[EDGEM + 1], Theta0[EDGEM + 1],
    SINETHETA0[EDGEM + 1], COSINETHETA0[EDGEM + 1];
extern float LMAX_N[EDGEM_N + 1], Plength_N[EDGEM_N + 1], kp_N[EDGEM_N + 1];
extern int B_index[IM_ + 1][JM_ + 1][KM_ + 1];
extern int DOMLIST[8500000][3], DOMMAX;
extern int BCLIST[1200000][4], BCNLIST[1200000][3], BCMAX;
extern float Xlattice[3][19 + 1];

void CGSM_ZFISHRBC_DATA_GEN(void);
void CGSM_FILAMENT_PARAMETERS(void);
void CGSM_EQUILIBRIUM_METRICS(void);
void LBM_DOM_SETUP(void);
void LBM_BC_SETUP(void);

/* D3Q19 vectors in the reference order (main() sets them at :2471-2497) */
static const int E[19][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},
                             {0, 0, -1}, {1, 1, 0},  {-1, -1, 0}, {-1, 1, 0}, {1, -1, 0},
                             {1, 0, 1},  {-1, 0, -1}, {-1, 0, 1}, {1, 0, -1}, {0, 1, 1},
                             {0, -1, -1}, {0, -1, 1}, {0, 1, -1}, {0, 0, 0}};

int main(int argc, char** argv) {
  const char* out = argc > 1 ? argv[1] : "ref_setup.bin";
  FILE* f = fopen(out, "wb");
  if (!f) return 1;
  /* membrane mesh, run as main() does at :2336-2346 */
  CGSM_ZFISHRBC_DATA_GEN();
  iter_local = 0;
  do {
    iter_local = iter_local + 1;
    CGSM_FILAMENT_PARAMETERS();
    CGSM_EQUILIBRIUM_METRICS();
  } while (iter_local <= 50);
  int ne = EDGEM, nen = EDGEM_N;
  fwrite(&ne, 4, 1, f);
  for (int e = 1; e <= EDGEM; ++e) fwrite(&EDGENODE_LIST[e][1], 4, 6, f);
  fwrite(&LMAX[1], 4, EDGEM, f);
  fwrite(&Plength[1], 4, EDGEM, f);
  fwrite(&kp[1], 4, EDGEM, f);
  fwrite(&SINETHETA0[1], 4, EDGEM, f);
  fwrite(&COSINETHETA0[1], 4, EDGEM, f);
  fwrite(&nen, 4, 1, f);
  fwrite(&LMAX_N[1], 4, EDGEM_N, f);
  fwrite(&Plength_N[1], 4, EDGEM_N, f);
  fwrite(&kp_N[1], 4, EDGEM_N, f);

  /* lattice: a tube of radius 6 along k through part of the box, fluid
     phase 1, wall points around it, everything else solid */
  for (int c = 1; c <= 19; ++c)
    for (int a = 0; a < 3; ++a) Xlattice[a][c] = (float)E[c - 1][a];
  for (int i = 1; i <= IM_; ++i)
    for (int j = 1; j <= JM_; ++j)
      for (int k = 1; k <= KM_; ++k) B_index[i][j][k] = -1;
  const int ci = 20, cj = 30;
  for (int i = ci - 9; i <= ci + 9; ++i)
    for (int j = cj - 9; j <= cj + 9; ++j)
      for (int k = 5; k <= 40; ++k) {
        const int r2 = (i - ci) * (i - ci) + (j - cj) * (j - cj);
        if (r2 < 36 && k > 6 && k < 38) B_index[i][j][k] = 1;
      }
  for (int i = ci - 9; i <= ci + 9; ++i)
    for (int j = cj - 9; j <= cj + 9; ++j)
      for (int k = 5; k <= 40; ++k) {
        if (B_index[i][j][k] > 0) continue;
        for (int q = 0; q < 18; ++q) {
          const int ii = i + E[q][0], jj = j + E[q][1], kk = k + E[q][2];
          if (B_index[ii][jj][kk] > 0) {
            B_index[i][j][k] = 0;
            break;
          }
        }
      }
  iter = 0;
  LBM_DOM_SETUP();
  LBM_BC_SETUP();
  fwrite(&DOMMAX, 4, 1, f);
  for (int l = 1; l <= DOMMAX; ++l) fwrite(&DOMLIST[l][0], 4, 3, f);
  fwrite(&BCMAX, 4, 1, f);
  for (int l = 1; l <= BCMAX; ++l) {
    fwrite(&BCLIST[l][0], 4, 4, f);
    fwrite(&BCNLIST[l][0], 4, 3, f);
  }
  fclose(f);
  return 0;
}
