/*
 * ORACLE — test infrastructure only.  Runs the reference's own LBM time step
 * on a small synthetic lattice and writes its inputs and outputs to a binary
 * file that the oracle tests compare with the CPU restatement.
 *
 * Linked against ZebraflowWT.c compiled where it lies (`main` renamed) and
 * passed through oracle/ref/expose_omp.py, which makes the OpenMP regions of
 * the reference's main() callable as zf_ref_omp_L<line of their pragma>.  One
 * LBM step is the three ROI regions main() runs in this order, each called
 * through GOMP_parallel exactly as main() calls it:
 *   zf_ref_omp_L6101  LBM_STREAM & LBM_COLLISION   ZebraflowWT.c:6101-6145
 *   zf_ref_omp_L6292  LBM_BC                       :6292-6433
 *   zf_ref_omp_L6601  LBM_FLUID & LBM_COPY         :6601-6626
 * The parent-domain regions between them work on the DA/PCV precursor arrays,
 * which this lattice leaves empty.  The set-up is the reference's own
 * LBM_DOM_SETUP and LBM_BC_SETUP; the lattice constants follow main()
 * (:2471-2503).  Declarations name the reference's globals with its sizes
 * (ZebraflowWT.c:81-83, :171-185, :272).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define IM_ 249
#define JM_ 547
#define KM_ 723
#define NL 8500000

extern int iter, RBCSOLVERFLAG;
extern float U[NL], V[NL], W[NL], D[NL];
extern float F[20][NL], F_OLD[20][NL], FEQ[20][NL];
extern int B_index[IM_ + 1][JM_ + 1][KM_ + 1];
extern float Xlattice[3][20], UC[20], VC[20], WC[20], Wcoeff[20];
extern float BODYFORCE[3][NL];
extern int BCLIST[1200000][4], BCNLIST[1200000][3], BCMAX, DOMLIST[NL][3], DOMMAX;

void LBM_DOM_SETUP(void);
void LBM_BC_SETUP(void);
void GOMP_parallel(void (*fn)(void*), void* data, unsigned num_threads, unsigned flags);
void zf_ref_omp_L6101(void*);
void zf_ref_omp_L6292(void*);
void zf_ref_omp_L6601(void*);

static const int E[19][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},
                             {0, 0, -1}, {1, 1, 0},  {-1, -1, 0}, {-1, 1, 0}, {1, -1, 0},
                             {1, 0, 1},  {-1, 0, -1}, {-1, 0, 1}, {1, 0, -1}, {0, 1, 1},
                             {0, -1, -1}, {0, -1, 1}, {0, 1, -1}, {0, 0, 0}};

/* the lattice: a tube of radius 4 along k (centre i = 20, j = 30), fluid for
   6 < k < 20, with a ball of phase 5 (tau from the phase) inside it and wall
   points (code 0) at every point linked to the fluid; all else unlisted.
   With argv[2] = "pressure" the tube's end layers k = 6 and k = 20 are
   pressure inlets/outlets of codes argv[3] and argv[4] (1001-1009, the
   reference's waveforms, ZebraflowWT.c:6316-6426) and the steps are
   iterations argv[5] + 1 ... of its time loop. */
#define CI 20
#define CJ 30
#define TUBE_R2 16
#define K_LO 6
#define K_HI 20
#define N_STEPS 5

static uint64_t rng = 0x9E3779B97F4A7C15ull;
static double u01(void) {
  rng ^= rng << 13;
  rng ^= rng >> 7;
  rng ^= rng << 17;
  return (double)(rng >> 11) * (1.0 / 9007199254740992.0);
}

static void put(FILE* f, const void* p, size_t bytes) {
  if (fwrite(p, 1, bytes, f) != bytes) exit(2);
}

static void put_pops(FILE* f, float (*a)[NL]) {
  for (int c = 1; c <= 19; ++c) put(f, &a[c][1], sizeof(float) * (size_t)DOMMAX);
}

int main(int argc, char** argv) {
  const char* out = argc > 1 ? argv[1] : "ref_step.bin";
  const int pressure = argc > 5 && !strcmp(argv[2], "pressure");
  const int code_lo = pressure ? atoi(argv[3]) : 0, code_hi = pressure ? atoi(argv[4]) : 0;
  const int iter0 = pressure ? atoi(argv[5]) : 0;
  FILE* f = fopen(out, "wb");
  if (!f) return 1;

  /* lattice constants as main() sets them (:2471-2503); C_LBM = 1 */
  for (int c = 1; c <= 19; ++c) {
    for (int a = 0; a < 3; ++a) Xlattice[a][c] = (float)E[c - 1][a];
    UC[c] = Xlattice[0][c];
    VC[c] = Xlattice[1][c];
    WC[c] = Xlattice[2][c];
    Wcoeff[c] = c <= 6 ? 1.f / 18.f : (c <= 18 ? 1.f / 36.f : 1.f / 3.f);
  }

  for (int i = 1; i <= IM_; ++i)
    for (int j = 1; j <= JM_; ++j)
      for (int k = 1; k <= KM_; ++k) B_index[i][j][k] = -1;
  for (int i = CI - 6; i <= CI + 6; ++i)
    for (int j = CJ - 6; j <= CJ + 6; ++j)
      for (int k = K_LO - 1; k <= K_HI + 1; ++k) {
        const int r2 = (i - CI) * (i - CI) + (j - CJ) * (j - CJ);
        const int b2 = r2 + (k - 13) * (k - 13);
        if (r2 < TUBE_R2 && k > K_LO && k < K_HI) B_index[i][j][k] = b2 < 5 ? 5 : 1;
        if (pressure && r2 < TUBE_R2 && k == K_LO) B_index[i][j][k] = code_lo;
        if (pressure && r2 < TUBE_R2 && k == K_HI) B_index[i][j][k] = code_hi;
      }
  for (int i = CI - 6; i <= CI + 6; ++i)
    for (int j = CJ - 6; j <= CJ + 6; ++j)
      for (int k = K_LO - 1; k <= K_HI + 1; ++k) {
        if (B_index[i][j][k] > 0) continue;
        for (int q = 0; q < 18; ++q)
          if (B_index[i + E[q][0]][j + E[q][1]][k + E[q][2]] > 0) {
            B_index[i][j][k] = 0;
            break;
          }
      }
  iter = iter0;
  LBM_DOM_SETUP();
  LBM_BC_SETUP();

  /* perturbed rest state and a body force with a mean along k */
  for (int l = 1; l <= DOMMAX; ++l) {
    for (int c = 1; c <= 19; ++c) {
      F_OLD[c][l] = (float)(Wcoeff[c] * (1.0 + 0.02 * (u01() - 0.5)));
      F[c][l] = F_OLD[c][l];
    }
    for (int a = 0; a < 3; ++a) BODYFORCE[a][l] = (float)(2e-3 * (u01() - 0.5) + (a == 2 ? 1e-3 : 0.0));
  }

  int n = DOMMAX, steps = N_STEPS;
  put(f, &n, 4);
  put(f, &steps, 4);
  if (pressure) put(f, &iter0, 4);
  for (int l = 1; l <= DOMMAX; ++l) {
    put(f, &DOMLIST[l][0], 12);
    put(f, &B_index[DOMLIST[l][0]][DOMLIST[l][1]][DOMLIST[l][2]], 4);
  }
  put_pops(f, F_OLD);
  for (int a = 0; a < 3; ++a) put(f, &BODYFORCE[a][1], sizeof(float) * (size_t)n);

  /* N_STEPS steps; the last one is a membrane step (RBCSOLVERFLAG = 1), which
     also clears the body force in LBM_FLUID & LBM_COPY */
  for (int s = 1; s <= N_STEPS; ++s) {
    iter = iter0 + s;
    RBCSOLVERFLAG = s == N_STEPS;
    GOMP_parallel(zf_ref_omp_L6101, NULL, 0, 0);
    GOMP_parallel(zf_ref_omp_L6292, NULL, 0, 0);
    GOMP_parallel(zf_ref_omp_L6601, NULL, 0, 0);
    if (s == 1 || s == N_STEPS) put_pops(f, F_OLD);
  }
  put(f, &D[1], sizeof(float) * (size_t)n);
  put(f, &U[1], sizeof(float) * (size_t)n);
  put(f, &V[1], sizeof(float) * (size_t)n);
  put(f, &W[1], sizeof(float) * (size_t)n);
  for (int a = 0; a < 3; ++a) put(f, &BODYFORCE[a][1], sizeof(float) * (size_t)n);
  fclose(f);
  return 0;
}
