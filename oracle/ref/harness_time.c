/*
 * ORACLE — test infrastructure only (the timed CPU baseline of bench.py).
 * Times the reference's own LBM time step on a lattice read from a file: the
 * stream-collide, wall and copy blocks of its main() (ZebraflowWT.c:6101-6145,
 * :6292-6433, :6601-6626), each called through GOMP_parallel with the default
 * OpenMP team exactly as main() calls it, after the reference's own
 * LBM_DOM_SETUP and LBM_BC_SETUP.  Linked against ZebraflowWT.c compiled where
 * it lies (`main` renamed) and passed through oracle/ref/expose_omp.py.
 *
 * Input file: int32 nx, ny, nz, then int32 codes [nx][ny][nz] (-1 unlisted,
 * 0 wall, 1..9 fluid phase); the lattice sits at reference index (i+1, j+1,
 * k+2) and must fit the reference's compile-time box.  The populations start
 * at rest with a uniform body force along k; every 50th step is a membrane
 * step (RBCSOLVERFLAG = 1, the body force cleared), as in main().
 * Prints: fluid_points steps seconds threads.
 */
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#define IM_ 249
#define JM_ 547
#define KM_ 723
#define NL 8500000

extern int iter, RBCSOLVERFLAG;
extern float F[20][NL], F_OLD[20][NL];
extern int B_index[IM_ + 1][JM_ + 1][KM_ + 1];
extern float Xlattice[3][20], UC[20], VC[20], WC[20], Wcoeff[20];
extern float BODYFORCE[3][NL];
extern int DOMLIST[NL][3], DOMMAX;

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

static void step(int s) {
  iter = s;
  RBCSOLVERFLAG = s % 50 == 0;
  GOMP_parallel(zf_ref_omp_L6101, NULL, 0, 0);
  GOMP_parallel(zf_ref_omp_L6292, NULL, 0, 0);
  GOMP_parallel(zf_ref_omp_L6601, NULL, 0, 0);
}

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: ref_time lattice.bin steps max_seconds\n");
    return 1;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 1;
  int dims[3];
  if (fread(dims, 4, 3, f) != 3) return 1;
  const int nx = dims[0], ny = dims[1], nz = dims[2];
  if (nx < 1 || ny < 1 || nz < 1 || nx > IM_ || ny > JM_ || nz + 3 > KM_) {
    fprintf(stderr, "lattice %d x %d x %d does not fit the reference box\n", nx, ny, nz);
    return 2;
  }
  const int steps = atoi(argv[2]);
  const double max_seconds = atof(argv[3]);
  for (int i = 1; i <= IM_; ++i)
    for (int j = 1; j <= JM_; ++j)
      for (int k = 1; k <= KM_; ++k) B_index[i][j][k] = -1;
  int32_t* row = malloc(sizeof(int32_t) * (size_t)nz);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (fread(row, 4, (size_t)nz, f) != (size_t)nz) return 1;
      for (int k = 0; k < nz; ++k) B_index[i + 1][j + 1][k + 2] = row[k];
    }
  fclose(f);
  free(row);

  for (int c = 1; c <= 19; ++c) {
    for (int a = 0; a < 3; ++a) Xlattice[a][c] = (float)E[c - 1][a];
    UC[c] = Xlattice[0][c];
    VC[c] = Xlattice[1][c];
    WC[c] = Xlattice[2][c];
    Wcoeff[c] = c <= 6 ? 1.f / 18.f : (c <= 18 ? 1.f / 36.f : 1.f / 3.f);
  }
  iter = 0;
  LBM_DOM_SETUP();
  LBM_BC_SETUP();
  long long fluid = 0;
#pragma omp parallel for reduction(+ : fluid) schedule(static, 5000)
  for (int l = 1; l <= DOMMAX; ++l) {
    const int b = B_index[DOMLIST[l][0]][DOMLIST[l][1]][DOMLIST[l][2]];
    fluid += b > 0 && b < 10;
    for (int c = 1; c <= 19; ++c) F[c][l] = F_OLD[c][l] = Wcoeff[c];
    BODYFORCE[0][l] = BODYFORCE[1][l] = 0.f;
    BODYFORCE[2][l] = 4e-6f;
  }
  for (int s = 1; s <= 3; ++s) step(s);
  int done = 0;
  const double t0 = omp_get_wtime();
  double t = 0;
  while (done < steps) {
    step(4 + done);
    ++done;
    t = omp_get_wtime() - t0;
    if (t >= max_seconds) break;
  }
  printf("%lld %d %.6f %d\n", fluid, done, t, omp_get_max_threads());
  return 0;
}
