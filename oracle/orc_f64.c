/* ORACLE — test infrastructure only: the CPU restatement compiled with fp64
 * arithmetic (the FP64 oracle of the precision form).  See orc_lbm.inc. */
#include <omp.h>
#define REAL double
#define SFX _f64
#include "orc_lbm.inc"
#include "orc_cells.inc"
#include "orc_ib.inc"

/* threads the OpenMP loops of the oracle use */
int orc_max_threads(void) { return omp_get_max_threads(); }
