/* ORACLE — test infrastructure only: the CPU restatement compiled with fp32
 * arithmetic (reference float state).  See orc_lbm.inc. */
#include <omp.h>
#define REAL float
#define SFX _f32
#include "orc_lbm.inc"
#include "orc_cells.inc"
#include "orc_ib.inc"
