/* Problem selector for the oracle build of KORAL: independent radiating
 * cells in the Kerr-Schild metric, used to drive the reference's per-cell
 * implicit radiation source solve (solve_implicit_lab, rad.c:1225) cell by
 * cell.  Stands in for the reference's problem.h so that the reference
 * sources compile unmodified (see oracle/ref/build_ref.sh). */
#define PROBLEM 202
#define PR_DEFINE "define.h"
#define PR_BC "bc.c"
#define PR_INIT "init.c"
#define PR_KAPPA "kappa.c"
#define PR_KAPPAES "kappaes.c"
#define PR_TOOLS "tools.c"

#ifdef _OPENMP
#define OMP
#endif

#include PR_DEFINE
