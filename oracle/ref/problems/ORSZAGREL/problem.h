/* Problem selector for the oracle build of KORAL: relativistic Orszag-Tang
 * vortex.  Stands in for the reference's problem.h (which hard-wires one
 * problem) so that the reference sources compile unmodified; every PR_*
 * hook named by the reference (problem.c:46-107, rad.c:22-36) points at the
 * plug-in files in this directory. */
#define PROBLEM 200
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
