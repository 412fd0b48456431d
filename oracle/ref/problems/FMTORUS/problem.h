/* Problem selector for the oracle build of KORAL: magnetised
 * Fishbone-Moncrief torus around a Kerr black hole in modified Kerr-Schild
 * coordinates.  Stands in for the reference's problem.h so that the
 * reference sources compile unmodified (see oracle/ref/build_ref.sh). */
#define PROBLEM 201
#define PR_DEFINE "define.h"
#define PR_BC "bc.c"
#define PR_INIT "init.c"
#define PR_POSTINIT "postinit.c"
#define PR_KAPPA "kappa.c"
#define PR_KAPPAES "kappaes.c"
#define PR_TOOLS "tools.c"
#define PR_DEFS "defs.h"

#ifdef _OPENMP
#define OMP
#endif

#include PR_DEFINE
