/* Declaration-only stand-in: forwards to the shared oracle shim header. */
#include <gsl/gsl_shim_all.h>
