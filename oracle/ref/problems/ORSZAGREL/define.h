/* Relativistic ideal-MHD Orszag-Tang vortex (KORAL plug-in format).
 * Minkowski, periodic [0,2pi]^2, Gamma=5/3, PPM + Lax-Friedrichs + flux-CT,
 * RK2 with Courant number 0.5.  Grid size may be overridden with -DTNX/-DTNY
 * for small parity builds. */
#define MYCOORDS MINKCOORDS
#define MAGNFIELD
#define INT_ORDER 2
#define FLUXMETHOD LAXF_FLUX
#define TIMESTEPPING RK2
#define TSTEPLIM 0.5
#define GAMMA (5./3.)

#define MINX 0.
#define MAXX (2.*M_PI)
#define MINY 0.
#define MAXY (2.*M_PI)
#define MINZ (-1.)
#define MAXZ 1.
#ifndef TNX
#define TNX 128
#endif
#ifndef TNY
#define TNY 128
#endif
#define TNZ 1
#define PERIODIC_XBC
#define PERIODIC_YBC
#define PERIODIC_ZBC

#define NOUTSTOP 1e50
#define DTOUT1 1.e50
#define DTOUT2 1.e50
#define SILOOUTPUT 0
#define OUTOUTPUT 0
#define AVGOUTPUT 0
#define SCAOUTPUT 0
#define RADOUTPUT 0

/* Limiter settings the reference reads unconditionally (finite.c:9-24,118);
 * unused with PPM. */
#define FLUXLIMITER 0
#define MINMOD_THETA 1.5
