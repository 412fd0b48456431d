/* Radiating cells around a spin-0.9 Kerr black hole (KORAL plug-in format).
 * The grid only provides storage: the test harness overwrites the metric,
 * the conserved and the primitive variables of every cell with independent
 * random draws and calls the implicit source solve on each.  M1 radiation
 * with Kramers-type absorption and electron scattering, Gamma = 13/9,
 * black-hole mass 10 solar masses (for the unit conversions). */
#define MYCOORDS KSCOORDS
#define BHSPIN 0.9
#define MASS 10.

#define RADIATION
#define MAGNFIELD

#define INT_ORDER 1
#define FLUXMETHOD LAXF_FLUX
#define TIMESTEPPING RK2IMEX
#define TSTEPLIM 0.5
#define FLUXLIMITER 0
#define MINMOD_THETA 1.5
#define GAMMA (13./9.)

/* Kramers absorption coefficient (cm^2 g^-1 at rho = 1 g cm^-3, T = 1 K)
 * and the electron-scattering opacity (cm^2 g^-1) */
#define RADCELLS_KRAMERS 6.4e22
#define RADCELLS_KES 0.34

#define MINX 2.
#define MAXX 100.
#define MINY 0.1
#define MAXY (M_PI - 0.1)
#define MINZ -1.
#define MAXZ 1.
#ifndef TNX
#define TNX 64
#endif
#ifndef TNY
#define TNY 64
#endif
#define TNZ 1
#define SPECIFIC_BC

#define NOUTSTOP 1e50
#define DTOUT1 1.e50
#define DTOUT2 1.e50
#define SILOOUTPUT 0
#define OUTOUTPUT 0
#define AVGOUTPUT 0
#define SCAOUTPUT 0
#define RADOUTPUT 0
