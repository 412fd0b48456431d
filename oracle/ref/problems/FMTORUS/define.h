/* 3D magnetised Kerr torus (KORAL plug-in format).
 * Spin 0.9, MKS2 coordinates (r = exp(x1)+R0, theta concentrated towards
 * the midplane by H0), r in [1.8, 1000] log-spaced, x2 in [0.005, 0.995]
 * (theta just off the poles), phi in [0, 2 pi].  Fishbone-Moncrief torus
 * with r_in = 6, r_max = 12, Gamma = 13/9, one poloidal loop from
 * A_phi = max(rho/rho_max - 0.2, 0) normalised to beta_min = 100, 2% seeded
 * pressure noise, density floor 1e-4 r^-1.5.  MP5 + HLL + flux-CT, RK2.
 * The grid may be overridden with -DTNX/-DTNY/-DTNZ for small parity builds.
 *
 * With -DTORUS_RADIATION the same torus carries M1 radiation, initialised
 * in local thermal equilibrium with the gas: the pressure of the torus
 * solution is shared by gas and radiation at one temperature T
 * (p = k rho T / (mu m_p) + 4 sigma T^4 / 3), E = 4 sigma T^4 in the frame
 * of the gas; Kramers-type absorption 6.4e22 rho T^-3.5 and electron
 * scattering 0.34 cm^2/g; the implicit lab-frame source solve; RK2IMEX
 * time stepping.  The torus keeps its code-unit density (maximum 1), as
 * without radiation; the black-hole mass (default 1e16 Msun) sets the
 * radiation units: with it the torus is optically thick to scattering
 * (kappa_es rho = 3.1e6 per GM/c^2 at the maximum) and radiation-pressure
 * dominated, and kappa dt of the implicit solve stays of order 1e4.  The
 * atmosphere keeps its gas energy and carries a faint radiation field at
 * rest with it (E = TORUS_ERADATM u, default 1e-6). */
#define MYCOORDS MKS2COORDS
#define MKSR0 0.
#define MKSH0 0.6
#define METRICAXISYMMETRIC
#define BHSPIN 0.9

#define MAGNFIELD
#define VECPOTGIVEN
#define TORUS_MAXBETA 0.01        /* max pmag/pgas, i.e. beta_min = 100 */

#define INT_ORDER 4
#define FLUXMETHOD HLL_FLUX
#ifdef TORUS_RADIATION
#define RADIATION
#define TIMESTEPPING RK2IMEX
#ifndef TORUS_KRAMERS
#define TORUS_KRAMERS 6.4e22
#endif
#ifndef TORUS_KES
#define TORUS_KES 0.34
#endif
#ifndef TORUS_MASS
#define TORUS_MASS 1.e16
#endif
/* radiative wave speeds from the rest-frame 1/sqrt(3) without the
 * optical-depth limiter (rad.c:2489-2502): with the limiter the time step
 * of this optically thick, radiation-supported torus follows the gas sound
 * speed alone and the explicit update is unstable */
#define SKIPRADWAVESPEEDLIMITER
#ifndef TORUS_ERADATM
#define TORUS_ERADATM 1.e-6
#endif
#else
#define TIMESTEPPING RK2
#endif
/* black-hole mass in solar masses: sets the units of the radiation physics
 * only */
#ifndef TORUS_MASS
#define TORUS_MASS 10.
#endif
#define MASS TORUS_MASS
#define TSTEPLIM 0.5
#define FLUXLIMITER 0
#define MINMOD_THETA 1.5
#define GAMMA (13./9.)

#define TORUS_RIN 6.
#define TORUS_RMAX 12.
#define TORUS_KAPPA 1.e-3
#define TORUS_NOISE 0.02
#define TORUS_SEED 12345ULL

/* floors: rho >= 1e-4 r^-1.5 via the reference's BH floor (u2p.c:546-557),
 * whose argument is r/r_horizon */
#define RHOFLOOR_BH
#define RHOFLOOR_BH_NORM (1.e-4 / pow(rhorizonBL, 1.5))
#define UURHORATIOMIN 1.e-10
#define UURHORATIOMAX 1.e2
#define B2RHORATIOMAX 100.
#define ATM_RHO0 1.e-4
#define ATM_UU0 1.e-6

#define MINX (log(1.8 - MKSR0))
#define MAXX (log(1000. - MKSR0))
#define MINY 0.005
#define MAXY 0.995
#define MINZ 0.
/* a phi wedge [0, TORUS_MAXZ] with TNZ cells and periodic phi boundaries
 * (e.g. -DTNZ=8 -DTORUS_MAXZ='(M_PI/4.)' keeps the phi cell size of the
 * 64-cell torus and the same cells, noise included, as its first 8 phi
 * columns) */
#ifndef TORUS_MAXZ
#define TORUS_MAXZ (2. * M_PI)
#endif
#define MAXZ TORUS_MAXZ
#ifndef TNX
#define TNX 192
#endif
#ifndef TNY
#define TNY 96
#endif
#ifndef TNZ
#define TNZ 64
#endif
#define SPECIFIC_BC

#define NOUTSTOP 1e50
#define DTOUT1 1.e50
#define DTOUT2 1.e50
#define SILOOUTPUT 0
#define OUTOUTPUT 0
#define AVGOUTPUT 0
#define SCAOUTPUT 0
#define RADOUTPUT 0
