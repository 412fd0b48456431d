/* Electron scattering, 0.34 cm^2/g, as an inverse length in code units with
 * radiation; zero without. */
#ifdef TORUS_RADIATION
return kappaCGS2GU(TORUS_KES) * rho;
#else
return 0.;
#endif
