/* Kramers-type absorption kappa_abs = 6.4e22 rho T^-3.5 cm^2/g as an
 * inverse length in code units with radiation; zero without. */
#ifdef TORUS_RADIATION
kappa = kappaCGS2GU(TORUS_KRAMERS * rhoGU2CGS(rho) * pow(T, -3.5)) * rho;
#else
kappa = 0.;
#endif
