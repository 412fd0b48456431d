/* Kramers-type absorption: kappa_abs = 6.4e22 rho T^-3.5 cm^2/g, as an
 * inverse length in code units (T from calc_PEQ_Tfromurho in rad.c:19). */
kappa = kappaCGS2GU(RADCELLS_KRAMERS * rhoGU2CGS(rho) * pow(T, -3.5)) * rho;
