/* Electron scattering, 0.34 cm^2/g, as an inverse length in code units. */
return kappaCGS2GU(RADCELLS_KES) * rho;
