/* No radiation in this problem: zero scattering opacity. */
return 0.;
