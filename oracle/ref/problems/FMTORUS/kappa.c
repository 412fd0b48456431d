/* No radiation in this problem: zero absorption opacity. */
kappa=0.;
