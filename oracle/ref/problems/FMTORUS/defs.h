/* Prototypes of the torus plug-in helpers (tools.c), included by ko.h. */
double fmtorus_lfish(double a, double r);
double fmtorus_lnh_raw(double a, double l, double r, double th);
double fmtorus_uphi(double a, double l, double r, double th);
double fmtorus_noise(unsigned long long seed, unsigned long long idx);
