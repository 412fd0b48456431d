/*
 * Abort-on-use bodies for the declaration-only GSL stand-in
 * (gsl/gsl_shim_all.h).  Test infrastructure for the parity oracle.
 *
 * The reference hot path (reconstruction, fluxes, flux-CT, u2p, M1
 * inversion, implicit lab-frame solve) never calls GSL; these bodies exist
 * only so that the off-path translation units link.  Reaching any of them
 * means the oracle left the hot path, so the process stops with a message
 * naming the routine.  The single exception is gsl_set_error_handler_off,
 * which the reference calls unconditionally from main() (ko.c:31).
 */
#include <stdio.h>
#include <stdlib.h>
#include "gsl/gsl_shim_all.h"

static void gsl_shim_unreachable(const char *name)
{
  fprintf(stderr, "oracle GSL stand-in: %s reached; the oracle left the hot path\n", name);
  abort();
}

#define SHIM_ABORT(name) gsl_shim_unreachable(name)

gsl_error_handler_t *gsl_set_error_handler_off(void) { return NULL; }
const char *gsl_strerror(const int e) { (void)e; return "gsl stand-in"; }

gsl_vector *gsl_vector_alloc(size_t n) { (void)n; SHIM_ABORT("gsl_vector_alloc"); return NULL; }
void gsl_vector_free(gsl_vector *v) { (void)v; SHIM_ABORT("gsl_vector_free"); }
double gsl_vector_get(const gsl_vector *v, size_t i) { (void)v; (void)i; SHIM_ABORT("gsl_vector_get"); return 0.; }
void gsl_vector_set(gsl_vector *v, size_t i, double x) { (void)v; (void)i; (void)x; SHIM_ABORT("gsl_vector_set"); }
int gsl_vector_fprintf(FILE *s, const gsl_vector *v, const char *f) { (void)s; (void)v; (void)f; SHIM_ABORT("gsl_vector_fprintf"); return 0; }
gsl_matrix *gsl_matrix_alloc(size_t a, size_t b) { (void)a; (void)b; SHIM_ABORT("gsl_matrix_alloc"); return NULL; }
void gsl_matrix_free(gsl_matrix *m) { (void)m; SHIM_ABORT("gsl_matrix_free"); }
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { (void)m; (void)i; (void)j; SHIM_ABORT("gsl_matrix_get"); return 0.; }
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) { (void)m; (void)i; (void)j; (void)x; SHIM_ABORT("gsl_matrix_set"); }
gsl_matrix_view gsl_matrix_view_array(double *b, size_t a, size_t c) { gsl_matrix_view v; (void)b; (void)a; (void)c; SHIM_ABORT("gsl_matrix_view_array"); return v; }
gsl_vector_view gsl_matrix_column(gsl_matrix *m, size_t j) { gsl_vector_view v; (void)m; (void)j; SHIM_ABORT("gsl_matrix_column"); return v; }
gsl_vector_complex *gsl_vector_complex_alloc(size_t n) { (void)n; SHIM_ABORT("gsl_vector_complex_alloc"); return NULL; }
void gsl_vector_complex_free(gsl_vector_complex *v) { (void)v; SHIM_ABORT("gsl_vector_complex_free"); }
gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, size_t i) { gsl_complex z; (void)v; (void)i; SHIM_ABORT("gsl_vector_complex_get"); return z; }
gsl_permutation *gsl_permutation_alloc(size_t n) { (void)n; SHIM_ABORT("gsl_permutation_alloc"); return NULL; }
void gsl_permutation_free(gsl_permutation *p) { (void)p; SHIM_ABORT("gsl_permutation_free"); }

int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *s) { (void)A; (void)p; (void)s; SHIM_ABORT("gsl_linalg_LU_decomp"); return 0; }
int gsl_linalg_LU_invert(const gsl_matrix *LU, const gsl_permutation *p, gsl_matrix *i) { (void)LU; (void)p; (void)i; SHIM_ABORT("gsl_linalg_LU_invert"); return 0; }
int gsl_linalg_cholesky_decomp(gsl_matrix *A) { (void)A; SHIM_ABORT("gsl_linalg_cholesky_decomp"); return 0; }
int gsl_linalg_cholesky_invert(gsl_matrix *A) { (void)A; SHIM_ABORT("gsl_linalg_cholesky_invert"); return 0; }
int gsl_blas_dgemm(CBLAS_TRANSPOSE_t a, CBLAS_TRANSPOSE_t b, double al, const gsl_matrix *A, const gsl_matrix *B, double be, gsl_matrix *C)
{ (void)a; (void)b; (void)al; (void)A; (void)B; (void)be; (void)C; SHIM_ABORT("gsl_blas_dgemm"); return 0; }

gsl_eigen_symm_workspace *gsl_eigen_symm_alloc(const size_t n) { (void)n; SHIM_ABORT("gsl_eigen_symm_alloc"); return NULL; }
void gsl_eigen_symm_free(gsl_eigen_symm_workspace *w) { (void)w; SHIM_ABORT("gsl_eigen_symm_free"); }
int gsl_eigen_symm(gsl_matrix *A, gsl_vector *e, gsl_eigen_symm_workspace *w) { (void)A; (void)e; (void)w; SHIM_ABORT("gsl_eigen_symm"); return 0; }
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(const size_t n) { (void)n; SHIM_ABORT("gsl_eigen_symmv_alloc"); return NULL; }
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) { (void)w; SHIM_ABORT("gsl_eigen_symmv_free"); }
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *e, gsl_matrix *v, gsl_eigen_symmv_workspace *w) { (void)A; (void)e; (void)v; (void)w; SHIM_ABORT("gsl_eigen_symmv"); return 0; }
gsl_eigen_nonsymm_workspace *gsl_eigen_nonsymm_alloc(const size_t n) { (void)n; SHIM_ABORT("gsl_eigen_nonsymm_alloc"); return NULL; }
void gsl_eigen_nonsymm_free(gsl_eigen_nonsymm_workspace *w) { (void)w; SHIM_ABORT("gsl_eigen_nonsymm_free"); }
int gsl_eigen_nonsymm(gsl_matrix *A, gsl_vector_complex *e, gsl_eigen_nonsymm_workspace *w) { (void)A; (void)e; (void)w; SHIM_ABORT("gsl_eigen_nonsymm"); return 0; }

gsl_complex gsl_complex_add(gsl_complex a, gsl_complex b) { (void)b; SHIM_ABORT("gsl_complex_add"); return a; }
gsl_complex gsl_complex_sub(gsl_complex a, gsl_complex b) { (void)b; SHIM_ABORT("gsl_complex_sub"); return a; }
gsl_complex gsl_complex_mul(gsl_complex a, gsl_complex b) { (void)b; SHIM_ABORT("gsl_complex_mul"); return a; }
gsl_complex gsl_complex_mul_real(gsl_complex a, double x) { (void)x; SHIM_ABORT("gsl_complex_mul_real"); return a; }
gsl_complex gsl_complex_add_real(gsl_complex a, double x) { (void)x; SHIM_ABORT("gsl_complex_add_real"); return a; }
gsl_complex gsl_complex_negative(gsl_complex a) { SHIM_ABORT("gsl_complex_negative"); return a; }
gsl_complex gsl_complex_sqrt(gsl_complex a) { SHIM_ABORT("gsl_complex_sqrt"); return a; }
gsl_complex gsl_complex_sqrt_real(double x) { gsl_complex z; (void)x; SHIM_ABORT("gsl_complex_sqrt_real"); return z; }
gsl_complex gsl_complex_inverse(gsl_complex a) { SHIM_ABORT("gsl_complex_inverse"); return a; }
gsl_complex gsl_complex_conjugate(gsl_complex a) { SHIM_ABORT("gsl_complex_conjugate"); return a; }
double gsl_complex_abs(gsl_complex a) { (void)a; SHIM_ABORT("gsl_complex_abs"); return 0.; }
int gsl_poly_complex_solve_quadratic(double a, double b, double c, gsl_complex *z0, gsl_complex *z1)
{ (void)a; (void)b; (void)c; (void)z0; (void)z1; SHIM_ABORT("gsl_poly_complex_solve_quadratic"); return 0; }

static const gsl_root_fsolver_type shim_brent = { "brent (stand-in)" };
static const gsl_root_fdfsolver_type shim_newton = { "newton (stand-in)" };
static const gsl_multiroot_fsolver_type shim_hybrids = { "hybrids (stand-in)" };
const gsl_root_fsolver_type *gsl_root_fsolver_brent = &shim_brent;
const gsl_root_fdfsolver_type *gsl_root_fdfsolver_newton = &shim_newton;
const gsl_multiroot_fsolver_type *gsl_multiroot_fsolver_hybrids = &shim_hybrids;

gsl_root_fsolver *gsl_root_fsolver_alloc(const gsl_root_fsolver_type *T) { (void)T; SHIM_ABORT("gsl_root_fsolver_alloc"); return NULL; }
int gsl_root_fsolver_set(gsl_root_fsolver *s, gsl_function *f, double a, double b) { (void)s; (void)f; (void)a; (void)b; SHIM_ABORT("gsl_root_fsolver_set"); return 0; }
int gsl_root_fsolver_iterate(gsl_root_fsolver *s) { (void)s; SHIM_ABORT("gsl_root_fsolver_iterate"); return 0; }
double gsl_root_fsolver_root(const gsl_root_fsolver *s) { (void)s; SHIM_ABORT("gsl_root_fsolver_root"); return 0.; }
double gsl_root_fsolver_x_lower(const gsl_root_fsolver *s) { (void)s; SHIM_ABORT("gsl_root_fsolver_x_lower"); return 0.; }
double gsl_root_fsolver_x_upper(const gsl_root_fsolver *s) { (void)s; SHIM_ABORT("gsl_root_fsolver_x_upper"); return 0.; }
const char *gsl_root_fsolver_name(const gsl_root_fsolver *s) { (void)s; SHIM_ABORT("gsl_root_fsolver_name"); return ""; }
void gsl_root_fsolver_free(gsl_root_fsolver *s) { (void)s; SHIM_ABORT("gsl_root_fsolver_free"); }
gsl_root_fdfsolver *gsl_root_fdfsolver_alloc(const gsl_root_fdfsolver_type *T) { (void)T; SHIM_ABORT("gsl_root_fdfsolver_alloc"); return NULL; }
int gsl_root_fdfsolver_set(gsl_root_fdfsolver *s, gsl_function_fdf *f, double r) { (void)s; (void)f; (void)r; SHIM_ABORT("gsl_root_fdfsolver_set"); return 0; }
int gsl_root_fdfsolver_iterate(gsl_root_fdfsolver *s) { (void)s; SHIM_ABORT("gsl_root_fdfsolver_iterate"); return 0; }
double gsl_root_fdfsolver_root(const gsl_root_fdfsolver *s) { (void)s; SHIM_ABORT("gsl_root_fdfsolver_root"); return 0.; }
const char *gsl_root_fdfsolver_name(const gsl_root_fdfsolver *s) { (void)s; SHIM_ABORT("gsl_root_fdfsolver_name"); return ""; }
void gsl_root_fdfsolver_free(gsl_root_fdfsolver *s) { (void)s; SHIM_ABORT("gsl_root_fdfsolver_free"); }
int gsl_root_test_delta(double a, double b, double c, double d) { (void)a; (void)b; (void)c; (void)d; SHIM_ABORT("gsl_root_test_delta"); return 0; }
int gsl_root_test_interval(double a, double b, double c, double d) { (void)a; (void)b; (void)c; (void)d; SHIM_ABORT("gsl_root_test_interval"); return 0; }
gsl_multiroot_fsolver *gsl_multiroot_fsolver_alloc(const gsl_multiroot_fsolver_type *T, size_t n) { (void)T; (void)n; SHIM_ABORT("gsl_multiroot_fsolver_alloc"); return NULL; }
int gsl_multiroot_fsolver_set(gsl_multiroot_fsolver *s, gsl_multiroot_function *f, const gsl_vector *x) { (void)s; (void)f; (void)x; SHIM_ABORT("gsl_multiroot_fsolver_set"); return 0; }
int gsl_multiroot_fsolver_iterate(gsl_multiroot_fsolver *s) { (void)s; SHIM_ABORT("gsl_multiroot_fsolver_iterate"); return 0; }
void gsl_multiroot_fsolver_free(gsl_multiroot_fsolver *s) { (void)s; SHIM_ABORT("gsl_multiroot_fsolver_free"); }
int gsl_multiroot_test_residual(const gsl_vector *f, double e) { (void)f; (void)e; SHIM_ABORT("gsl_multiroot_test_residual"); return 0; }
int gsl_multiroot_test_delta(const gsl_vector *dx, const gsl_vector *x, double a, double r) { (void)dx; (void)x; (void)a; (void)r; SHIM_ABORT("gsl_multiroot_test_delta"); return 0; }
int gsl_deriv_central(const gsl_function *f, double x, double h, double *r, double *e) { (void)f; (void)x; (void)h; (void)r; (void)e; SHIM_ABORT("gsl_deriv_central"); return 0; }
