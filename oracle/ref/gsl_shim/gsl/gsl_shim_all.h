/*
 * Declaration-only stand-in for the GNU Scientific Library headers.
 *
 * Test infrastructure: it exists so that the reference KORAL sources can be
 * compiled into the parity oracle on a machine without GSL.  No GSL
 * arithmetic sits on the hot path that the oracle exercises (the 4x4
 * inverse the implicit solver uses is KORAL's own cofactor routine,
 * misc.c:502-602).  Every function declared here is defined in
 * gsl_shim.c; all but the error-handler switch abort when reached, so a
 * run that strays off the hot path fails loudly instead of computing
 * something different.
 *
 * Only type layouts and prototypes are provided, written for this build.
 */
#ifndef KORAL_ORACLE_GSL_SHIM_ALL_H
#define KORAL_ORACLE_GSL_SHIM_ALL_H

#include <stddef.h>
#include <stdio.h>
#include <float.h>

#define GSL_SUCCESS 0
#define GSL_FAILURE (-1)
#define GSL_CONTINUE (-2)
#define GSL_MAX(a, b) ((a) > (b) ? (a) : (b))
#define GSL_MIN(a, b) ((a) < (b) ? (a) : (b))

typedef struct { double dat[2]; } gsl_complex;
#define GSL_REAL(z) ((z).dat[0])
#define GSL_IMAG(z) ((z).dat[1])
#define GSL_SET_COMPLEX(zp, x, y) do { (zp)->dat[0] = (x); (zp)->dat[1] = (y); } while (0)

typedef struct { size_t size; size_t stride; double *data; } gsl_vector;
typedef struct { size_t size1; size_t size2; size_t tda; double *data; } gsl_matrix;
typedef struct { gsl_matrix matrix; } gsl_matrix_view;
typedef struct { gsl_vector vector; } gsl_vector_view;
typedef struct { size_t size; size_t stride; double *data; } gsl_vector_complex;
typedef struct { size_t size; size_t *data; } gsl_permutation;

typedef struct { double (*function)(double x, void *params); void *params; } gsl_function;
typedef struct {
  double (*f)(double x, void *params);
  double (*df)(double x, void *params);
  void (*fdf)(double x, void *params, double *f, double *df);
  void *params;
} gsl_function_fdf;
typedef struct {
  int (*f)(const gsl_vector *x, void *params, gsl_vector *f);
  size_t n;
  void *params;
} gsl_multiroot_function;

typedef struct { const char *name; } gsl_root_fsolver_type;
typedef struct { const char *name; } gsl_root_fdfsolver_type;
typedef struct { const char *name; } gsl_multiroot_fsolver_type;
typedef struct { const gsl_root_fsolver_type *type; double root, x_lower, x_upper; } gsl_root_fsolver;
typedef struct { const gsl_root_fdfsolver_type *type; double root; } gsl_root_fdfsolver;
typedef struct { const gsl_multiroot_fsolver_type *type; gsl_vector *x, *f, *dx; } gsl_multiroot_fsolver;

typedef struct { size_t n; } gsl_eigen_symm_workspace;
typedef struct { size_t n; } gsl_eigen_symmv_workspace;
typedef struct { size_t n; } gsl_eigen_nonsymm_workspace;
typedef struct { const char *name; } gsl_rng_type;
typedef struct { const gsl_rng_type *type; } gsl_rng;
typedef struct { size_t size; } gsl_spline;
typedef struct { size_t size; } gsl_interp_accel;

enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_TRANSPOSE CBLAS_TRANSPOSE_t;

typedef void gsl_error_handler_t(const char *reason, const char *file, int line, int gsl_errno);
gsl_error_handler_t *gsl_set_error_handler_off(void);
const char *gsl_strerror(const int gsl_errno);

gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
int gsl_vector_fprintf(FILE *stream, const gsl_vector *v, const char *format);
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);
gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2);
gsl_vector_view gsl_matrix_column(gsl_matrix *m, size_t j);
gsl_vector_complex *gsl_vector_complex_alloc(size_t n);
void gsl_vector_complex_free(gsl_vector_complex *v);
gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, size_t i);
gsl_permutation *gsl_permutation_alloc(size_t n);
void gsl_permutation_free(gsl_permutation *p);

int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum);
int gsl_linalg_LU_invert(const gsl_matrix *LU, const gsl_permutation *p, gsl_matrix *inverse);
int gsl_linalg_cholesky_decomp(gsl_matrix *A);
int gsl_linalg_cholesky_invert(gsl_matrix *LLT);
int gsl_blas_dgemm(CBLAS_TRANSPOSE_t TransA, CBLAS_TRANSPOSE_t TransB, double alpha,
                   const gsl_matrix *A, const gsl_matrix *B, double beta, gsl_matrix *C);

gsl_eigen_symm_workspace *gsl_eigen_symm_alloc(const size_t n);
void gsl_eigen_symm_free(gsl_eigen_symm_workspace *w);
int gsl_eigen_symm(gsl_matrix *A, gsl_vector *eval, gsl_eigen_symm_workspace *w);
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(const size_t n);
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w);
gsl_eigen_nonsymm_workspace *gsl_eigen_nonsymm_alloc(const size_t n);
void gsl_eigen_nonsymm_free(gsl_eigen_nonsymm_workspace *w);
int gsl_eigen_nonsymm(gsl_matrix *A, gsl_vector_complex *eval, gsl_eigen_nonsymm_workspace *w);

gsl_complex gsl_complex_add(gsl_complex a, gsl_complex b);
gsl_complex gsl_complex_sub(gsl_complex a, gsl_complex b);
gsl_complex gsl_complex_mul(gsl_complex a, gsl_complex b);
gsl_complex gsl_complex_mul_real(gsl_complex a, double x);
gsl_complex gsl_complex_add_real(gsl_complex a, double x);
gsl_complex gsl_complex_negative(gsl_complex a);
gsl_complex gsl_complex_sqrt(gsl_complex z);
gsl_complex gsl_complex_sqrt_real(double x);
gsl_complex gsl_complex_inverse(gsl_complex a);
gsl_complex gsl_complex_conjugate(gsl_complex z);
double gsl_complex_abs(gsl_complex z);
int gsl_poly_complex_solve_quadratic(double a, double b, double c, gsl_complex *z0, gsl_complex *z1);
int gsl_poly_complex_solve_quartic(double a, double b, double c, double d,
                                   gsl_complex *z0, gsl_complex *z1, gsl_complex *z2, gsl_complex *z3);

extern const gsl_root_fsolver_type *gsl_root_fsolver_brent;
extern const gsl_root_fdfsolver_type *gsl_root_fdfsolver_newton;
extern const gsl_multiroot_fsolver_type *gsl_multiroot_fsolver_hybrids;
gsl_root_fsolver *gsl_root_fsolver_alloc(const gsl_root_fsolver_type *T);
int gsl_root_fsolver_set(gsl_root_fsolver *s, gsl_function *f, double x_lower, double x_upper);
int gsl_root_fsolver_iterate(gsl_root_fsolver *s);
double gsl_root_fsolver_root(const gsl_root_fsolver *s);
double gsl_root_fsolver_x_lower(const gsl_root_fsolver *s);
double gsl_root_fsolver_x_upper(const gsl_root_fsolver *s);
const char *gsl_root_fsolver_name(const gsl_root_fsolver *s);
void gsl_root_fsolver_free(gsl_root_fsolver *s);
gsl_root_fdfsolver *gsl_root_fdfsolver_alloc(const gsl_root_fdfsolver_type *T);
int gsl_root_fdfsolver_set(gsl_root_fdfsolver *s, gsl_function_fdf *fdf, double root);
int gsl_root_fdfsolver_iterate(gsl_root_fdfsolver *s);
double gsl_root_fdfsolver_root(const gsl_root_fdfsolver *s);
const char *gsl_root_fdfsolver_name(const gsl_root_fdfsolver *s);
void gsl_root_fdfsolver_free(gsl_root_fdfsolver *s);
int gsl_root_test_delta(double x1, double x0, double epsabs, double epsrel);
int gsl_root_test_interval(double x_lower, double x_upper, double epsabs, double epsrel);
gsl_multiroot_fsolver *gsl_multiroot_fsolver_alloc(const gsl_multiroot_fsolver_type *T, size_t n);
int gsl_multiroot_fsolver_set(gsl_multiroot_fsolver *s, gsl_multiroot_function *f, const gsl_vector *x);
int gsl_multiroot_fsolver_iterate(gsl_multiroot_fsolver *s);
void gsl_multiroot_fsolver_free(gsl_multiroot_fsolver *s);
int gsl_multiroot_test_residual(const gsl_vector *f, double epsabs);
int gsl_multiroot_test_delta(const gsl_vector *dx, const gsl_vector *x, double epsabs, double epsrel);
int gsl_deriv_central(const gsl_function *f, double x, double h, double *result, double *abserr);

#endif
