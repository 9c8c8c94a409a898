/*
 * Project-written stand-in for the subset of GSL that the reference program
 * PIC/3d_pic458_domain.c uses (its includes are at PIC/3d_pic458_domain.c:12-19).
 * TEST INFRASTRUCTURE ONLY: it exists so that the reference's own C source can be
 * compiled here as the CPU oracle. GSL itself is not installed and not vendored
 * under the reference (no version is pinned anywhere in the reference tree).
 *
 * What is restated and how it differs from GSL:
 *  - physical constants GSL_CONST_MKSA_* : taken from compile-time macros
 *    ORACLE_Q, ORACLE_MI, ... so that one build can run in MKSA units (the
 *    reference's own) and another in normalized units (c = e0 = mu0 = 1).
 *  - gsl_rng: NOT GSL's generators. Every generator object is a Philox4x32-10
 *    counter stream (Salmon et al., SC'11) keyed by its seed, so the GPU code can
 *    reproduce any draw by index. gsl_rng_uniform returns 53-bit uniforms in [0,1).
 *  - gsl_ran_flat(r,a,b) = a*(1-u) + b*u  (GSL's published formula).
 *  - gsl_ran_gaussian(r,s): Box-Muller with exactly two draws per call
 *    (GSL uses the polar method with rejection, whose draw count is random).
 *  - gsl_linalg_cholesky_decomp / gsl_blas_dgemv: textbook algorithms.
 *  - gsl_integration_qags: link stub returning an error; it is only reached
 *    from coil-field code that the time step never calls.
 */
#ifndef ORACLE_GSL_SHIM_H
#define ORACLE_GSL_SHIM_H

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---- constants (MKSA defaults; overridden per oracle build) ---- */
#ifndef ORACLE_Q
#define ORACLE_Q 1.602176487e-19
#endif
#ifndef ORACLE_MP
#define ORACLE_MP 1.672621637e-27
#endif
#ifndef ORACLE_ME
#define ORACLE_ME 9.10938188e-31
#endif
#ifndef ORACLE_MU0
#define ORACLE_MU0 1.25663706144e-6
#endif
#ifndef ORACLE_E0
#define ORACLE_E0 8.854187817e-12
#endif
#ifndef ORACLE_KB
#define ORACLE_KB 1.3806504e-23
#endif
#ifndef ORACLE_C
#define ORACLE_C 2.99792458e8
#endif

#define GSL_CONST_MKSA_ELECTRON_CHARGE ORACLE_Q
#define GSL_CONST_MKSA_MASS_PROTON ORACLE_MP
#define GSL_CONST_MKSA_MASS_ELECTRON ORACLE_ME
#define GSL_CONST_MKSA_VACUUM_PERMEABILITY ORACLE_MU0
#define GSL_CONST_MKSA_VACUUM_PERMITTIVITY ORACLE_E0
#define GSL_CONST_MKSA_BOLTZMANN ORACLE_KB
#define GSL_CONST_MKSA_SPEED_OF_LIGHT ORACLE_C

static inline double gsl_pow_2(const double x) { return x * x; }

/* ---- random numbers ---- */
typedef struct { const char *name; } gsl_rng_type;
typedef struct {
  const gsl_rng_type *type;
  uint64_t seed;     /* Philox key */
  uint64_t counter;  /* index of the next 53-bit draw */
} gsl_rng;

extern const gsl_rng_type *gsl_rng_rand;
extern const gsl_rng_type *gsl_rng_ranlxd2;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_free(gsl_rng *r);
void gsl_rng_set(gsl_rng *r, unsigned long int seed);
double gsl_rng_uniform(gsl_rng *r);
double gsl_ran_flat(const gsl_rng *r, double a, double b);
double gsl_ran_gaussian(const gsl_rng *r, double sigma);

/* Philox4x32-10 block and the 53-bit uniform for draw index d of stream seed. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double oracle_uniform53(uint64_t seed, uint64_t d);

/* ---- vectors / matrices ---- */
typedef struct { size_t size; size_t stride; double *data; int owner; } gsl_vector;
typedef struct { gsl_vector vector; } gsl_vector_view;
typedef struct { size_t size1, size2, tda; double *data; } gsl_matrix;

gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
double gsl_vector_get(const gsl_vector *v, size_t i);
gsl_vector_view gsl_vector_view_array(double *base, size_t n);

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);

typedef enum { CblasNoTrans = 111, CblasTrans = 112 } CBLAS_TRANSPOSE_t;
int gsl_blas_dgemv(CBLAS_TRANSPOSE_t TransA, double alpha, const gsl_matrix *A,
                   const gsl_vector *X, double beta, gsl_vector *Y);
int gsl_linalg_cholesky_decomp(gsl_matrix *A);

/* ---- integration (never reached on the time-step path) ---- */
typedef struct { double (*function)(double x, void *params); void *params; } gsl_function;
typedef struct { size_t limit; } gsl_integration_workspace;
gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n);
void gsl_integration_workspace_free(gsl_integration_workspace *w);
int gsl_integration_qags(const gsl_function *f, double a, double b, double epsabs,
                         double epsrel, size_t limit, gsl_integration_workspace *w,
                         double *result, double *abserr);

#endif
