/*
 * Implementation of the project-written GSL subset declared in gsl/gsl_shim.h.
 * TEST INFRASTRUCTURE ONLY (links into the compiled reference oracle).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "gsl/gsl_shim.h"

static const gsl_rng_type oracle_type_rand = {"philox-for-rand"};
static const gsl_rng_type oracle_type_ranlxd2 = {"philox-for-ranlxd2"};
const gsl_rng_type *gsl_rng_rand = &oracle_type_rand;
const gsl_rng_type *gsl_rng_ranlxd2 = &oracle_type_ranlxd2;

/* Philox4x32-10: Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11. Round multipliers and Weyl key increments as published. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Draw d of the stream keyed by seed: block d/2, word pair (d&1). */
double oracle_uniform53(uint64_t seed, uint64_t d)
{
  uint32_t ctr[4] = {(uint32_t)(d >> 1), (uint32_t)(d >> 33), 0u, 0u};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  oracle_philox4x32_10(ctr, key, o);
  const uint32_t a = (d & 1) ? o[2] : o[0];
  const uint32_t b = (d & 1) ? o[3] : o[1];
  const uint64_t m = ((uint64_t)a << 21) | (uint64_t)(b >> 11);
  return (double)m * (1.0 / 9007199254740992.0);
}

gsl_rng *gsl_rng_alloc(const gsl_rng_type *T)
{
  gsl_rng *r = (gsl_rng *)malloc(sizeof(gsl_rng));
  if (!r) return NULL;
  r->type = T;
  r->seed = 0;
  r->counter = 0;
  return r;
}

void gsl_rng_free(gsl_rng *r) { free(r); }

void gsl_rng_set(gsl_rng *r, unsigned long int seed)
{
  r->seed = (uint64_t)seed;
  r->counter = 0;
}

double gsl_rng_uniform(gsl_rng *r)
{
  const double u = oracle_uniform53(r->seed, r->counter);
  r->counter++;
  return u;
}

double gsl_ran_flat(const gsl_rng *r, double a, double b)
{
  const double u = gsl_rng_uniform((gsl_rng *)r);
  return a * (1.0 - u) + b * u;
}

double gsl_ran_gaussian(const gsl_rng *r, double sigma)
{
  const double u1 = 1.0 - gsl_rng_uniform((gsl_rng *)r); /* (0,1] */
  const double u2 = gsl_rng_uniform((gsl_rng *)r);
  return sigma * (sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2));
}

gsl_vector *gsl_vector_alloc(size_t n)
{
  gsl_vector *v = (gsl_vector *)malloc(sizeof(gsl_vector));
  v->size = n;
  v->stride = 1;
  v->data = (double *)calloc(n, sizeof(double));
  v->owner = 1;
  return v;
}

void gsl_vector_free(gsl_vector *v)
{
  if (!v) return;
  if (v->owner) free(v->data);
  free(v);
}

void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i * v->stride] = x; }
double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i * v->stride]; }

gsl_vector_view gsl_vector_view_array(double *base, size_t n)
{
  gsl_vector_view vv;
  vv.vector.size = n;
  vv.vector.stride = 1;
  vv.vector.data = base;
  vv.vector.owner = 0;
  return vv;
}

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2)
{
  gsl_matrix *m = (gsl_matrix *)malloc(sizeof(gsl_matrix));
  m->size1 = n1;
  m->size2 = n2;
  m->tda = n2;
  m->data = (double *)calloc(n1 * n2, sizeof(double));
  return m;
}

void gsl_matrix_free(gsl_matrix *m)
{
  if (!m) return;
  free(m->data);
  free(m);
}

void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) { m->data[i * m->tda + j] = x; }
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->tda + j]; }

/* y = alpha*op(A)*x + beta*y, BLAS semantics (beta == 0 ignores y's input). */
int gsl_blas_dgemv(CBLAS_TRANSPOSE_t TransA, double alpha, const gsl_matrix *A,
                   const gsl_vector *X, double beta, gsl_vector *Y)
{
  const size_t M = (TransA == CblasNoTrans) ? A->size1 : A->size2;
  const size_t N = (TransA == CblasNoTrans) ? A->size2 : A->size1;
  for (size_t i = 0; i < M; ++i) {
    double acc = 0.0;
    for (size_t j = 0; j < N; ++j) {
      const double a = (TransA == CblasNoTrans) ? gsl_matrix_get(A, i, j) : gsl_matrix_get(A, j, i);
      acc += a * gsl_vector_get(X, j);
    }
    const double y0 = (beta == 0.0) ? 0.0 : beta * gsl_vector_get(Y, i);
    gsl_vector_set(Y, i, y0 + alpha * acc);
  }
  return 0;
}

/* In-place Cholesky A = L L^T; the lower triangle holds L, the upper its transpose. */
int gsl_linalg_cholesky_decomp(gsl_matrix *A)
{
  const size_t n = A->size1;
  for (size_t j = 0; j < n; ++j) {
    double d = gsl_matrix_get(A, j, j);
    for (size_t k = 0; k < j; ++k) d -= gsl_matrix_get(A, j, k) * gsl_matrix_get(A, j, k);
    if (d <= 0.0) return 1;
    const double ljj = sqrt(d);
    gsl_matrix_set(A, j, j, ljj);
    for (size_t i = j + 1; i < n; ++i) {
      double s = gsl_matrix_get(A, i, j);
      for (size_t k = 0; k < j; ++k) s -= gsl_matrix_get(A, i, k) * gsl_matrix_get(A, j, k);
      gsl_matrix_set(A, i, j, s / ljj);
    }
  }
  for (size_t i = 0; i < n; ++i)
    for (size_t j = i + 1; j < n; ++j) gsl_matrix_set(A, i, j, gsl_matrix_get(A, j, i));
  return 0;
}

gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n)
{
  gsl_integration_workspace *w = (gsl_integration_workspace *)malloc(sizeof(*w));
  w->limit = n;
  return w;
}

void gsl_integration_workspace_free(gsl_integration_workspace *w) { free(w); }

int gsl_integration_qags(const gsl_function *f, double a, double b, double epsabs,
                         double epsrel, size_t limit, gsl_integration_workspace *w,
                         double *result, double *abserr)
{
  (void)f; (void)a; (void)b; (void)epsabs; (void)epsrel; (void)limit; (void)w;
  fprintf(stderr, "oracle shim: gsl_integration_qags is not available\n");
  *result = 0.0;
  *abserr = 0.0;
  return 1;
}
