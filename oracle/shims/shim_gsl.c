/*
 * GSL shim implementation -- TEST INFRASTRUCTURE (oracle only).
 * See gsl/gsl_rng.h, gsl/gsl_integration.h, gsl/gsl_sf_hyperg.h.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "gsl/gsl_rng.h"
#include "gsl/gsl_integration.h"
#include "gsl/gsl_sf_hyperg.h"

/* ------------------------------------------------------------ RANLUX-48 */

static const gsl_rng_type ranlxd1_type = {"ranlxd1", 202};
static const gsl_rng_type ranlxd2_type = {"ranlxd2", 397};
const gsl_rng_type* gsl_rng_ranlxd1 = &ranlxd1_type;
const gsl_rng_type* gsl_rng_ranlxd2 = &ranlxd2_type;

/* 2^-48: the resolution of one 48-bit word held as a double in [0,1). */
#define RLX_ULP (1.0 / 281474976710656.0)

gsl_rng* gsl_rng_alloc(const gsl_rng_type* T)
{
  gsl_rng* r = (gsl_rng*)calloc(1, sizeof(gsl_rng));
  r->type = T;
  gsl_rng_set(r, 0);
  return r;
}

void gsl_rng_free(gsl_rng* r) { free(r); }

void gsl_rng_set(gsl_rng* r, unsigned long int seed)
{
  if (seed == 0) seed = 1;
  /* 31-bit shift register: bit(n+31) = bit(n) xor bit(n+18). */
  int bits[31];
  unsigned long s = seed & 0xFFFFFFFFUL;
  for (int k = 0; k < 31; k++) { bits[k] = (int)(s & 1UL); s >>= 1; }
  int ib = 0, jb = 18;
  for (int w = 0; w < 12; w++) {
    double acc = 0.0;
    for (int l = 0; l < 48; l++) {
      acc = 2.0 * acc + (double)(bits[ib] ^ 1);
      bits[ib] ^= bits[jb];
      ib = (ib + 1) % 31;
      jb = (jb + 1) % 31;
    }
    r->x[w] = acc * RLX_ULP;
  }
  r->carry = 0.0;
  r->ir = 11;      /* the first draw advances to slot 0 and refills */
  r->jr = 7;       /* slot of the lag-5 word when slot 0 is written */
  r->ir_old = 0;
  r->pr = r->type->luxury;
}

/* Run pr subtract-with-borrow steps  y = x[k-5] - x[k-12] - carry (mod 1)
 * on the 12-word ring, starting at slot r->ir. */
static void rlx_refill(gsl_rng* r)
{
  int ir = r->ir, jr = r->jr;
  double carry = r->carry;
  for (unsigned k = 0; k < r->pr; k++) {
    double y = r->x[jr] - r->x[ir] - carry;
    if (y < 0.0) { carry = RLX_ULP; y += 1.0; }
    else carry = 0.0;
    r->x[ir] = y;
    ir = (ir + 1) % 12;
    jr = (jr + 1) % 12;
  }
  r->ir = ir;
  r->jr = jr;
  r->ir_old = ir;
  r->carry = carry;
}

double gsl_rng_uniform(gsl_rng* r)
{
  r->ir = (r->ir + 1) % 12;
  if (r->ir == r->ir_old) rlx_refill(r);
  return r->x[r->ir];
}

/* ------------------------------------------------------------ quadrature */

#define GL_N 20
static double gl_x[GL_N], gl_w[GL_N];
static int gl_ready = 0;

static void gl_init(void)
{
  /* Gauss-Legendre nodes by Newton iteration on P_n (Abramowitz & Stegun
   * 25.4.29), initial guesses cos(pi (i - 1/4)/(n + 1/2)). */
  const double pi = 3.14159265358979323846264338327950288;
  for (int i = 0; i < GL_N; i++) {
    double z = cos(pi * (i + 0.75) / (GL_N + 0.5));
    double pp = 0.0;
    for (int it = 0; it < 100; it++) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= GL_N; j++) {
        double p3 = p2; p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = GL_N * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (fabs(z - z1) < 1e-16) break;
    }
    gl_x[i] = z;
    gl_w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
  gl_ready = 1;
}

static double gl_panel(const gsl_function* f, double a, double b)
{
  const double c = 0.5 * (a + b), h = 0.5 * (b - a);
  double s = 0.0;
  for (int i = 0; i < GL_N; i++) s += gl_w[i] * f->function(c + h * gl_x[i], f->params);
  return s * h;
}

gsl_integration_workspace* gsl_integration_workspace_alloc(size_t n)
{
  gsl_integration_workspace* w = (gsl_integration_workspace*)malloc(sizeof(*w));
  w->limit = n;
  return w;
}

void gsl_integration_workspace_free(gsl_integration_workspace* w) { free(w); }

typedef struct { double a, b, val, err; } panel;

int gsl_integration_qag(const gsl_function* f, double a, double b,
                        double epsabs, double epsrel, size_t limit, int key,
                        gsl_integration_workspace* workspace,
                        double* result, double* abserr)
{
  (void)key;
  if (!gl_ready) gl_init();
  size_t cap = limit < 16 ? 16 : limit;
  if (workspace && workspace->limit < cap) cap = workspace->limit < 16 ? 16 : workspace->limit;
  panel* P = (panel*)malloc(sizeof(panel) * cap);
  size_t np = 1;
  P[0].a = a; P[0].b = b;
  P[0].val = gl_panel(f, a, b);
  {
    double m = 0.5 * (a + b);
    P[0].err = fabs(P[0].val - gl_panel(f, a, m) - gl_panel(f, m, b));
  }
  double tot = P[0].val, err = P[0].err;
  while (np < cap) {
    double tol = fmax(epsabs, 1e-3 * epsrel * fabs(tot));
    if (err <= tol) break;
    size_t imax = 0;
    for (size_t i = 1; i < np; i++) if (P[i].err > P[imax].err) imax = i;
    panel q = P[imax];
    double m = 0.5 * (q.a + q.b);
    panel l = {q.a, m, gl_panel(f, q.a, m), 0.0};
    panel r = {m, q.b, gl_panel(f, m, q.b), 0.0};
    double lm = 0.5 * (l.a + l.b), rm = 0.5 * (r.a + r.b);
    l.err = fabs(l.val - gl_panel(f, l.a, lm) - gl_panel(f, lm, l.b));
    r.err = fabs(r.val - gl_panel(f, r.a, rm) - gl_panel(f, rm, r.b));
    P[imax] = l;
    P[np++] = r;
    tot = 0.0; err = 0.0;
    for (size_t i = 0; i < np; i++) { tot += P[i].val; err += P[i].err; }
  }
  free(P);
  *result = tot;
  *abserr = err;
  return 0;
}

/* ------------------------------------------------------- hypergeometric */

static double f21_series(double a, double b, double c, double x)
{
  double term = 1.0, sum = 1.0;
  for (int n = 0; n < 100000; n++) {
    term *= (a + n) * (b + n) / ((c + n) * (n + 1.0)) * x;
    sum += term;
    if (fabs(term) < 1e-17 * fabs(sum)) break;
  }
  return sum;
}

double gsl_sf_hyperg_2F1(double a, double b, double c, double x)
{
  if (x < 0.0) {
    const double w = x / (x - 1.0);
    return pow(1.0 - x, -a) * f21_series(a, c - b, c, w);
  }
  return f21_series(a, b, c, x);
}
