// Host-side double-precision time coefficients of the COLA integrator and
// the linear power spectrum / growth used by the 2LPT setup.
//
// cola.c:156-292 evaluates the growth factors in a float/double mix; here the
// same formulas are evaluated in double (branch decisions are taken on the
// single-precision values the reference branches on, so the same branch of
// its piecewise growth formula is used for the same scale factor).
// power.c:62-222 (table reader, log-log interpolation, linear growth, sigma_8
// check) is restated in double.
#include "cosmo.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

namespace {

// Gauss hypergeometric series, with Pfaff's transformation
// 2F1(a,b;c;x) = (1-x)^(-a) 2F1(a,c-b;c;x/(x-1)) for x < 0 so that the
// series argument lies in [0, 1/2] (Abramowitz & Stegun 15.3.4, 15.1.1).
double f21_series(double a, double b, double c, double x) {
  double term = 1.0, sum = 1.0;
  for (int n = 0; n < 200000; n++) {
    term *= (a + n) * (b + n) / ((c + n) * (n + 1.0)) * x;
    sum += term;
    if (fabs(term) <= 1e-17 * fabs(sum)) break;
  }
  return sum;
}

double hyp2f1(double a, double b, double c, double x) {
  if (x < 0.0) return pow(1.0 - x, -a) * f21_series(a, c - b, c, x / (x - 1.0));
  return f21_series(a, b, c, x);
}

// Gauss-Legendre panels (20 nodes) by Newton iteration on P_20.
struct GL {
  double x[20], w[20];
  GL() {
    const int n = 20;
    for (int i = 0; i < n; i++) {
      double z = cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0.0;
      for (int it = 0; it < 100; it++) {
        double p1 = 1.0, p2 = 0.0;
        for (int j = 1; j <= n; j++) {
          double p3 = p2;
          p2 = p1;
          p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
        }
        pp = n * (z * p1 - p2) / (z * z - 1.0);
        double z1 = z;
        z = z1 - p1 / pp;
        if (fabs(z - z1) < 1e-16) break;
      }
      x[i] = z;
      w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
  }
};
const GL& gl() {
  static GL g;
  return g;
}

template <class F>
double panel(const F& f, double a, double b) {
  const GL& g = gl();
  const double c = 0.5 * (a + b), h = 0.5 * (b - a);
  double s = 0.0;
  for (int i = 0; i < 20; i++) s += g.w[i] * f(c + h * g.x[i]);
  return s * h;
}

// Globally adaptive bisection on Gauss-Legendre panels to relative
// tolerance rel (absolute floor abs_tol).
template <class F>
double integrate(const F& f, double a, double b, double rel, double abs_tol = 0.0) {
  struct P { double a, b, v, e; };
  std::vector<P> ps;
  auto mk = [&](double lo, double hi) {
    double m = 0.5 * (lo + hi);
    double v = panel(f, lo, hi);
    double e = fabs(v - panel(f, lo, m) - panel(f, m, hi));
    return P{lo, hi, v, e};
  };
  ps.push_back(mk(a, b));
  for (int it = 0; it < 4000; it++) {
    double tot = 0.0, err = 0.0;
    size_t imax = 0;
    for (size_t i = 0; i < ps.size(); i++) {
      tot += ps[i].v;
      err += ps[i].e;
      if (ps[i].e > ps[imax].e) imax = i;
    }
    if (err <= fmax(abs_tol, rel * fabs(tot))) return tot;
    P q = ps[imax];
    double m = 0.5 * (q.a + q.b);
    ps[imax] = mk(q.a, m);
    ps.push_back(mk(m, q.b));
  }
  double tot = 0.0;
  for (auto& p : ps) tot += p.v;
  return tot;
}

}  // namespace

// --------------------------------------------------------------- COLA time
ColaTime::ColaTime(double omega_m) {
  om32 = (float)omega_m;                // cola.c:83  Om is a float
  Om = (double)om32;
  d1_norm = growth_temp(1.0);
  d2_norm = growth_d2_temp(1.0);
}

// growthDtemp (cola.c:156-194) in double.
double ColaTime::growth_temp(double a) const {
  const float a32 = (float)a;
  const float x32 = (float)(-(double)om32 / ((double)om32 - 1.0) / (double)(a32 * a32 * a32));
  const double x = -Om / (Om - 1.0) / (a * a * a);
  double hp = 0.0, hm = 0.0;
  if (fabs((double)x32 - 1.0) < 1.e-3) {
    const double t = x - 1.0;
    hp = 0.859596768064608 - 0.1016599912520404 * t + 0.025791094277821357 * pow(t, 2) -
         0.008194025861121475 * pow(t, 3) + 0.0029076305993447644 * pow(t, 4) -
         0.0011025426387159761 * pow(t, 5) + 0.00043707304964624546 * pow(t, 6) -
         0.0001788889964687831 * pow(t, 7);
    hm = 1.1765206505266006 + 0.15846194123099624 * t - 0.014200487494738975 * pow(t, 2) +
         0.002801728034399257 * pow(t, 3) - 0.0007268267888593511 * pow(t, 4) +
         0.00021801569226706922 * pow(t, 5) - 0.00007163321597397065 * pow(t, 6) +
         0.000025063737576245116 * pow(t, 7);
  } else {
    if ((double)x32 < 1.0) {
      hp = hyp2f1(1.0 / 2.0, 2.0 / 3.0, 5.0 / 3.0, -x);
      hm = hyp2f1(-1.0 / 2.0, 2.0 / 3.0, 5.0 / 3.0, -x);
    }
    const float xi32 = (float)(1.0 / (double)x32);
    const double xi = 1.0 / x;
    if (((double)xi32 < 1.0) && ((double)xi32 > 1.0 / 30)) {
      hp = hyp2f1(-1.0 / 6.0, 0.5, 5.0 / 6.0, -xi);
      hp *= 4 * sqrt(xi);
      hp += -3.4494794123063873799 * pow(xi, 2.0 / 3.0);
      hm = hyp2f1(-7.0 / 6.0, -0.5, -1.0 / 6.0, -xi);
      hm *= 4.0 / 7.0 / sqrt(xi);
      hm += pow(xi, 2.0 / 3.0) * (-1.4783483195598803057);
    }
    if ((double)xi32 <= 1.0 / 30.0) {
      hp = 3.9999999999999996 * sqrt(xi) - 3.4494794123063865 * pow(xi, 0.6666666666666666) +
           0.3999999999999999 * pow(xi, 1.5) - 0.13636363636363635 * pow(xi, 2.5) +
           0.07352941176470587 * pow(xi, 3.5) - 0.04755434782608695 * pow(xi, 4.5) +
           0.033943965517241374 * pow(xi, 5.5) - 0.02578125 * pow(xi, 6.5) +
           0.020436356707317072 * pow(xi, 7.5) - 0.01671324384973404 * pow(xi, 8.5) +
           0.013997779702240564 * pow(xi, 9.5) - 0.011945562847590041 * pow(xi, 10.5) +
           0.01035003662109375 * pow(xi, 11.5) - 0.009080577904069926 * pow(xi, 12.5);
      hm = 0.5714285714285715 / sqrt(xi) + 2.000000000000001 * sqrt(xi) -
           1.4783483195598794 * pow(xi, 0.66666666666666666) +
           0.10000000000000002 * pow(xi, 1.5) - 0.022727272727272735 * pow(xi, 2.5) +
           0.009191176470588237 * pow(xi, 3.5) - 0.004755434782608697 * pow(xi, 4.5) +
           0.002828663793103449 * pow(xi, 5.5) - 0.0018415178571428578 * pow(xi, 6.5) +
           0.0012772722942073172 * pow(xi, 7.5) - 0.0009285135472074472 * pow(xi, 8.5) +
           0.0006998889851120285 * pow(xi, 9.5) - 0.0005429801294359111 * pow(xi, 10.5) +
           0.0004312515258789064 * pow(xi, 11.5) - 0.00034925299631038194 * pow(xi, 12.5);
    }
  }
  if ((double)a32 > 0.2)
    return sqrt(1.0 + (-1.0 + pow(a, -3)) * Om) *
           (3.4494794123063873799 * pow(-1.0 + 1.0 / Om, 0.666666666666666666666666666) +
            (hp * (4 * pow(a, 3) * (-1.0 + Om) - Om) - 7.0 * pow(a, 3) * hm * (-1.0 + Om)) /
                (pow(a, 5) * (-1.0 + Om) - pow(a, 2) * Om));
  return (a * pow(1 - Om, 1.5) *
          (1291467969.0 * pow(a, 12) * pow(-1 + Om, 4) +
           1956769650.0 * pow(a, 9) * pow(-1 + Om, 3) * Om +
           8000000000.0 * pow(a, 3) * (-1 + Om) * pow(Om, 3) + 37490640625.0 * pow(Om, 4))) /
         (1.5625e10 * pow(Om, 5));
}

double ColaTime::D1(double a) const { return growth_temp(a) / d1_norm; }

double ColaTime::Q(double a) const { return sqrt(Om / (a * a * a) + 1.0 - Om) * a * a * a; }

double ColaTime::growth_d2_temp(double a) const {
  const double d = D1(a);
  const double omega = Om / (Om + (1.0 - Om) * a * a * a);
  return d * d * pow(omega, -1.0 / 143.);
}

double ColaTime::D2(double a) const { return growth_d2_temp(a) / d2_norm; }

double ColaTime::D2v(double a) const {
  const double omega = Om / (Om + (1.0 - Om) * a * a * a);
  return Q(a) * (D2(a) / a) * 2.0 * pow(omega, 6.0 / 11.);
}

double ColaTime::DprimeQ(double a, double n_growth) const {
  const double n_decay = 0.0;
  const double nn = 6.0 * pow(1.0 - Om, 1.5) / d1_norm;
  const double decay = sqrt(Om / (a * a * a) + 1.0 - Om);
  const double d = D1(a);
  return pow(decay, -1.0 + n_decay) * pow(d, -1.0 + n_growth) *
         (n_growth * nn - (3.0 * (n_decay + n_growth) * Om * d) / (2. * a));
}

double ColaTime::Sq(double ai, double af, double aref) const {
  const double n = kNLPT;
  auto f = [&](double a) { return pow(a, n) / Q(a); };
  return integrate(f, ai, af, 1e-13) / pow(aref, n);
}

double ColaTime::Sphi(double ai, double af, double aref) const {
  const double n = kNLPT;
  return (pow(af, n) - pow(ai, n)) * aref / Q(aref) / (n * pow(aref, n - 1));
}

void ColaTime::kick(float a_v, float a_x, float avel1, float* dda, float* q1, float* q2) const {
  const double AI = a_v, A = a_x, AF = avel1;
  const double om143 = pow(Om / (Om + (1 - Om) * A * A * A), 1.0 / 143.0);
  const double g1 = D1(A);
  *dda = (float)Sphi(AI, AF, A);
  *q2 = (float)(1.5 * Om * g1 * g1 * (1.0 + 7.0 / 3.0 * om143));
  *q1 = (float)(1.5 * Om * g1);
}

void ColaTime::drift(float a_x, float a_v, float apos1, float* dyyy, float* da1,
                     float* da2) const {
  const double A = a_x, AC = a_v, AF = apos1;
  *dyyy = (float)Sq(A, AF, AC);
  *da1 = (float)(D1(AF) - D1(A));
  *da2 = (float)(D2(AF) - D2(A));
}

// ------------------------------------------------------- power spectrum
bool PowerTable::read(const char* path, char* err, size_t errlen) {
  FILE* fp = fopen(path, "r");
  if (!fp) {
    snprintf(err, errlen, "unable to read input power spectrum: %s", path);
    return false;
  }
  logk.clear();
  logD.clear();
  const double fac = 1.0 / (2.0 * M_PI * M_PI);
  double k, p;
  while (fscanf(fp, " %lg %lg ", &k, &p) == 2) {      // power.c:88-97
    logk.push_back(log10(k));
    logD.push_back(log10(fac * k * k * k * p));
  }
  fclose(fp);
  if (logk.size() < 2) {
    snprintf(err, errlen, "power spectrum table %s has fewer than 2 rows", path);
    return false;
  }
  return true;
}

double PowerTable::operator()(double k) const {       // power.c:120-151
  const double lk = log10(k);
  const int n = (int)logk.size();
  if (lk < logk[0] || lk > logk[n - 1]) return 0;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    int mid = (hi + lo) / 2;
    if (lk < logk[mid]) hi = mid;
    else lo = mid;
  }
  const double u = (lk - logk[lo]) / (logk[hi] - logk[lo]);
  const double ld = (1 - u) * logD[lo] + u * logD[hi];
  return norm * pow(10.0, ld) / (4.0 * M_PI * k * k * k);
}

double PowerTable::sigma2(double R) const {           // power.c:155-170, 204-222
  auto f = [&](double k) {
    const double kr = R * k;
    if (kr < 1e-8) return 0.0;
    const double w = 3 * (sin(kr) / (kr * kr * kr) - cos(kr) / (kr * kr));
    return 4 * M_PI * k * k * w * w * (*this)(k);
  };
  // integrate piecewise between table nodes (the integrand has kinks there)
  double tot = 0.0, lo = 0.0;
  const double hi = 500.0 / R;
  for (size_t i = 0; i < logk.size() && lo < hi; i++) {
    double kn = pow(10.0, logk[i]);
    if (kn <= lo) continue;
    if (kn > hi) kn = hi;
    tot += integrate(f, lo, kn, 1e-10, 1e-300);
    lo = kn;
  }
  if (lo < hi) tot += integrate(f, lo, hi, 1e-10, 1e-300);
  return tot;
}

double linear_growth(double a, double omega_m, double omega_lambda) {  // power.c:177-197
  const double ok = 1 - omega_m - omega_lambda;
  const double h = sqrt(omega_m / (a * a * a) + ok / (a * a) + omega_lambda);
  auto f = [&](double x) { return pow(x / (omega_m + ok * x + omega_lambda * x * x * x), 1.5); };
  return h * integrate(f, 0.0, a, 1e-13);
}
