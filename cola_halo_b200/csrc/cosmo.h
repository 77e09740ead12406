// Host-side double-precision cosmology for the COLA path (see cosmo.cpp).
#pragma once
#include <stddef.h>

#include <vector>

// Growth factors and COLA time coefficients (cola.c:156-292).
struct ColaTime {
  static constexpr double kNLPT = -2.5;   // cola.c:60
  float om32;    // Omega_m as the reference stores it (float)
  double Om;     // (double)om32
  double d1_norm, d2_norm;

  explicit ColaTime(double omega_m);
  double growth_temp(double a) const;
  double growth_d2_temp(double a) const;
  double D1(double a) const;       // growthD
  double D2(double a) const;       // growthD2
  double D2v(double a) const;      // growthD2v
  double Q(double a) const;        // Qfactor
  double DprimeQ(double a, double n_growth) const;
  double Sq(double ai, double af, double aref) const;
  double Sphi(double ai, double af, double aref) const;
  // cola.c:77-91 and cola.c:123-134: float coefficients of one kick / drift
  void kick(float a_v, float a_x, float avel1, float* dda, float* q1, float* q2) const;
  void drift(float a_x, float a_v, float apos1, float* dyyy, float* da1, float* da2) const;
};

// Tabulated k P(k) input spectrum (power.c:62-151).
struct PowerTable {
  std::vector<double> logk, logD;
  double norm = 1.0;
  bool read(const char* path, char* err, size_t errlen);
  double operator()(double k) const;        // PowerSpec
  double sigma2(double R) const;            // TopHatSigma2
};

// growth(a) of power.c:177-197 (Omega_k = 1 - Omega_m - Omega_Lambda).
double linear_growth(double a, double omega_m, double omega_lambda);
