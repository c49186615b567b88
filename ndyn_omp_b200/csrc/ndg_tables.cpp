// ndg_tables.cpp -- host tabulation of the pair potentials.
//
// Restates buildPairTables with pot()/dpot() (src/potentials.f90:2-247):
// for pair j, PTrc2 = rc^2, PTdr2 = (rc^2 - PTrMin)/(PTsize-1), and on the
// grid s_i = PTrMin + (i-1)*PTdr2 (i = 1..PTsize+1), r = sqrt(s_i):
//   PPairTable(i,j) = V(r),   FPairTable(i,j) = r * dpot(r).
// dpot is -dV/dr except for Morse, where it carries an extra 1/r
// (src/potentials.f90:197-198); the tables keep that, since the force loop
// (src/nd.f90:310) divides by r^2 and the reference's results depend on it.
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/ndyn_gpu.h"

namespace {

enum class Pot { none, sine, cosine, soft, spring, morse, buck, lj, john };

struct PairFn {
  Pot kind = Pot::none;
  bool coulomb = false;  // the 'C' variants add a damped shifted Coulomb term
};

PairFn classify(const std::string &n) {
  PairFn f;
  if (n == "sine") f.kind = Pot::sine;
  else if (n == "cosine") f.kind = Pot::cosine;
  else if (n == "soft") f.kind = Pot::soft;
  else if (n == "spring") f.kind = Pot::spring;
  else if (n == "morse" || n == "Morse" || n == "morsec" || n == "morseC" || n == "MorseC") {
    f.kind = Pot::morse;
    f.coulomb = (n == "MorseC" || n == "morseC");
  } else if (n == "Buck" || n == "BuckC" || n == "buck" || n == "buckC" || n == "buckc") {
    f.kind = Pot::buck;
    f.coulomb = (n == "BuckC");
  } else if (n == "LJ" || n == "LJC") {
    f.kind = Pot::lj;
    f.coulomb = (n == "LJC");
  } else if (n == "John") {
    f.kind = Pot::john;
  }
  return f;
}

constexpr double kPi = 3.141592653589793;
constexpr double kAlpha = 0.2;  // Coulomb damping, src/potentials.f90:10

double powi(double x, int n) {
  // integer power by squaring (Fortran x**n with a constant n)
  double r = 1.0, b = x;
  bool first = true;
  while (n > 0) {
    if (n & 1) {
      r = first ? b : r * b;
      first = false;
    }
    n >>= 1;
    if (n) b = b * b;
  }
  return r;
}

struct Dsf {
  double vcon, fcon;
  explicit Dsf(double rc) {
    const double rc2 = rc * rc;
    vcon = std::erfc(kAlpha * rc) / rc;
    fcon = (std::erfc(kAlpha * rc) / rc2 +
            2. * kAlpha / std::sqrt(kPi) * std::exp(-kAlpha * kAlpha * rc2) / rc);
  }
};

double energy(const PairFn &f, double r, const double *p, double q, const Dsf &c) {
  double v = 0.0;
  switch (f.kind) {
    case Pot::sine: v = std::sin(r) * std::sin(r) - 1.0; break;
    case Pot::cosine: v = std::cos(r) * std::cos(r) - 1.0; break;
    case Pot::soft: v = p[1] * (1.0 + std::cos(kPi * r / p[2])); break;
    case Pot::spring: {
      const double x = r / p[0] * p[2];
      v = p[1] * (x * x - p[2] * p[2]);
      break;
    }
    case Pot::morse: {
      double t = r - p[3];
      if (p[3] <= 0.0) t = 0.0;
      const double e = std::exp(-p[2] * t);
      v = p[1] * (e * e - 2.0 * e);
      break;
    }
    case Pot::buck:
      v = p[1] * std::exp(-r / p[2]) - p[3] / powi(r, 6);
      if (p[2] <= 0.0) v = p[1] - p[3] / powi(r, 6);
      break;
    case Pot::lj: {
      const double t = p[2] / r;
      v = 4. * p[1] * (powi(t, 12) - powi(t, 6));
      break;
    }
    case Pot::john: {
      const double A = 2. * powi(p[2], 3) / powi(p[3] - p[2], 3);
      const double B = 3. * powi(p[2], 2) / powi(p[3] - p[2], 2);
      const double t = (r - p[3]) / p[2];
      v = (r < p[3]) ? -p[1] * (A * powi(t, 3) + B * powi(t, 2)) : 0.0;
      break;
    }
    default: return NAN;
  }
  if (f.coulomb) v = v + q * (std::erfc(kAlpha * r) / r - c.vcon + c.fcon * (r - p[0]));
  return v;
}

double derivative(const PairFn &f, double r, const double *p, double q, const Dsf &c) {
  double d = 0.0;
  switch (f.kind) {
    case Pot::sine: d = std::sin(2.0 * r); break;
    case Pot::cosine: d = -std::sin(2.0 * r); break;
    case Pot::soft:  // parameters 1 and 2 here, 2 and 3 in the energy
      d = kPi * p[0] * std::sin(kPi * r / p[1]) / p[1];
      break;
    case Pot::spring: d = -2.0 * p[1] * (r / p[0] * p[2]); break;
    case Pot::morse: {
      double t = r - p[3];
      if (p[3] <= 0.0) t = 0.0;
      const double e = std::exp(-p[2] * t);
      d = 2. * p[1] * p[2] * (e * e - e) / r;
      break;
    }
    case Pot::buck:
      d = p[1] * std::exp(-r / p[2]) / p[2] - 6. * p[3] / powi(r, 7);
      if (p[2] <= 0.0) d = p[1] - 6. * p[3] / powi(r, 7);
      break;
    case Pot::lj: {
      const double t = p[2] / r;
      d = 24. * p[1] * (2. * powi(t, 12) / r - powi(t, 6) / r);
      break;
    }
    case Pot::john: {
      const double A = 2. * powi(p[2], 3) / powi(p[3] - p[2], 3);
      const double B = 3. * powi(p[2], 2) / powi(p[3] - p[2], 2);
      const double t = (r - p[3]) / p[2];
      d = (r < p[3]) ? p[1] / p[2] * (3. * A * powi(t, 2) + 2. * B * t) : 0.0;
      break;
    }
    default: return NAN;
  }
  if (f.coulomb)
    d = d + q * (std::erfc(kAlpha * r) / (r * r) +
                 2. * kAlpha / std::sqrt(kPi) * std::exp(-(kAlpha * kAlpha) * (r * r)) / r -
                 c.fcon);
  return d;
}

}  // namespace

extern "C" int ndg_build_pair_tables(int npairs, int ptsize, double ptrmin, const char *names,
                                     const double *params, const double *qprod, double *ppair,
                                     double *fpair, double *rc2, double *dr2) {
  if (npairs < 1 || ptsize < 2 || !names || !params || !ppair || !fpair) return NDG_ERR_ARG;
  for (int j = 0; j < npairs; ++j) {
    std::string nm(names + 8 * j, names + 8 * j + 8);
    while (!nm.empty() && (nm.back() == ' ' || nm.back() == '\0')) nm.pop_back();
    const PairFn f = classify(nm);
    if (f.kind == Pot::none) return NDG_ERR_POTENTIAL;
    const double *p = params + 4 * j;
    const double rc = p[0];
    const double q = qprod ? qprod[j] : 0.0;
    const Dsf c(rc);
    const double prc2 = rc * rc;
    const double pdr2 = (prc2 - ptrmin) / (ptsize - 1);
    if (rc2) rc2[j] = prc2;
    if (dr2) dr2[j] = pdr2;
    double *P = ppair + (size_t)(ptsize + 1) * j;
    double *F = fpair + (size_t)(ptsize + 1) * j;
    for (int i = 0; i <= ptsize; ++i) {
      const double s = ptrmin + (double)i * pdr2;
      const double r = std::sqrt(s);
      P[i] = energy(f, r, p, q, c);
      F[i] = r * derivative(f, r, p, q, c);
    }
  }
  return NDG_OK;
}
