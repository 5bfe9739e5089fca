// FP64 host-side basic state of the disk from complete elliptic integrals, and the map
// from physical sweep parameters (Q_min, M_d/M_*, softening/r, Gamma) to dg_params.
//
// Potential of the axisymmetric disk with the same scale-free softening as the Kalnajs
// kernel (kalnajs.hpp:7, K = (2 cosh du - 2 cos dphi + eps)^{-1/2}, i.e. in physical
// variables 1/sqrt(R^2 + R'^2 - 2 R R' cos phi + eps R R')):
//   Phi(R) = -G int Sigma0(R') R' I(R, R') dR',
//   I = int_0^{2pi} dphi / sqrt(A - B cos phi) = 4 K(m) / sqrt(A + B),
//   A = R^2 + R'^2 + eps R R', B = 2 R R', m = 2B / (A + B).
// (The same closed form as lka98/selfgravity.py:35-51, there with a field-point softening.)
// K(m), E(m) by the arithmetic-geometric mean; the R' integral by composite 16-point
// Gauss-Legendre on panels in u = ln R' refined around the field point.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "diskgpu.h"

namespace {

// Complete elliptic integrals of the first and second kind, parameter m = k^2 (AGM).
void ellipke(double m, double *K, double *E) {
  double a = 1.0, b = std::sqrt(1.0 - m), c = std::sqrt(m);
  double sum = 0.5 * c * c;  // 2^{n-1} c_n^2 with n = 0
  double p2 = 0.5;
  for (int n = 0; n < 60 && std::fabs(c) > 1e-17 * a; ++n) {
    double an = 0.5 * (a + b);
    double bn = std::sqrt(a * b);
    c = 0.5 * (a - b);
    a = an;
    b = bn;
    p2 *= 2.0;
    sum += p2 * c * c;
  }
  *K = M_PI / (2.0 * a);
  *E = *K * (1.0 - sum);
}

// 16-point Gauss-Legendre nodes / weights on [-1, 1] (Golub-Welsch, computed once)
struct GL16 {
  double x[16], w[16];
  GL16() {
    const int n = 16;
    for (int i = 0; i < n; ++i) {
      double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0;
      for (int it = 0; it < 100; ++it) {
        double p1 = 1.0, p2 = 0.0;
        for (int j = 1; j <= n; ++j) {
          double p3 = p2;
          p2 = p1;
          p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
        }
        pp = n * (z * p1 - p2) / (z * z - 1.0);
        double z1 = z;
        z = z1 - p1 / pp;
        if (std::fabs(z - z1) < 1e-16) break;
      }
      x[i] = z;
      w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
  }
};

const GL16 &gl16() {
  static GL16 g;
  return g;
}

struct Disk {
  double S0, R0, w2, eps, G, Rin, Rout;
  double sigma(double R) const { return S0 * std::exp(-(R - R0) * (R - R0) / w2); }
};

// Phi(R) and dPhi/dR of the softened disk (FP64).
void disk_potential(const Disk &d, double R, double *phi, double *dphidR) {
  const GL16 &g = gl16();
  const double umin = std::log(d.Rin), umax = std::log(d.Rout), u = std::log(R);
  // panel edges: uniform coarse panels plus geometric refinement toward u
  std::vector<double> edges;
  const int ncoarse = 48;
  for (int k = 0; k <= ncoarse; ++k) edges.push_back(umin + (umax - umin) * k / ncoarse);
  const double width = std::sqrt(d.eps > 1e-12 ? d.eps : 1e-12);
  for (int k = 0; k < 24; ++k) {
    double h = 0.5 * (umax - umin) * std::pow(0.6, k);
    if (h < 1e-3 * width) break;
    for (double e : {u - h, u + h})
      if (e > umin && e < umax) edges.push_back(e);
  }
  if (u > umin && u < umax) edges.push_back(u);
  std::sort(edges.begin(), edges.end());
  double P = 0.0, D = 0.0;
  for (size_t k = 0; k + 1 < edges.size(); ++k) {
    const double a = edges[k], b = edges[k + 1];
    if (b - a <= 0) continue;
    const double hm = 0.5 * (b - a), c = 0.5 * (a + b);
    for (int q = 0; q < 16; ++q) {
      const double up = c + hm * g.x[q];
      const double Rp = std::exp(up);
      const double wq = hm * g.w[q] * Rp;  // dR' = R' du'
      const double A = R * R + Rp * Rp + d.eps * R * Rp, B = 2.0 * R * Rp;
      const double S = A + B;
      const double m = 2.0 * B / S;
      double K, E;
      ellipke(m < 1.0 ? m : 1.0 - 1e-16, &K, &E);
      const double sq = std::sqrt(S);
      const double I = 4.0 * K / sq;
      // dI/dR
      const double dS = 2.0 * (R + Rp) + d.eps * Rp;
      const double dm = (4.0 * Rp * S - 4.0 * R * Rp * dS) / (S * S);
      const double dKdm = (E - (1.0 - m) * K) / (2.0 * m * (1.0 - m));
      const double dI = 4.0 * (dKdm * dm / sq - K * dS / (2.0 * S * sq));
      const double f = d.sigma(Rp) * Rp * wq;
      P += f * I;
      D += f * dI;
    }
  }
  *phi = -d.G * P;
  *dphidR = -d.G * D;
}

// vphi^2, kappa^2 and Toomre Q on radii R[0..n) (R increasing).  gdisk (may be NULL)
// supplies the disk force at those radii (it depends only on S0 and eps).
void rotation_curve(const dg_params &p, int n, const double *R, double *gR, double *vphi2, double *kappa2, double *Q,
                    const double *gdisk = nullptr) {
  Disk d{p.S0, p.R0, p.w2, p.eps, p.G, p.Rin, p.Rout};
  std::vector<double> L2(n), Om2(n);
  for (int i = 0; i < n; ++i) {
    double phi, dphi;
    double g = 0.0;
    if (gdisk) {
      g = gdisk[i];
    } else if (p.selfgrav) {
      disk_potential(d, R[i], &phi, &dphi);
      g = -dphi;
    }
    const double s0 = d.sigma(R[i]);
    const double dS = s0 * (-2.0 * (R[i] - p.R0) / p.w2);
    const double dPdR = p.Kpoly * p.gamma_gas * std::pow(s0, p.gamma_gas - 1.0) * dS;
    // diskmain.cpp:55: v^2 = GM/R + (R / Sigma0) dP/dR - R gR
    const double v2 = p.gmstar / R[i] + (R[i] / s0) * dPdR - R[i] * g;
    if (gR) gR[i] = g;
    if (vphi2) vphi2[i] = v2;
    Om2[i] = v2 / (R[i] * R[i]);
    L2[i] = std::pow(R[i], 4) * Om2[i];  // (R^2 Omega)^2
  }
  for (int i = 0; i < n; ++i) {
    // kappa^2 = R^{-3} d(R^4 Omega^2)/dR, centred differences (one-sided at the ends)
    int a = i > 0 ? i - 1 : i, b = i < n - 1 ? i + 1 : i;
    double k2 = (L2[b] - L2[a]) / (R[b] - R[a]) / (R[i] * R[i] * R[i]);
    if (kappa2) kappa2[i] = k2;
    if (Q) {
      const double s0 = d.sigma(R[i]);
      const double cs = std::sqrt(p.gamma_gas * p.Kpoly * std::pow(s0, p.gamma_gas - 1.0));
      Q[i] = cs * std::sqrt(k2 > 0 ? k2 : 0.0) / (M_PI * p.G * s0);
    }
  }
}

double disk_mass(const dg_params &p) {
  // 2 pi int R Sigma0 dR over [Rin, Rout], Gauss-Legendre on 64 panels
  const GL16 &g = gl16();
  double m = 0.0;
  const int np = 64;
  for (int k = 0; k < np; ++k) {
    double a = p.Rin + (p.Rout - p.Rin) * k / np, b = p.Rin + (p.Rout - p.Rin) * (k + 1) / np;
    double hm = 0.5 * (b - a), c = 0.5 * (a + b);
    for (int q = 0; q < 16; ++q) {
      double R = c + hm * g.x[q];
      m += hm * g.w[q] * 2.0 * M_PI * R * p.S0 * std::exp(-(R - p.R0) * (R - p.R0) / p.w2);
    }
  }
  return m;
}

// Minimum Toomre Q over the disk body (Sigma0 >= 0.1 S0; the tenuous Gaussian wings are
// excluded) and whether the equilibrium exists there (vphi^2 > 0 and kappa^2 > 0).
double qmin_of(const dg_params &p, int n, bool *valid, const double *gdisk) {
  std::vector<double> R(n), Q(n), v2(n), k2(n);
  for (int i = 0; i < n; ++i) R[i] = std::exp(std::log(p.Rin) + (i + 0.5) * std::log(p.Rout / p.Rin) / n);
  rotation_curve(p, n, R.data(), nullptr, v2.data(), k2.data(), Q.data(), gdisk);
  double q = 1e300;
  bool ok = true;
  for (int i = 0; i < n; ++i) {
    if (std::exp(-(R[i] - p.R0) * (R[i] - p.R0) / p.w2) < 0.1) continue;
    if (!(v2[i] > 0) || !(k2[i] > 0)) ok = false;
    if (Q[i] < q) q = Q[i];
  }
  if (valid) *valid = ok;
  return q;
}

}  // namespace

extern "C" {

int dg_rotation_curve_elliptic(const dg_params *p, int n, const double *R, double *gR, double *vphi2,
                               double *kappa2, double *Q) {
  if (!p || !R || n < 2 || !(p->Rin > 0) || !(p->Rout > p->Rin) || !(p->eps >= 0)) return DG_ERR_INVALID;
  for (int i = 0; i < n; ++i)
    if (!(R[i] > 0)) return DG_ERR_INVALID;
  rotation_curve(*p, n, R, gR, vphi2, kappa2, Q);
  return DG_OK;
}

int dg_params_physical(double Qmin, double mass_ratio, double soft_over_r, double gamma_gas, dg_params *p,
                       double *Qmin_achieved) {
  if (!p || !(Qmin > 0) || !(mass_ratio > 0) || !(soft_over_r >= 0) || !(gamma_gas > 1.0)) return DG_ERR_INVALID;
  p->gamma_gas = gamma_gas;
  p->eps = soft_over_r * soft_over_r;  // kernel softening eps R R' = (s/r)^2 R R'
  // S0 so that m_D = mass_ratio * m_* (G M_* = gmstar, G = 1)
  dg_params q = *p;
  q.S0 = 1.0;
  const double m1 = disk_mass(q);
  p->S0 = mass_ratio * (p->gmstar / p->G) / m1;
  const int n = 96;
  dg_params t = *p;
  // the disk force depends on S0 and eps only: evaluate it once for the whole search
  std::vector<double> Rg(n), gd(n, 0.0);
  for (int i = 0; i < n; ++i) Rg[i] = std::exp(std::log(p->Rin) + (i + 0.5) * std::log(p->Rout / p->Rin) / n);
  if (p->selfgrav) rotation_curve(*p, n, Rg.data(), gd.data(), nullptr, nullptr, nullptr);
  const double *gdp = gd.data();
  // largest K for which the equilibrium exists over the disk body
  double lo = std::log(1e-5), hi = std::log(20.0);
  bool valid = false;
  t.Kpoly = std::exp(hi);
  qmin_of(t, n, &valid, gdp);
  if (!valid) {
    double a = lo, b = hi;
    for (int it = 0; it < 60; ++it) {
      double mid = 0.5 * (a + b);
      t.Kpoly = std::exp(mid);
      qmin_of(t, n, &valid, gdp);
      if (valid) a = mid; else b = mid;
    }
    hi = a;
  }
  // Q_min(K) rises with the sound speed and then falls as pressure support erodes kappa:
  // locate its maximum on [lo, hi] (golden section on log K), then bisect below it
  {
    const double gr = 0.5 * (std::sqrt(5.0) - 1.0);
    double a = lo, b = hi;
    double c = b - gr * (b - a), d = a + gr * (b - a);
    auto qat = [&](double lk) { t.Kpoly = std::exp(lk); return qmin_of(t, n, nullptr, gdp); };
    double fc = qat(c), fd = qat(d);
    for (int it = 0; it < 60; ++it) {
      if (fc > fd) { b = d; d = c; fd = fc; c = b - gr * (b - a); fc = qat(c); }
      else { a = c; c = d; fc = fd; d = a + gr * (b - a); fd = qat(d); }
    }
    hi = 0.5 * (a + b);
  }
  t.Kpoly = std::exp(hi);
  double qcap = qmin_of(t, n, nullptr, gdp);
  if (qcap <= Qmin) {
    p->Kpoly = t.Kpoly;
    if (Qmin_achieved) *Qmin_achieved = qcap;
    return DG_OK;
  }
  for (int it = 0; it < 80; ++it) {
    double mid = 0.5 * (lo + hi);
    t.Kpoly = std::exp(mid);
    double qm = qmin_of(t, n, nullptr, gdp);
    if (qm < Qmin) lo = mid; else hi = mid;
  }
  p->Kpoly = std::exp(0.5 * (lo + hi));
  t.Kpoly = p->Kpoly;
  if (Qmin_achieved) *Qmin_achieved = qmin_of(t, n, nullptr, gdp);
  return DG_OK;
}

}  // extern "C"
