// forcing.cpp -- Eswaran-Pope stochastic forcing, host side.
//
// Restates PSDNS/force.f:60-166 (velocity increments of all modes with
// 0 < |k| <= kforce, mapped onto a solenoidal vector, kx = 0 plane made
// conjugate-symmetric), PSDNS/vfuo.f (Uhlenbeck-Ornstein processes),
// PSDNS/vfiuo.f + PSDNS/raniuo.f (integrated UO processes) and the Gaussian
// generator PSDNS/rann2.f (table inversion, ntab = 201) with its uniform
// source PSDNS/ranu2.f / PSDNS/vrand.f, which share the ranu LCG state.
// The table for(kfor,k2fo,k2fo,3) is a few hundred complex numbers; it is
// built here once per step and copied to the device, where the stage
// kernel adds it to the forced modes (proc4a.f:588-651, proc4b.f:118-163).
#include <cmath>
#include <cstdio>
#include <vector>

#include "psdns_host.h"

namespace psdns {

// erff of rann2.f:238-254 (Abramowitz & Stegun 7.1.26)
static double erf_as(double x) {
  const double p = .3275911, a1 = .254829592, a2 = -.284496736, a3 = 1.421413741, a4 = -1.453152027,
               a5 = 1.061405429;
  double t = 1. / (1. + p * std::fabs(x));
  double q = t * (a1 + t * (a2 + t * (a3 + t * (a4 + t * a5))));
  double e = 1. - q * std::exp(-x * x);
  if (x < 0.) e = -e;
  return e;
}

// rann2.f:149-226: table of the standard normal inverse distribution
void Rann2::init() {
  const int ntab = 201;
  const double pi = 3.1415927, rtpii = 0.3989423, rti = 0.7071068;
  auto fdens = [&](double xx) { return rtpii * std::exp(-0.5 * xx * xx); };
  auto fdist = [&](double xx) { return 0.5 * (1. + erf_as(rti * xx)); };
  tab.assign(ntab + 1, 0.0);   // 1-based
  dtab.assign(ntab + 1, 0.0);
  ntabm = ntab - 1;
  const int ntabmm = ntabm - 1;
  const int ntsq = ntab * ntab;
  const double dy = 1. / double(ntabm);
  const double p3 = ntsq * 5.800e-6 - ntab * 4.35160e-3 - 1.7006542;
  const double p2 = ntsq * 6.035e-6 - ntab * 4.46257e-3 - 1.8738435;
  p1 = ntabm * std::exp(-p2 * p2 / 2.) / std::sqrt(2. * pi);
  double xmin = 2. * pi * p1 * p1 * 1.e-14;
  xmin = -std::log(xmin);
  xmin = -std::sqrt(xmin);
  const double xmax = -xmin;
  tab[1] = xmin;
  tab[2] = p2;
  tab[3] = p3;
  tab[ntab] = xmax;
  tab[ntabm] = -p2;
  tab[ntabmm] = -p3;
  // bisection / Newton solve of y = fdist(x) (rann2.f:180-214), kept as written
  double y = 2. * dy;
  double xx = tab[3] + dy * (xmax - xmin);
  const int ntabh = ntab / 2;
  for (int i = 4; i <= ntabh; i++) {
    y = y + dy;
    double xxmin = tab[i - 1];
    double xxmax = xmax;
    for (int iter = 1; iter <= 50; iter++) {
      const double yy = fdist(xx);
      const double err = yy - y;
      if (std::fabs(err) < 1.e-6) break;
      if (err > 0.) xxmax = xx;
      if (err < 0.) xxmin = xx;
      xx = xx + err / std::max(fdens(xx), 1.e-10);
      if (xx <= xxmin || xx >= xxmax) xx = 0.5 * (xxmin + xxmax);
    }
    tab[i] = xx;
  }
  for (int i = 1; i <= ntabh; i++) tab[ntab - i + 1] = -tab[i];
  tab[ntabh + 1] = 0.;
  for (int i = 1; i <= ntabm; i++) dtab[i] = tab[i + 1] - tab[i];
  ready = true;
}

// rann2.f:114-143: n Gaussian numbers from n uniforms of the active sequence
void Rann2::draw(Rng& r, double* x, int n) {
  if (!ready) init();
  const double pi = 3.1415927, azer = 1.e-20;
  for (int j = 0; j < n; j++) x[j] = r.ranu();   // ranu2 -> vrand: same LCG and state
  for (int j = 0; j < n; j++) {
    double y = x[j] * ntabm + 1;
    const int i = (int)y;
    if (i == 1) {
      double y1 = x[j];
      y1 = 2. * pi * p1 * p1 * y1 * y1;
      if (y1 <= 0.) y1 = azer;
      y1 = -std::log(y1);
      x[j] = -std::sqrt(y1);
      continue;
    }
    if (i == ntabm) {
      double y1 = 1. - x[j];
      y1 = 2. * pi * p1 * p1 * y1 * y1;
      y1 = -std::log(y1);
      x[j] = std::sqrt(y1);
      continue;
    }
    y = y - i;
    x[j] = tab[i] + y * dtab[i];
  }
}

void EPForcing::setup(int kfor_, int nx, double kforce_, double tforce_, double epsfor_, double tfiuo_,
                      int kranf1_, int kranf2_, double b11_, double b22_, double b33_) {
  kfor = kfor_;
  k2fo = 2 * kfor - 1;
  nrproc = 4 * kfor * k2fo * k2fo;   // param_set.f:87
  n = nx;
  kforce = kforce_; tforce = tforce_; epsfor = epsfor_; tfiuo = tfiuo_;
  kranf1 = kranf1_; kranf2 = kranf2_;
  b11 = b11_; b22 = b22_; b33 = b33_;
  suo.assign(nrproc, 0.0);
  svo.assign(nrproc, 0.0);
  velinc.assign(nrproc, 0.0);
  w1.assign(nrproc, 0.0);
  w2.assign(nrproc, 0.0);
  table.assign((size_t)2 * kfor * k2fo * k2fo * 3, 0.0);
  first = true;
}

// raniuo.f:56-109 (init when dt < 0)
void EPForcing::raniuo(Rng& r, double dtv) {
  if (t2 <= 0. || t1 <= 0.) return;
  const double diff = std::fabs(t1 / t2 - 1.);
  if (diff < 0.05) t1 = 0.95 * t2;
  if (dtv < 0.) {
    const double rr = t1 / (t1 + t2);
    const double be = std::sqrt(rr), ga = std::sqrt(1. - rr);
    g.draw(r, w1.data(), nrproc);
    g.draw(r, w2.data(), nrproc);
    for (int i = 0; i < nrproc; i++) {
      suo[i] = w1[i];
      svo[i] = be * w1[i] + ga * w2[i];
    }
    return;
  }
  const double om1 = 1. / t1, om2 = 1. / t2, s = om1 + om2, d = om2 - om1;
  const double a = std::exp(-om1 * dtv), b = std::exp(-om2 * dtv);
  const double c = (a - b) / d;
  const double sco = c * std::sqrt(s * om2);
  const double rr = std::sqrt(om2 / s);
  const double uu = 1. - a * a;
  const double vv = ((1. - b * b) + ((((4. * om1) * om2) * b) * c) / d) - ((om2 * s) * (a * a - b * b)) / (d * d);
  const double uv = rr * ((1. - a * b) - (s * a) * c);
  const double al = std::sqrt(uu);
  const double be = uv / al;
  const double ga = std::sqrt(std::max(vv - be * be, 0.));
  g.draw(r, w1.data(), nrproc);
  g.draw(r, w2.data(), nrproc);
  for (int i = 0; i < nrproc; i++) {
    svo[i] = b * svo[i] + sco * suo[i] + be * w1[i] + ga * w2[i];
    suo[i] = a * suo[i] + al * w1[i];
  }
}

// force.f:60-166 for one step of size dt; fills `table` = for(kfor,k2fo,k2fo,3)
// as interleaved complex doubles.
void EPForcing::step(Rng& r, double dt, int istart) {
  if (kforce == 0.) return;
  if (tforce * tfiuo == 0.) {
    // vfuo.f:25-55
    if (first) {
      first = false;
      if (istart == 0) {
        r.ranseq(kranf1);
        g.draw(r, suo.data(), nrproc);
      }
    }
    double exp1 = 0.;
    if (tforce > 0.05 * dt) exp1 = std::exp(-dt / tforce);
    const double exp2 = exp1 * exp1;
    const double rana = std::sqrt(1. - exp2);
    const double ranua = std::sqrt(epsfor * tforce) * ((1. - exp1) * (1. - exp1)) / std::sqrt(1. - exp2);
    double ranub = (epsfor * (2. * dt + tforce * (-3. + 4. * exp1 - exp2)) - ranua * ranua);
    ranub = std::sqrt(std::max(ranub, 0.));
    const double ranud = std::sqrt(epsfor * tforce) * (1. - exp1);
    r.ranseq(kranf2);
    g.draw(r, w1.data(), nrproc);
    g.draw(r, w2.data(), nrproc);
    for (int i = 0; i < nrproc; i++) {
      velinc[i] = ranud * suo[i] + ranua * w1[i] + ranub * w2[i];
      suo[i] = exp1 * suo[i] + rana * w1[i];
    }
  } else {
    // vfiuo.f:33-57
    if (first) {
      first = false;
      t1 = 0.5 * tforce * (1. + std::sqrt(1. - 4. * std::fabs(tfiuo) * std::fabs(tfiuo)));
      t2 = 0.5 * tforce * (1. - std::sqrt(1. - 4. * std::fabs(tfiuo) * std::fabs(tfiuo)));
      siga = std::sqrt(epsfor / tforce);
      if (istart <= 0 && tfiuo > 0.) {
        r.ranseq(kranf1);
        raniuo(r, -1.);
      }
    }
    r.ranseq(kranf2);
    raniuo(r, dt);
    const double fmult = siga * dt;
    for (int i = 0; i < nrproc; i++) velinc[i] = svo[i] * fmult;
  }
  // force.f:81-161
  const double s1 = std::sqrt(b11), s2 = std::sqrt(b22), s3 = std::sqrt(b33);
  auto kwave = [&](int idx1, int nn) {   // ky/kz of 1-based index ifwave(idx)
    const int i = idx1 + (idx1 / (kfor + 1)) * (nn - k2fo);
    int k = i - 1;
    if (i > nn / 2 + 1) k -= nn;
    return (double)k;
  };
  auto F = [&](int x, int y, int z, int i) -> double* {   // 1-based, complex
    const size_t o = ((((size_t)(i - 1) * k2fo + (z - 1)) * k2fo + (y - 1)) * kfor + (x - 1));
    return &table[2 * o];
  };
  auto V = [&](int c, int x, int y, int z) -> const double* {   // velinc(c,x,y,z), complex
    const size_t o = (size_t)(c - 1) + 2 * ((size_t)(x - 1) + (size_t)kfor * ((y - 1) + (size_t)k2fo * (z - 1)));
    return &velinc[2 * o];
  };
  for (int z = 1; z <= k2fo; z++)
    for (int y = 1; y <= k2fo; y++) {
      const double k2u = s2 * kwave(y, n);
      const double k3u = s3 * kwave(z, n);
      for (int x = 1; x <= kfor; x++) {
        const double* al = V(1, x, y, z);
        const double* be = V(2, x, y, z);
        const double k1u = s1 * (double)(x - 1);
        const double k = std::sqrt(k1u * k1u + k2u * k2u + k3u * k3u);
        const double k12 = std::sqrt(k1u * k1u + k2u * k2u);
        double* f1 = F(x, y, z, 1);
        double* f2 = F(x, y, z, 2);
        double* f3 = F(x, y, z, 3);
        if (k > kforce || k == 0.) {
          f1[0] = f1[1] = f2[0] = f2[1] = f3[0] = f3[1] = 0.;
        } else if (k12 == 0.) {
          f1[0] = al[0] / s1; f1[1] = al[1] / s1;
          f2[0] = be[0] / s2; f2[1] = be[1] / s2;
          f3[0] = 0.; f3[1] = 0.;
        } else {
          const double d1 = (k * k12) * s1, d2 = (k * k12) * s2, d3 = k * s3;
          f1[0] = ((al[0] * k) * k2u + (be[0] * k1u) * k3u) / d1;
          f1[1] = ((al[1] * k) * k2u + (be[1] * k1u) * k3u) / d1;
          f2[0] = ((be[0] * k2u) * k3u - (al[0] * k) * k1u) / d2;
          f2[1] = ((be[1] * k2u) * k3u - (al[1] * k) * k1u) / d2;
          f3[0] = -((be[0] * k12) / d3);
          f3[1] = -((be[1] * k12) / d3);
        }
      }
    }
  for (int i = 1; i <= 3; i++) {
    for (int y = kfor + 1; y <= k2fo; y++) {
      const double* s = F(1, k2fo + 2 - y, 1, i);
      double* d = F(1, y, 1, i);
      d[0] = s[0]; d[1] = -s[1];
    }
    for (int z = kfor + 1; z <= k2fo; z++) {
      {
        const double* s = F(1, 1, k2fo + 2 - z, i);
        double* d = F(1, 1, z, i);
        d[0] = s[0]; d[1] = -s[1];
      }
      for (int y = 2; y <= k2fo; y++) {
        const double* s = F(1, k2fo + 2 - y, k2fo + 2 - z, i);
        double* d = F(1, y, z, i);
        d[0] = s[0]; d[1] = -s[1];
      }
    }
  }
}

}  // namespace psdns
