/*
 * cusp_fit.c -- see cusp_fit.h.  Plain C99, compiled into libqmcb200.so.
 * Each function names the reference routine whose steps it restates.
 */
#include "cusp_fit.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- complex */
/* The Complex arithmetic of QMcBeaver/src/Complex.cpp (Numerical Recipes'
 * Cmul / Cdiv / Cabs / Csqrt forms). */
typedef struct {
  double re, im;
} cx;

static cx cx_make(double re, double im)
{
  cx c;
  c.re = re;
  c.im = im;
  return c;
}
static cx cx_add(cx a, cx b) { return cx_make(a.re + b.re, a.im + b.im); }
static cx cx_sub(cx a, cx b) { return cx_make(a.re - b.re, a.im - b.im); }
static cx cx_mul(cx a, cx b) { return cx_make(a.re * b.re - a.im * b.im, a.im * b.re + a.re * b.im); }
static cx cx_muld(cx a, double d) { return cx_make(a.re * d, a.im * d); }
static cx cx_div(cx a, cx b)
{
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re;
    double den = b.re + r * b.im;
    return cx_make((a.re + r * a.im) / den, (a.im - r * a.re) / den);
  } else {
    double r = b.re / b.im;
    double den = b.im + r * b.re;
    return cx_make((a.re * r + a.im) / den, (a.im * r - a.re) / den);
  }
}
static double cx_abs(cx a)
{
  double x = fabs(a.re), y = fabs(a.im);
  if (x == 0.0) return y;
  if (y == 0.0) return x;
  if (x > y) {
    double t = y / x;
    return x * sqrt(1.0 + t * t);
  }
  double t = x / y;
  return y * sqrt(1.0 + t * t);
}
static cx cx_sqrt(cx a)
{
  if (a.re == 0.0 && a.im == 0.0) return cx_make(0.0, 0.0);
  double x = fabs(a.re), y = fabs(a.im), w, r;
  if (x >= y) {
    r = y / x;
    w = sqrt(x) * sqrt(0.5 * (1.0 + sqrt(1.0 + r * r)));
  } else {
    r = x / y;
    w = sqrt(y) * sqrt(0.5 * (r + sqrt(1.0 + r * r)));
  }
  cx c;
  if (a.re >= 0.0) {
    c.re = w;
    c.im = a.im / (2.0 * w);
  } else {
    c.im = (a.im >= 0) ? w : -w;
    c.re = a.im / (2.0 * c.im);
  }
  return c;
}

/* Polynomial::laguer (QMcBeaver/src/Polynomial.cpp:301-357): one root of the
 * degree-m polynomial a[0..m] from the start x.  Returns 0 when converged. */
static int laguer(const cx *a, int m, cx *xp)
{
  static const double frac[9] = {0.0, 0.5, 0.25, 0.75, 0.13, 0.38, 0.62, 0.88, 1.0};
  const double EPSS = 1.0e-14;
  const int MR = 8, MT = 10, MAXIT = MT * MR;
  cx x = *xp;
  for (int iter = 1; iter <= MAXIT; iter++) {
    cx b = a[m], d = cx_make(0.0, 0.0), f = cx_make(0.0, 0.0);
    double err = cx_abs(b), abx = cx_abs(x);
    for (int j = m - 1; j >= 0; j--) {
      f = cx_add(cx_mul(x, f), d);
      d = cx_add(cx_mul(x, d), b);
      b = cx_add(cx_mul(x, b), a[j]);
      err = cx_abs(b) + abx * err;
    }
    err *= EPSS;
    if (cx_abs(b) <= err) {
      *xp = x;
      return 0;
    }
    cx g = cx_div(d, b);
    cx g2 = cx_mul(g, g);
    cx h = cx_sub(g2, cx_muld(cx_div(f, b), 2.0));
    cx sq = cx_sqrt(cx_muld(cx_sub(cx_muld(h, (double)m), g2), (double)(m - 1)));
    cx gp = cx_add(g, sq), gm = cx_sub(g, sq);
    double abp = cx_abs(gp), abm = cx_abs(gm);
    if (abp < abm) gp = gm;
    cx dx = ((abp > abm ? abp : abm) > 0.0) ? cx_div(cx_make((double)m, 0.0), gp)
                                           : cx_muld(cx_make(cos((double)iter), sin((double)iter)), 1 + abx);
    cx x1 = cx_sub(x, dx);
    if (x.re == x1.re && x.im == x1.im) {
      *xp = x;
      return 0;
    }
    if (iter % MT)
      x = x1;
    else
      x = cx_sub(x, cx_muld(dx, frac[iter / MT]));
  }
  *xp = x;
  return -1;
}

/* Polynomial::getRoots / zroots (QMcBeaver/src/Polynomial.cpp:253-430) for
 * real coefficients c[0..n-1]: roots sorted by real part. Returns the root
 * count, or -1 when Laguerre did not converge. */
static int poly_roots(const double *c, int n, cx *roots)
{
  int nc = n;
  for (int i = n - 1; i >= 0; i--) {
    if (fabs(c[i]) < 1.0e-50)
      nc--;
    else
      break;
  }
  int m = nc - 1;
  if (m < 1) return 0;
  cx a[16], ad[16];
  for (int j = 0; j <= m; j++) a[j] = ad[j] = cx_make(c[j], 0.0);
  const double EPS = 2.0e-13;
  int ok = 1;
  for (int j = m; j >= 1; j--) {
    cx x = cx_make(0.0, 0.0);
    if (laguer(ad, j, &x)) ok = 0;
    if (fabs(x.im) <= 2.0 * EPS * fabs(x.re)) x = cx_make(x.re, 0.0);
    roots[j - 1] = x;
    cx b = ad[j];
    for (int jj = j - 1; jj >= 0; jj--) {
      cx cc = ad[jj];
      ad[jj] = b;
      b = cx_add(cx_mul(x, b), cc);
    }
  }
  for (int j = 1; j <= m; j++)
    if (laguer(a, m, &roots[j - 1])) ok = 0;
  for (int j = 2; j <= m; j++) {
    cx x = roots[j - 1];
    int i;
    for (i = j - 1; i >= 1; i--) {
      if (roots[i - 1].re <= x.re) break;
      roots[i] = roots[i - 1];
    }
    roots[i] = x;
  }
  return ok ? m : -1;
}

/* Polynomial::evaluateAll (QMcBeaver/src/Polynomial.cpp:127-148). */
static void poly_eval(const double *c, int n, double x, double *f, double *df, double *d2f)
{
  int k = n - 1;
  *f = c[k];
  *df = 0.0;
  *d2f = 0.0;
  for (int i = k - 1; i >= 0; i--) {
    *d2f = *d2f * x + *df;
    *df = *df * x + *f;
    *f = *f * x + c[i];
  }
  *d2f *= 2;
}
static double poly_value(const double *c, int n, double x)
{
  double f, df, d2f;
  poly_eval(c, n, x, &f, &df, &d2f);
  return f;
}

/* ------------------------------------------------------ one orbital's fit */
typedef struct {
  int Z;
  int ns;
  const double *s;   /* [ns][2] exponent, coefficient x orbital coefficient */
  double n0;
  double rc;
  double ideal[9];
  int nideal;
} cusp_ctx;

typedef struct {
  double phi0, C, Zeff, sigma_sq;
  int sgn0, noC;
  double alpha[5];
} cusp_par;

/* QMCElectronNucleusCusp::evaluateOrigOrbital / getOrigGradient /
 * getOrigLocalEnergy (QMcBeaver/src/QMCElectronNucleusCusp.cpp:694-766). */
static double orig_value(const cusp_ctx *c, double r)
{
  double r_sq = r * r, v = 0.0;
  for (int i = 0; i < c->ns; i++) {
    double p0 = c->s[2 * i], p1 = c->s[2 * i + 1];
    v += p1 * exp(-p0 * r_sq);
  }
  return v;
}
static double orig_gradient(const cusp_ctx *c, double r)
{
  double r_sq = r * r, g = 0.0;
  for (int i = 0; i < c->ns; i++) {
    double p0 = c->s[2 * i], p1 = c->s[2 * i + 1];
    g += -p0 * 2 * r * p1 * exp(-p0 * r_sq);
  }
  return g;
}
static double orig_local_energy(const cusp_ctx *c, double r)
{
  double r_sq = r * r, v = 0.0, lap = 0.0;
  for (int i = 0; i < c->ns; i++) {
    double p0 = c->s[2 * i], p1 = c->s[2 * i + 1];
    double t = p1 * exp(-p0 * r_sq);
    v += t;
    lap += 2 * p0 * (2 * p0 * r_sq - 3) * t;
  }
  lap = lap / v;
  return -0.5 * lap - c->Z / r;
}

/* QMCElectronNucleusCuspParameters::calculateLocalEnergy (:287-329). */
static double rep_local_energy(const cusp_ctx *c, const cusp_par *p, double r, int rIsZero)
{
  double f, df, d2f;
  if (rIsZero) {
    poly_eval(p->alpha, 5, 0.0, &f, &df, &d2f);
    if (p->noC) return -0.5 * (d2f + df * df);
    double e = p->sgn0 * exp(f);
    return (-0.5 * e / (p->C + e)) * (d2f + df * df);
  }
  poly_eval(p->alpha, 5, r, &f, &df, &d2f);
  double localKE = -0.5 * (d2f + df * (2.0 / r + df));
  if (p->noC) return localKE - p->Zeff / r;
  double e = p->sgn0 * exp(f);
  return localKE * e / (p->C + e) - p->Zeff / r;
}

static double deviation(const cusp_ctx *c, const cusp_par *p, double r, int rIsZero)
{
  double rep = rep_local_energy(c, p, r, rIsZero);
  double ideal = c->Z * c->Z * poly_value(c->ideal, c->nideal, r);
  return (rep - ideal) * (rep - ideal);
}

/* QMCElectronNucleusCuspParameters::findMaxDeviation (:529-587). */
static int find_max_deviation(const cusp_ctx *c, const cusp_par *p, double lower, double upper, int lowerZero,
                              double *max)
{
  const double GOLD = 0.61803399;
  double lowR = lower, lowValue = deviation(c, p, lowR, lowerZero);
  double highR = upper, highValue = deviation(c, p, highR, 0);
  double midR = GOLD * (upper - lower) + lower, midValue = deviation(c, p, midR, 0);
  int it = 0;
  while (highR - lowR > 1e-4) {
    if (++it > 100000) return -1;
    if (highValue > lowValue) {
      lowR = midR;
      lowValue = midValue;
      if (highValue > midValue)
        midR = lowR + GOLD * (highR - lowR);
      else if (highValue <= midValue)
        midR = highR - GOLD * (highR - lowR);
    } else if (highValue < lowValue) {
      highR = midR;
      highValue = midValue;
      if (lowValue > midValue)
        midR = highR - GOLD * (highR - lowR);
      else if (lowValue <= midValue)
        midR = lowR + GOLD * (highR - lowR);
    }
    midValue = deviation(c, p, midR, 0);
  }
  if (highValue > midValue)
    *max = highValue > lowValue ? highValue : lowValue;
  else if (midValue >= highValue)
    *max = midValue > lowValue ? midValue : lowValue;
  return 0;
}

/* QMCElectronNucleusCuspParameters::calculateSigmaSq (:465-527). */
static int sigma_sq(const cusp_ctx *c, cusp_par *p)
{
  if (p->noC) return find_max_deviation(c, p, 0.0, c->rc, 1, &p->sigma_sq);
  double co[5];
  for (int i = 0; i < 5; i++) co[i] = p->alpha[i];
  co[0] -= log(fabs(p->C));
  cx roots[8];
  int nr = poly_roots(co, 5, roots);
  if (nr < 0) return -2;
  double root = -2;
  const double tol = 1e-8;
  for (int i = 0; i < nr; i++) {
    double re = roots[i].re, im = roots[i].im;
    if (re > 0 && re < c->rc && fabs(im) < tol) {
      root = re;
      break;
    }
  }
  if (root < 0) return find_max_deviation(c, p, 0.0, c->rc, 1, &p->sigma_sq);
  double max1 = 0.0, max2 = 0.0;
  if (root - c->rc / 5 > 0.0 && find_max_deviation(c, p, 0.0, root - c->rc / 5, 1, &max1)) return -1;
  if (root + c->rc / 5 < c->rc && find_max_deviation(c, p, root + c->rc / 5, c->rc, 0, &max2)) return -1;
  p->sigma_sq = max1 > max2 ? max1 : max2;
  return 0;
}

/* QMCElectronNucleusCuspParameters::fitReplacementOrbital (:331-463). */
static int fit_replacement(const cusp_ctx *c, double phi0, cusp_par *p)
{
  p->phi0 = phi0;
  double rc = c->rc, rc_sq = rc * rc;
  double ov = 0.0, od1 = 0.0, od2 = 0.0;
  for (int i = 0; i < c->ns; i++) {
    double p0 = c->s[2 * i], p1 = c->s[2 * i + 1];
    double t = p1 * exp(-p0 * rc_sq);
    ov += t;
    od1 += -2 * p0 * rc * t;
    od2 += 2 * p0 * (2 * p0 * rc_sq - 1) * t;
  }
  p->sgn0 = (phi0 - ov > 0) ? 1 : -1;
  p->noC = 1;
  p->C = 0.0;
  if (ov * phi0 < 0) {
    p->noC = 0;
    if (ov > 0.0 && ov < 0.1)
      p->C = ov + 0.1;
    else if (ov < 0.0 && ov > -0.1)
      p->C = ov - 0.1;
    else
      p->C = 2 * ov;
  } else {
    if (ov > 0.0 && ov < 0.1) {
      p->noC = 0;
      p->C = ov - 0.1;
    } else if (ov < 0.0 && ov > -0.1) {
      p->noC = 0;
      p->C = ov + 0.1;
    }
  }
  if (p->sgn0 == 1 && phi0 < 0.0) {
    p->noC = 0;
    if (ov > -0.1)
      p->C = ov - 0.1;
    else
      p->C = 2 * ov;
  } else if (p->sgn0 == -1 && phi0 > 0.0) {
    p->noC = 0;
    if (ov < 0.1)
      p->C = ov + 0.1;
    else
      p->C = 2 * ov;
  }
  p->Zeff = c->Z * fabs(1 + (c->n0 / phi0));
  double x1 = log(fabs(ov - p->C));
  double x2 = od1 / (ov - p->C);
  double x3 = od2 / (ov - p->C);
  double x4;
  if (c->n0 / phi0 >= -1.0)
    x4 = -c->Z * (phi0 + c->n0) / (phi0 - p->C);
  else
    x4 = c->Z * (phi0 + c->n0) / (phi0 - p->C);
  if ((p->sgn0 == 1 && phi0 < 0.0) || (p->sgn0 == -1 && phi0 > 0.0)) x4 *= -1;
  double x5 = log(fabs(phi0 - p->C));
  double rc_inv = 1 / rc;
  p->alpha[0] = x5;
  p->alpha[1] = x4;
  p->alpha[2] = (6 * (x1 - x5) * rc_inv - 3 * (x2 + x4)) * rc_inv + 0.5 * (x3 - x2 * x2);
  p->alpha[3] = ((8 * (x5 - x1) * rc_inv + 5 * x2 + 3 * x4) * rc_inv + x2 * x2 - x3) * rc_inv;
  p->alpha[4] = ((3 * (x1 - x5) * rc_inv - 2 * x2 - x4) * rc_inv + 0.5 * (x3 - x2 * x2)) * rc_inv * rc_inv;
  return sigma_sq(c, p);
}

/* QMCElectronNucleusCusp::determineRc (QMcBeaver/src/QMCElectronNucleusCusp.cpp:175-425). */
static int determine_rc(cusp_ctx *c, char *err)
{
  const int Z = c->Z;
  const double rcmax = 1.0 / Z;
  if (Z > 1) {
    const double p[9] = {0.0, 0.0, 3.25819, -15.0126, 33.7308, -42.8705, 31.2276, -12.1316, 1.94692};
    memcpy(c->ideal, p, sizeof(p));
    c->nideal = 9;
    double f = poly_value(c->ideal, 9, rcmax);
    c->ideal[0] = orig_local_energy(c, rcmax) / (Z * Z) - f;
  } else if (Z == 1) {
    c->nideal = 1;
    c->ideal[0] = orig_local_energy(c, rcmax);
  } else {
    snprintf(err, 256, "cusp fit: nuclear charge %d", Z);
    return -1;
  }
  const double dr = rcmax / 100;
  double old_value = orig_value(c, rcmax), new_value;
  int ridx[101], nRoots = 0;
  for (int i = 0; i < 101; i++) {
    new_value = orig_value(c, rcmax - i * dr);
    if (new_value * old_value < 0) ridx[nRoots++] = i;
    old_value = new_value;
  }
  double roots[101];
  int counter = 0;
  const double tol = 1e-8;
  for (int q = 0; q < nRoots; q++) {
    double rl = rcmax - ridx[q] * dr, fl = orig_value(c, rl);
    double rh = rl + dr, fh = orig_value(c, rh);
    if (fl * fh > 0) {
      snprintf(err, 256, "cusp fit: %g and %g do not bracket a root", rl, rh);
      return -1;
    }
    if (fabs(fl) < tol) {
      roots[counter++] = rl;
      continue;
    } else if (fabs(fh) < tol) {
      roots[counter++] = rh;
      continue;
    }
    int found = 0;
    for (int i = 0; i < 10000; i++) {
      if (i == 9999) {
        snprintf(err, 256, "cusp fit: too many iterations in finding a root");
        return -1;
      }
      double rm = (rl + rh) / 2, fm = orig_value(c, rm);
      if (fabs(fm) < tol) {
        roots[counter++] = rm;
        found = 1;
        break;
      } else if (fm * fl < 0) {
        rh = rm;
        fh = fm;
      } else {
        rl = rm;
        fl = fm;
      }
    }
    (void)found;
  }
  const double gradNear = orig_gradient(c, rcmax / 1000);
  const double origAt0 = orig_value(c, 0.0);
  double rc = rcmax, r_trial = rcmax, r_bound = 0.0;
  int rootIndex = -1;
  const double ddr = dr / 10;
  const double maxdev = Z * Z / 50.0;
  if (nRoots > 0) {
    rootIndex = nRoots - 1;
    r_bound = roots[rootIndex] + rcmax / 5;
  }
  long guard = 0;
  while (r_trial > 0.0) {
    if (++guard > 10000000L) {
      snprintf(err, 256, "cusp fit: the search for rc does not end");
      return -1;
    }
    if (gradNear * (orig_value(c, r_trial) - origAt0) > 0.0) {
      if (r_trial > r_bound) {
        double ideal = poly_value(c->ideal, c->nideal, r_trial);
        old_value = orig_local_energy(c, r_trial);
        if (fabs(Z * Z * ideal - old_value) > maxdev) {
          r_trial += dr;
          while (r_trial > 0.0) {
            r_trial -= ddr;
            if (gradNear * (orig_value(c, r_trial) - origAt0) > 0.0) {
              ideal = poly_value(c->ideal, c->nideal, r_trial);
              old_value = orig_local_energy(c, r_trial);
              if (fabs(Z * Z * ideal - old_value) > maxdev) {
                rc = r_trial;
                break;
              }
            }
          }
          break;
        }
      } else {
        double ideal = poly_value(c->ideal, c->nideal, r_bound);
        old_value = orig_local_energy(c, r_bound);
        if ((gradNear * (orig_value(c, r_trial) - origAt0) > 0.0) && (fabs(Z * Z * ideal - old_value) > maxdev)) {
          while (r_trial > 0.0) {
            r_trial -= ddr;
            ideal = poly_value(c->ideal, c->nideal, r_trial);
            old_value = orig_local_energy(c, r_trial);
            if (fabs(Z * Z * ideal - old_value) > maxdev) {
              rc = r_trial;
              break;
            }
          }
          break;
        } else {
          r_trial = roots[rootIndex] - rcmax / 5 + dr;
          if (rootIndex > 0) {
            rootIndex--;
            r_bound = roots[rootIndex] + rcmax / 5;
          } else if (rootIndex == 0) {
            r_bound = 0.0;
          }
        }
      }
    }
    r_trial -= dr;
  }
  c->rc = rc;
  if (Z > 1) {
    c->ideal[0] = 0.0;
    double f = poly_value(c->ideal, 9, rc);
    c->ideal[0] = orig_local_energy(c, rc) / (Z * Z) - f;
  } else {
    c->ideal[0] = orig_local_energy(c, rc);
  }
  return 0;
}

/* QMCElectronNucleusCusp::fitOrbitalParameters (:427-572): golden-section
 * search of phi0 (within 10% of the original value at the nucleus) for the
 * smallest maximum deviation from the ideal local energy. */
static int fit_orbital(const cusp_ctx *c, cusp_par *best, char *err)
{
  const double GOLD = 0.618034;
  cusp_par lo, mid, hi;
  double a0 = orig_value(c, 0.0), arc = orig_value(c, c->rc);
  double lo_phi, mid_phi, hi_phi;
  if (a0 - arc < 0.0) {
    hi_phi = a0;
    mid_phi = a0 - 0.05 * fabs(a0 - arc);
    lo_phi = a0 - 0.1 * fabs(a0 - arc);
  } else {
    lo_phi = a0;
    mid_phi = a0 + 0.05 * fabs(a0 - arc);
    hi_phi = a0 + 0.1 * fabs(a0 - arc);
  }
  if (fit_replacement(c, lo_phi, &lo) || fit_replacement(c, mid_phi, &mid) || fit_replacement(c, hi_phi, &hi))
    goto fail;
  {
    double loS = lo.sigma_sq, midS = mid.sigma_sq, hiS = hi.sigma_sq;
    int it = 0;
    while (hi_phi - lo_phi > fabs(mid_phi / 10000)) {
      if (++it > 100000) goto fail;
      if (loS < midS) {
        if (midS < hiS) {
          hi_phi = mid_phi;
          hiS = midS;
          mid_phi = lo_phi + GOLD * (hi_phi - lo_phi);
        } else if (loS < hiS) {
          hi_phi = mid_phi;
          hiS = midS;
          mid_phi = lo_phi + GOLD * (hi_phi - lo_phi);
        } else {
          lo_phi = mid_phi;
          loS = midS;
          mid_phi = hi_phi - GOLD * (hi_phi - lo_phi);
        }
      } else {
        if (hiS < midS) {
          lo_phi = mid_phi;
          loS = midS;
          mid_phi = hi_phi - GOLD * (hi_phi - lo_phi);
        } else if (loS < hiS) {
          hi_phi = mid_phi;
          hiS = midS;
          mid_phi = hi_phi - GOLD * (hi_phi - lo_phi);
        } else {
          lo_phi = mid_phi;
          loS = midS;
          mid_phi = lo_phi + GOLD * (hi_phi - lo_phi);
        }
      }
      if (fit_replacement(c, mid_phi, &mid)) goto fail;
      midS = mid.sigma_sq;
    }
  }
  *best = mid;
  return 0;
fail:
  snprintf(err, 256, "cusp fit: the search for the replacement orbital does not end");
  return -1;
}

int qmcb_cusp_fit(int M, const double *xyz, const double *Zd, int K, const int *bf_atom, const int *bf_pow,
                  const int *bf_nprim, const int *bf_off, const double *pexp, const double *pcoef, int n_orb,
                  const double *mo, double *out, char *err)
{
  char dummy[256];
  if (!err) err = dummy;
  err[0] = 0;
  for (int t = 0; t < M * n_orb * QMCB_CUSP_REC; t++) out[t] = 0.0;
  int nprim_total = 0;
  for (int k = 0; k < K; k++) nprim_total += bf_nprim[k];
  double *s = (double *)malloc(sizeof(double) * 2 * (nprim_total > 0 ? nprim_total : 1));
  if (!s) {
    snprintf(err, 256, "cusp fit: out of memory");
    return -1;
  }
  for (int i = 0; i < M; i++) {
    int first = -1, nbf = 0, ns_count = 0;
    for (int k = 0; k < K; k++)
      if (bf_atom[k] == i) {
        if (first < 0) first = k;
        nbf++;
        if (bf_pow[3 * k] + bf_pow[3 * k + 1] + bf_pow[3 * k + 2] == 0) ns_count += bf_nprim[k];
      }
    if (ns_count == 0) continue;
    for (int m = 0; m < n_orb; m++) {
      cusp_ctx c;
      memset(&c, 0, sizeof(c));
      c.Z = (int)Zd[i];
      int cnt = 0, needed = 0;
      for (int k = first; k < first + nbf; k++) {
        if (bf_pow[3 * k] + bf_pow[3 * k + 1] + bf_pow[3 * k + 2] != 0) continue;
        for (int l = 0; l < bf_nprim[k]; l++) {
          s[2 * cnt] = pexp[bf_off[k] + l];
          s[2 * cnt + 1] = pcoef[bf_off[k] + l] * mo[(size_t)m * K + k];
          if (fabs(s[2 * cnt + 1]) > 1e-15) needed = 1;
          cnt++;
        }
      }
      if (!needed) continue;
      c.ns = cnt;
      c.s = s;
      if (determine_rc(&c, err)) {
        free(s);
        return -1;
      }
      /* n0: the orbital at this nucleus from the functions of the other nuclei */
      double n0 = 0.0;
      for (int j = 0; j < M; j++) {
        if (j == i) continue;
        double xr = xyz[3 * i] - xyz[3 * j], yr = xyz[3 * i + 1] - xyz[3 * j + 1], zr = xyz[3 * i + 2] - xyz[3 * j + 2];
        double rsq = xr * xr + yr * yr + zr * zr;
        for (int k = 0; k < K; k++) {
          if (bf_atom[k] != j) continue;
          double pw = pow(xr, bf_pow[3 * k]) * pow(yr, bf_pow[3 * k + 1]) * pow(zr, bf_pow[3 * k + 2]);
          double temp = 0.0;
          for (int l = 0; l < bf_nprim[k]; l++) temp += pcoef[bf_off[k] + l] * exp(-pexp[bf_off[k] + l] * rsq);
          n0 += temp * pw * mo[(size_t)m * K + k];
        }
      }
      c.n0 = n0;
      cusp_par p;
      if (fit_orbital(&c, &p, err)) {
        free(s);
        return -1;
      }
      double *o = out + ((size_t)i * n_orb + m) * QMCB_CUSP_REC;
      o[0] = c.rc;
      o[1] = (double)p.sgn0;
      o[2] = p.C;
      for (int q = 0; q < 5; q++) o[3 + q] = p.alpha[q];
    }
  }
  free(s);
  return 0;
}
