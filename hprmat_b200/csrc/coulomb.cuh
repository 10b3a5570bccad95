// Boundary functions of the R-matrix -> collision-matrix step, FP64.
//
// Restatement of HPRMAT's src/special_functions.f for the forms the R-matrix path uses:
//   coulfg_single -- COULFG (src/special_functions.f:1-275) with MODE1=1, KFN=0 and
//                    XLMIN=XLMAX, the call at src/rmatrix_hp.F90:232 (LXTRA=0, so no
//                    recurrence in lambda);
//   jwkb          -- JWKB (src/special_functions.f:277-306);
//   whit_l        -- WHIT (src/special_functions.f:309-416), W_l and dW_l/dr at one l.
// WHIT's Fortran literals such as 10.0/12.0 and 0.15 are default (single) precision; they
// are reproduced as the single-precision value widened to double, because they shift W at
// the 1e-8 level and W enters C(E) through the closed-channel Bloch term.
//
// The functions are __host__ __device__ so the energy scan can evaluate them per solve on
// the device; rmatrix() evaluates them on the host (O(nch) calls per energy).
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define HPR_HD __host__ __device__
#else
#define HPR_HD
#endif

namespace hprmat {

struct CoulombFG {
  double f, g, fp, gp;
  int ifail;
};

struct JwkbOut {
  double fjwkb, gjwkb;
  int iexp;
  bool set;
};

HPR_HD inline JwkbOut jwkb(double xx, double eta1, double xl) {
  JwkbOut o{0.0, 0.0, 0, false};
  const double rl35 = 35.0;
  const double aloge = log(10.0);
  double x = xx, eta = eta1;
  double gh2 = x * (eta + eta - x);
  double xll1 = fmax(xl * xl + xl, 0.0);
  if (gh2 + xll1 <= 0.0) return o;
  double hll = xll1 + 6.0 / rl35;
  double hl = sqrt(hll);
  double sl = eta / hl + hl / x;
  double rl2 = 1.0 + eta * eta / hll;
  double gh = sqrt(gh2 + hll) / x;
  double gs = gh + sl;
  double phi = x * gh - 0.5 * (hl * log(gs * gs / rl2) - log(gh));
  if (eta != 0.0) phi = phi - eta * atan2(x * gh, x - eta);
  double phi10 = -phi * aloge;
  int iexp = (int)phi10;
  double gj;
  if (iexp > 70) {
    gj = pow(10.0, phi10 - iexp);
  } else {
    gj = exp(-phi);
    iexp = 0;
  }
  o.fjwkb = 0.5 / (gh * gj);
  o.gjwkb = gj;
  o.iexp = iexp;
  o.set = true;
  return o;
}

// F_l, G_l and their derivatives with respect to x at one lambda = xl.
HPR_HD inline CoulombFG coulfg_single(double xx, double eta1, double xl) {
  CoulombFG r{0.0, 0.0, 0.0, 0.0, 0};
  const double abort_ = 2.0e4, tm30 = 1.0e-30, accur = 1.0e-16;
  double eta = eta1;
  double gjwkb = 0.0, fjwkb = 0.0;
  double acc = accur * 10.0;
  double acc4 = acc * 100.0 * 100.0;
  double acch = sqrt(acc);
  if (xx <= acch) { r.ifail = -1; return r; }
  double x = xx, xlm = xl;
  if (xlm <= -1.0) { r.ifail = -2; return r; }
  double e2mm1 = eta * eta + xlm * xlm + xlm;
  bool xlturn = x * (x - 2.0 * eta) < xlm * xlm + xlm;
  double xll = xlm;
  // CF1 (src/special_functions.f:88-115)
  double xi = 1.0 / x;
  double fcl = 1.0;
  double pk = xll + 1.0;
  double px = pk + abort_;
  double f = eta / pk + pk * xi;
  if (fabs(f) < tm30) f = tm30;
  double d = 0.0, c = f, df;
  for (;;) {
    double pk1 = pk + 1.0;
    double ek = eta / pk;
    double rk2 = 1.0 + ek * ek;
    double tk = (pk + pk1) * (xi + ek / pk1);
    d = tk - rk2 * d;
    c = tk - rk2 / c;
    if (fabs(c) < tm30) c = tm30;
    if (fabs(d) < tm30) d = tm30;
    d = 1.0 / d;
    df = d * c;
    f = f * df;
    if (d < 0.0) fcl = -fcl;
    pk = pk1;
    if (pk > px) { r.ifail = -3; return r; }
    if (!(fabs(df - 1.0) >= acc)) break;
  }
  // CF2 (src/special_functions.f:153-196)
  int iexp = 1;
  if (xlturn) {
    JwkbOut jw = jwkb(x, eta, fmax(xlm, 0.0));
    if (jw.set) { fjwkb = jw.fjwkb; gjwkb = jw.gjwkb; iexp = jw.iexp; }
  }
  double p, q, gam, w;
  if (!(iexp > 1 || gjwkb > 1.0 / (acch * 100.0))) {
    xlturn = false;
    double ta = 2.0 * abort_;
    pk = 0.0;
    double wi = eta + eta;
    p = 0.0;
    q = 1.0 - eta * xi;
    double ar = -e2mm1, ai = eta;
    double br = 2.0 * (x - eta), bi = 2.0;
    double dr = br / (br * br + bi * bi);
    double di = -bi / (br * br + bi * bi);
    double dp = -xi * (ar * di + ai * dr);
    double dq = xi * (ar * dr - ai * di);
    for (;;) {
      p = p + dp;
      q = q + dq;
      pk = pk + 2.0;
      ar = ar + pk;
      ai = ai + wi;
      bi = bi + 2.0;
      double dd = ar * dr - ai * di + br;
      di = ai * dr + ar * di + bi;
      double cc = 1.0 / (dd * dd + di * di);
      dr = cc * dd;
      di = -cc * di;
      double a = br * dr - bi * di - 1.0;
      double b = bi * dr + br * di;
      cc = dp * a - dq * b;
      dq = dp * b + dq * a;
      dp = cc;
      if (pk > ta) { r.ifail = -4; return r; }
      if (!(fabs(dp) + fabs(dq) >= (fabs(p) + fabs(q)) * acc)) break;
    }
    gam = (f - p) / q;
    if (q <= acc4 * fabs(p)) { r.ifail = -5; return r; }
    w = 1.0 / sqrt((f - p) * gam + q);
  } else {
    // src/special_functions.f:198-201
    w = fjwkb;
    gam = gjwkb * w;
    p = f;
    q = 1.0;
  }
  // KFN = 0 normalisation (src/special_functions.f:205-221)
  double fcm = copysign(w, fcl);
  double gcl = xlturn ? gjwkb : fcm * gam;
  r.f = fcm;
  r.g = gcl;
  r.gp = gcl * (p - q / gam);
  r.fp = fcm * f;
  return r;
}

// Single-precision Fortran literals of WHIT, widened to double.
#define HPR_W_10_12 0.83333331346511840820  /* REAL(10.0/12.0) */
#define HPR_W_1_6   0.16666667163372039795  /* REAL(1.0/6.0)   */
#define HPR_W_1_12  0.08333333581686019897  /* REAL(1.0/12.0)  */
#define HPR_W_1_60  0.01666666753590106964  /* REAL(1.0/60.0)  */
#define HPR_W_0_15  0.15000000596046447754  /* REAL(0.15)      */

struct WhitOut {
  double w;    // W_l(k r), scaled by e**ie
  double wd;   // dW_l/dr (k * dW/d(kr)), same scaling
  int ie;
};

// Whittaker W_l and its r-derivative at r for bound-state wave number xk (e = -xk^2).
HPR_HD inline WhitOut whit_l(double heta, double r, double xk, int ll) {
  const double fpmax = 1.0e290;
  const double ee = -1.0;
  int L = ll + 1;
  double ak = xk, eta = heta, rho = ak * r;
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double t[4] = {0, 0, 0, 0};
  int is = 7;
  double pje = 30.0 * rho + 1.0;
  int ih = (int)pje;
  double h = (double)(ih > 4 ? ih : 4);
  h = rho / h;
  double rhoa = 10.0 * (eta + 1.0);
  int ifeql;
  if (rhoa - rho <= 0.0) {
    ifeql = 1;
    rhoa = rho;
  } else {
    ifeql = 0;
  }
  pje = rhoa / h + 0.5;
  rhoa = h * (double)(int)pje;
  if (ifeql <= 0) {
    if (rhoa - rho - 1.5 * h < 0.0) rhoa = rho + 2.0 * h;
  }
  int ie = 0;
  double f1 = 0.0, fd1 = 0.0;
  for (;;) {
    // label 55: asymptotic series at rhoa
    double c = 1.0 / rhoa;
    double a = 1.0;
    double b = 1.0 - c * eta;
    f1 = a;
    fd1 = b;
    for (int m = 1; m <= 26; ++m) {
      double d = 0.5 * (eta + (double)(m - 1)) * (eta + (double)m) * c / (double)m;
      a = -a * d;
      b = -b * d - a * c;
      f1 += a;
      fd1 += b;
    }
    a = -eta * log(2.0 * rhoa) - rhoa;
    double fpminl = -log(fpmax);
    if (ie == 0 && a < fpminl) ie = (int)(fpminl - a);
    a = exp(a + ie);
    f1 = a * f1;
    fd1 = a * fd1 * (-1.0 - 2 * eta / rhoa);
    if (ifeql > 0) break;
    s[is] = f1;
    if (is == 7) {
      is = 6;
      rhoa = rhoa + h;
      continue;
    }
    // label 27: Numerov inwards
    double A = 2.0 - HPR_W_10_12 * h * h * ee;
    double B = HPR_W_1_6 * h * eta;
    double C = 1.0 + HPR_W_1_12 * h * h * ee;
    int m1 = (int)(rhoa / h - 0.5);
    int m2 = (int)(rho / h - 1.5);
    t[2] = B / (double)(m1 + 1);
    t[3] = B / (double)m1;
    int js = m1;
    for (int it = m2; it <= m1; ++it) {
      for (int i = 1; i <= 6; ++i) s[i] = s[i + 1];
      t[1] = t[2];
      t[2] = t[3];
      t[3] = B / (double)(js - 1);
      s[7] = ((A + 10.0 * t[2]) * s[6] - (C - t[1]) * s[5]) / (C - t[3]);
      js -= 1;
      if (fabs(s[7]) > fpmax)
        for (int i = 2; i <= 7; ++i) s[i] = s[i] / fpmax;
    }
    t[1] = s[4];
    t[2] = (HPR_W_1_60 * (s[1] - s[7]) + HPR_W_0_15 * (s[6] - s[2]) + 0.75 * (s[3] - s[5])) / h;
    f1 = t[1];
    fd1 = t[2];
    break;
  }
  // label 61: upward recurrence to l = ll
  double c = 1.0 / rho;
  double fm = f1, fdm = fd1;
  for (int m = 1; m <= L - 1; ++m) {
    double a = eta / (double)m;
    double b = a + c * (double)m;
    double fn = (b * fm - fdm) / (a + 1.0);
    double fdn = (a - 1.0) * fm - b * fn;
    fm = fn;
    fdm = fdn;
  }
  WhitOut o;
  o.w = fm;
  o.wd = ak * fdm;
  o.ie = ie;
  return o;
}

}  // namespace hprmat
