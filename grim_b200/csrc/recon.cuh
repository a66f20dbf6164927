// recon.cuh -- face reconstruction of one variable from its 5-point stencil
// y0..y4 = v[i-2..i+2] along one direction.  Returns the value on the left
// face (i-1/2) and the right face (i+1/2) of zone i, as primLeft / primRight
// of the reference's reconstruct (reconstruction.cpp:3-36).
#pragma once
#include "common.cuh"

namespace grim {

// minmod.cpp:3-19; ArrayFire's sign() is 1 for x < 0 and 0 otherwise
GRIM_D double af_sgn(double x) { return (x < 0.) ? 1. : 0.; }
GRIM_D double minmod3(double x, double y, double z) {
  double m = fmin(fmin(fabs(x), fabs(y)), fabs(z));
  double sx = 1. - 2. * af_sgn(x), sy = 1. - 2. * af_sgn(y), sz = 1. - 2. * af_sgn(z);
  return 0.25 * fabs(sx + sy) * (sx + sz) * m;
}
// minmod.cpp:21-71 with dX
GRIM_D double slope_mm(double y1, double y2, double y3, double dX, double theta) {
  double fwd = (y3 - y2) / dX;
  double bwd = (y2 - y1) / dX;
  double cen = bwd + fwd;
  return minmod3(theta * bwd, 0.5 * cen, theta * fwd);
}
// weno5.cpp:39-65 (the live code: centred 5-point derivative)
GRIM_D double slope_5pt(double y0, double y1, double y3, double y4, double dX) {
  return (-y4 + 8. * y3 - 8. * y1 + y0) / 12. / dX;
}
// ppm.cpp:41-75 / :120-159
GRIM_D void ppm_faces(double y0, double y1, double y2, double y3, double y4, double& leftV, double& rightV) {
  double d0 = 2. * (y1 - y0), d1 = 2. * (y2 - y1), d2 = 2. * (y3 - y2), d3 = 2. * (y4 - y3);
  double D1 = 0.5 * (y2 - y0), D2 = 0.5 * (y3 - y1), D3 = 0.5 * (y4 - y2);
  double DQ1 = (d1 * d0 <= 0.) ? 0. : ((D1 > 0.) ? 1. : -1.) * fmin(fabs(D1), fmin(fabs(d0), fabs(d1)));
  double DQ2 = (d2 * d1 <= 0.) ? 0. : ((D2 > 0.) ? 1. : -1.) * fmin(fabs(D2), fmin(fabs(d1), fabs(d2)));
  double DQ3 = (d3 * d2 <= 0.) ? 0. : ((D3 > 0.) ? 1. : -1.) * fmin(fabs(D3), fmin(fabs(d2), fabs(d3)));
  double l = 0.5 * (y2 + y1) - 1. / 6. * (DQ2 - DQ1);
  double r = 0.5 * (y3 + y2) - 1. / 6. * (DQ3 - DQ2);
  bool corr1 = ((r - y2) * (y2 - l) <= 0.);
  double qd = r - l;
  double qe = 6. * (y2 - 0.5 * (r + l));
  bool corr2 = (qd * (qd - qe) < 0.);
  bool corr3 = (qd * (qd + qe) < 0.);
  if (corr1) { l = y2; r = y2; }
  if (corr2) l = 3. * y2 - 2. * r;
  if (!corr2 && corr3) r = 3. * y2 - 2. * l;
  leftV = l;
  rightV = r;
}
GRIM_D double slope_ppm(double y0, double y1, double y2, double y3, double y4, double dX) {
  double l, r;
  ppm_faces(y0, y1, y2, y3, y4, l, r);
  return (r - l) / dX;
}
// WENO5 (weno5.cpp:111-257)
GRIM_D void weno5_faces(double y0, double y1, double y2, double y3, double y4, double& lo, double& ro) {
  const double eps2 = 1.0e-17;
  double beta1 = ((4.0 / 3.0) * y0 * y0 - (19.0 / 3.0) * y0 * y1 + (25.0 / 3.0) * y1 * y1 +
                  (11.0 / 3.0) * y0 * y2 - (31.0 / 3.0) * y1 * y2 + (10.0 / 3.0) * y2 * y2) +
                 eps2 * (1.0 + fabs(y0) + fabs(y1) + fabs(y2));
  double beta2 = ((4.0 / 3.0) * y1 * y1 - (13.0 / 3.0) * y1 * y2 + (13.0 / 3.0) * y2 * y2 +
                  (5.0 / 3.0) * y1 * y3 - (13.0 / 3.0) * y2 * y3 + (4.0 / 3.0) * y3 * y3) +
                 eps2 * (1.0 + fabs(y1) + fabs(y2) + fabs(y3));
  double beta3 = ((10.0 / 3.0) * y2 * y2 - (31.0 / 3.0) * y2 * y3 + (25.0 / 3.0) * y3 * y3 +
                  (11.0 / 3.0) * y2 * y4 - (19.0 / 3.0) * y3 * y4 + (4.0 / 3.0) * y4 * y4) +
                 eps2 * (1.0 + fabs(y2) + fabs(y3) + fabs(y4));
  double w1r = 1.0 / (16.0 * beta1 * beta1);
  double w2r = 5.0 / (8.0 * beta2 * beta2);
  double w3r = 5.0 / (16.0 * beta3 * beta3);
  double w1l = 5.0 / (16.0 * beta1 * beta1);
  double w2l = 5.0 / (8.0 * beta2 * beta2);
  double w3l = 1.0 / (16.0 * beta3 * beta3);
  double denl = w1l + w2l + w3l;
  double denr = w1r + w2r + w3r;
  double u1r = 0.375 * y0 - 1.25 * y1 + 1.875 * y2;
  double u2r = -0.125 * y1 + 0.75 * y2 + 0.375 * y3;
  double u3r = 0.375 * y2 + 0.75 * y3 - 0.125 * y4;
  double u1l = -0.125 * y0 + 0.75 * y1 + 0.375 * y2;
  double u2l = 0.375 * y1 + 0.75 * y2 - 0.125 * y3;
  double u3l = 1.875 * y2 - 1.25 * y3 + 0.375 * y4;
  lo = (w1l * u1l + w2l * u2l + w3l * u3l) / denl;
  ro = (w1r * u1r + w2r * u2r + w3r * u3r) / denr;
}
// MP5 (Suresh & Huynh 1997, alpha = 4): interface value at i+1/2 from the
// left-biased stencil.  No counterpart in the reference.
GRIM_D double mm2(double a, double b) {
  return 0.5 * (copysign(1., a) + copysign(1., b)) * fmin(fabs(a), fabs(b));
}
GRIM_D double mm4(double a, double b, double c, double d) {
  double s = 0.125 * (copysign(1., a) + copysign(1., b)) *
             fabs((copysign(1., a) + copysign(1., c)) * (copysign(1., a) + copysign(1., d)));
  return s * fmin(fmin(fabs(a), fabs(b)), fmin(fabs(c), fabs(d)));
}
GRIM_D double mp5(double vm2, double vm1, double v0, double vp1, double vp2) {
  const double alpha = 4.;
  double f = (2. * vm2 - 13. * vm1 + 47. * v0 + 27. * vp1 - 3. * vp2) / 60.;
  double vmp = v0 + mm2(vp1 - v0, alpha * (v0 - vm1));
  if ((f - v0) * (f - vmp) <= 0.) return f;
  double djm1 = vm2 - 2. * vm1 + v0;
  double dj = vm1 - 2. * v0 + vp1;
  double djp1 = v0 - 2. * vp1 + vp2;
  double dm4jph = mm4(4. * dj - djp1, 4. * djp1 - dj, dj, djp1);
  double dm4jmh = mm4(4. * dj - djm1, 4. * djm1 - dj, dj, djm1);
  double vul = v0 + alpha * (v0 - vm1);
  double vav = 0.5 * (v0 + vp1);
  double vmd = vav - 0.5 * dm4jph;
  double vlc = v0 + 0.5 * (v0 - vm1) + 4. / 3. * dm4jmh;
  double vmin = fmax(fmin(fmin(v0, vp1), vmd), fmin(fmin(v0, vul), vlc));
  double vmax = fmin(fmax(fmax(v0, vp1), vmd), fmax(fmax(v0, vul), vlc));
  return f + mm2(vmin - f, vmax - f);
}

// WENO5 with the same weights in fewer divisions (fast path only): the
// normalised weights are unchanged when every weight is multiplied by
// beta1^2 beta2^2 beta3^2, which leaves one division per face value instead
// of four.  Equal to weno5_faces to a few ulp.
GRIM_D void weno5_faces_fast(double y0, double y1, double y2, double y3, double y4, double& lo, double& ro) {
  const double eps2 = 1.0e-17;
  double beta1 = ((4.0 / 3.0) * y0 * y0 - (19.0 / 3.0) * y0 * y1 + (25.0 / 3.0) * y1 * y1 +
                  (11.0 / 3.0) * y0 * y2 - (31.0 / 3.0) * y1 * y2 + (10.0 / 3.0) * y2 * y2) +
                 eps2 * (1.0 + fabs(y0) + fabs(y1) + fabs(y2));
  double beta2 = ((4.0 / 3.0) * y1 * y1 - (13.0 / 3.0) * y1 * y2 + (13.0 / 3.0) * y2 * y2 +
                  (5.0 / 3.0) * y1 * y3 - (13.0 / 3.0) * y2 * y3 + (4.0 / 3.0) * y3 * y3) +
                 eps2 * (1.0 + fabs(y1) + fabs(y2) + fabs(y3));
  double beta3 = ((10.0 / 3.0) * y2 * y2 - (31.0 / 3.0) * y2 * y3 + (25.0 / 3.0) * y3 * y3 +
                  (11.0 / 3.0) * y2 * y4 - (19.0 / 3.0) * y3 * y4 + (4.0 / 3.0) * y4 * y4) +
                 eps2 * (1.0 + fabs(y2) + fabs(y3) + fabs(y4));
  const double b1 = beta1 * beta1, b2 = beta2 * beta2, b3 = beta3 * beta3;
  const double p23 = b2 * b3, p13 = b1 * b3, p12 = b1 * b2;
  // w1 ~ 1/b1 -> p23, w2 ~ 1/b2 -> p13, w3 ~ 1/b3 -> p12
  const double w1r = 0.0625 * p23, w2r = 0.625 * p13, w3r = 0.3125 * p12;
  const double w1l = 0.3125 * p23, w2l = 0.625 * p13, w3l = 0.0625 * p12;
  double u1r = 0.375 * y0 - 1.25 * y1 + 1.875 * y2;
  double u2r = -0.125 * y1 + 0.75 * y2 + 0.375 * y3;
  double u3r = 0.375 * y2 + 0.75 * y3 - 0.125 * y4;
  double u1l = -0.125 * y0 + 0.75 * y1 + 0.375 * y2;
  double u2l = 0.375 * y1 + 0.75 * y2 - 0.125 * y3;
  double u3l = 1.875 * y2 - 1.25 * y3 + 0.375 * y4;
  lo = (w1l * u1l + w2l * u2l + w3l * u3l) / (w1l + w2l + w3l);
  ro = (w1r * u1r + w2r * u2r + w3r * u3r) / (w1r + w2r + w3r);
}

// face values of zone i
GRIM_D void recon_faces(int scheme, double theta, double y0, double y1, double y2, double y3, double y4,
                        double& lo, double& ro) {
  switch (scheme) {
    case GRIM_WENO5: weno5_faces(y0, y1, y2, y3, y4, lo, ro); return;
    case GRIM_PPM: ppm_faces(y0, y1, y2, y3, y4, lo, ro); return;
    case GRIM_MP5:
      ro = mp5(y0, y1, y2, y3, y4);
      lo = mp5(y4, y3, y2, y1, y0);
      return;
    default: {
      // minmod.cpp:73-95 (dX = 1)
      double s = slope_mm(y1, y2, y3, 1., theta);
      lo = y2 - 0.5 * s;
      ro = y2 + 0.5 * s;
      return;
    }
  }
}
GRIM_D void recon_faces_fast(int scheme, double theta, double y0, double y1, double y2, double y3, double y4,
                             double& lo, double& ro) {
  if (scheme == GRIM_WENO5) {
    weno5_faces_fast(y0, y1, y2, y3, y4, lo, ro);
    return;
  }
  recon_faces(scheme, theta, y0, y1, y2, y3, y4, lo, ro);
}

// the slope() used by the EMHD gradients (reconstruction.cpp:39-64); MP5
// uses the centred 5-point derivative
GRIM_D double recon_slope(int scheme, double theta, double y0, double y1, double y2, double y3,
                          double y4, double dX) {
  switch (scheme) {
    case GRIM_WENO5: return slope_5pt(y0, y1, y3, y4, dX);
    case GRIM_PPM: return slope_ppm(y0, y1, y2, y3, y4, dX);
    case GRIM_MP5: return slope_5pt(y0, y1, y3, y4, dX);
    default: return slope_mm(y1, y2, y3, dX, theta);
  }
}

}  // namespace grim
