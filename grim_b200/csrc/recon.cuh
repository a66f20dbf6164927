// recon.cuh -- face reconstruction of one variable from its 5-point stencil
// (templated on the scalar so the op-counting build can run the same code)
// y0..y4 = v[i-2..i+2] along one direction.  Returns the value on the left
// face (i-1/2) and the right face (i+1/2) of zone i, as primLeft / primRight
// of the reference's reconstruct (reconstruction.cpp:3-36).
#pragma once
#include "common.cuh"

namespace grim {

// minmod.cpp:3-19; ArrayFire's sign() is 1 for x < 0 and 0 otherwise
template <class S>
GRIM_D S af_sgn(S x) { return (x < S(0.)) ? S(1.) : S(0.); }
template <class S>
GRIM_D S minmod3(S x, S y, S z) {
  S m = fmin(fmin(fabs(x), fabs(y)), fabs(z));
  S sx = 1. - 2. * af_sgn(x), sy = 1. - 2. * af_sgn(y), sz = 1. - 2. * af_sgn(z);
  return 0.25 * fabs(sx + sy) * (sx + sz) * m;
}
// minmod.cpp:21-71 with dX
template <class S>
GRIM_D S slope_mm(S y1, S y2, S y3, double dX, double theta) {
  S fwd = (y3 - y2) / dX;
  S bwd = (y2 - y1) / dX;
  S cen = bwd + fwd;
  return minmod3(theta * bwd, 0.5 * cen, theta * fwd);
}
// weno5.cpp:39-65 (the live code: centred 5-point derivative)
template <class S>
GRIM_D S slope_5pt(S y0, S y1, S y3, S y4, double dX) {
  return (-y4 + 8. * y3 - 8. * y1 + y0) / 12. / dX;
}
// ppm.cpp:41-75 / :120-159
template <class S>
GRIM_D void ppm_faces(S y0, S y1, S y2, S y3, S y4, S& leftV, S& rightV) {
  S d0 = 2. * (y1 - y0), d1 = 2. * (y2 - y1), d2 = 2. * (y3 - y2), d3 = 2. * (y4 - y3);
  S D1 = 0.5 * (y2 - y0), D2 = 0.5 * (y3 - y1), D3 = 0.5 * (y4 - y2);
  S DQ1 = (d1 * d0 <= 0.) ? 0. : ((D1 > 0.) ? 1. : -1.) * fmin(fabs(D1), fmin(fabs(d0), fabs(d1)));
  S DQ2 = (d2 * d1 <= 0.) ? 0. : ((D2 > 0.) ? 1. : -1.) * fmin(fabs(D2), fmin(fabs(d1), fabs(d2)));
  S DQ3 = (d3 * d2 <= 0.) ? 0. : ((D3 > 0.) ? 1. : -1.) * fmin(fabs(D3), fmin(fabs(d2), fabs(d3)));
  S l = 0.5 * (y2 + y1) - 1. / 6. * (DQ2 - DQ1);
  S r = 0.5 * (y3 + y2) - 1. / 6. * (DQ3 - DQ2);
  bool corr1 = ((r - y2) * (y2 - l) <= 0.);
  S qd = r - l;
  S qe = 6. * (y2 - 0.5 * (r + l));
  bool corr2 = (qd * (qd - qe) < 0.);
  bool corr3 = (qd * (qd + qe) < 0.);
  if (corr1) { l = y2; r = y2; }
  if (corr2) l = 3. * y2 - 2. * r;
  if (!corr2 && corr3) r = 3. * y2 - 2. * l;
  leftV = l;
  rightV = r;
}
template <class S>
GRIM_D S slope_ppm(S y0, S y1, S y2, S y3, S y4, double dX) {
  S l, r;
  ppm_faces(y0, y1, y2, y3, y4, l, r);
  return (r - l) / dX;
}
// WENO5 (weno5.cpp:111-257)
template <class S>
GRIM_D void weno5_faces(S y0, S y1, S y2, S y3, S y4, S& lo, S& ro) {
  const S eps2 = 1.0e-17;
  S beta1 = ((4.0 / 3.0) * y0 * y0 - (19.0 / 3.0) * y0 * y1 + (25.0 / 3.0) * y1 * y1 +
                  (11.0 / 3.0) * y0 * y2 - (31.0 / 3.0) * y1 * y2 + (10.0 / 3.0) * y2 * y2) +
                 eps2 * (1.0 + fabs(y0) + fabs(y1) + fabs(y2));
  S beta2 = ((4.0 / 3.0) * y1 * y1 - (13.0 / 3.0) * y1 * y2 + (13.0 / 3.0) * y2 * y2 +
                  (5.0 / 3.0) * y1 * y3 - (13.0 / 3.0) * y2 * y3 + (4.0 / 3.0) * y3 * y3) +
                 eps2 * (1.0 + fabs(y1) + fabs(y2) + fabs(y3));
  S beta3 = ((10.0 / 3.0) * y2 * y2 - (31.0 / 3.0) * y2 * y3 + (25.0 / 3.0) * y3 * y3 +
                  (11.0 / 3.0) * y2 * y4 - (19.0 / 3.0) * y3 * y4 + (4.0 / 3.0) * y4 * y4) +
                 eps2 * (1.0 + fabs(y2) + fabs(y3) + fabs(y4));
  S w1r = 1.0 / (16.0 * beta1 * beta1);
  S w2r = 5.0 / (8.0 * beta2 * beta2);
  S w3r = 5.0 / (16.0 * beta3 * beta3);
  S w1l = 5.0 / (16.0 * beta1 * beta1);
  S w2l = 5.0 / (8.0 * beta2 * beta2);
  S w3l = 1.0 / (16.0 * beta3 * beta3);
  S denl = w1l + w2l + w3l;
  S denr = w1r + w2r + w3r;
  S u1r = 0.375 * y0 - 1.25 * y1 + 1.875 * y2;
  S u2r = -0.125 * y1 + 0.75 * y2 + 0.375 * y3;
  S u3r = 0.375 * y2 + 0.75 * y3 - 0.125 * y4;
  S u1l = -0.125 * y0 + 0.75 * y1 + 0.375 * y2;
  S u2l = 0.375 * y1 + 0.75 * y2 - 0.125 * y3;
  S u3l = 1.875 * y2 - 1.25 * y3 + 0.375 * y4;
  lo = (w1l * u1l + w2l * u2l + w3l * u3l) / denl;
  ro = (w1r * u1r + w2r * u2r + w3r * u3r) / denr;
}
// MP5 (Suresh & Huynh 1997, alpha = 4): interface value at i+1/2 from the
// left-biased stencil.  No counterpart in the reference.
template <class S>
GRIM_D S mm2(S a, S b) {
  return 0.5 * (copysign(1., a) + copysign(1., b)) * fmin(fabs(a), fabs(b));
}
template <class S>
GRIM_D S mm4(S a, S b, S c, S d) {
  S s = 0.125 * (copysign(1., a) + copysign(1., b)) *
             fabs((copysign(1., a) + copysign(1., c)) * (copysign(1., a) + copysign(1., d)));
  return s * fmin(fmin(fabs(a), fabs(b)), fmin(fabs(c), fabs(d)));
}
template <class S>
GRIM_D S mp5(S vm2, S vm1, S v0, S vp1, S vp2) {
  const S alpha = 4.;
  S f = (2. * vm2 - 13. * vm1 + 47. * v0 + 27. * vp1 - 3. * vp2) / 60.;
  S vmp = v0 + mm2(vp1 - v0, alpha * (v0 - vm1));
  if ((f - v0) * (f - vmp) <= 0.) return f;
  S djm1 = vm2 - 2. * vm1 + v0;
  S dj = vm1 - 2. * v0 + vp1;
  S djp1 = v0 - 2. * vp1 + vp2;
  S dm4jph = mm4(4. * dj - djp1, 4. * djp1 - dj, dj, djp1);
  S dm4jmh = mm4(4. * dj - djm1, 4. * djm1 - dj, dj, djm1);
  S vul = v0 + alpha * (v0 - vm1);
  S vav = 0.5 * (v0 + vp1);
  S vmd = vav - 0.5 * dm4jph;
  S vlc = v0 + 0.5 * (v0 - vm1) + 4. / 3. * dm4jmh;
  S vmin = fmax(fmin(fmin(v0, vp1), vmd), fmin(fmin(v0, vul), vlc));
  S vmax = fmin(fmax(fmax(v0, vp1), vmd), fmax(fmax(v0, vul), vlc));
  return f + mm2(vmin - f, vmax - f);
}

// WENO5 with the same weights in fewer divisions (fast path only): the
// normalised weights are unchanged when every weight is multiplied by
// beta1^2 beta2^2 beta3^2, which leaves one division per face value instead
// of four.  Equal to weno5_faces to a few ulp.
template <class S>
GRIM_D void weno5_faces_fast(S y0, S y1, S y2, S y3, S y4, S& lo, S& ro) {
  const S eps2 = 1.0e-17;
  S beta1 = ((4.0 / 3.0) * y0 * y0 - (19.0 / 3.0) * y0 * y1 + (25.0 / 3.0) * y1 * y1 +
                  (11.0 / 3.0) * y0 * y2 - (31.0 / 3.0) * y1 * y2 + (10.0 / 3.0) * y2 * y2) +
                 eps2 * (1.0 + fabs(y0) + fabs(y1) + fabs(y2));
  S beta2 = ((4.0 / 3.0) * y1 * y1 - (13.0 / 3.0) * y1 * y2 + (13.0 / 3.0) * y2 * y2 +
                  (5.0 / 3.0) * y1 * y3 - (13.0 / 3.0) * y2 * y3 + (4.0 / 3.0) * y3 * y3) +
                 eps2 * (1.0 + fabs(y1) + fabs(y2) + fabs(y3));
  S beta3 = ((10.0 / 3.0) * y2 * y2 - (31.0 / 3.0) * y2 * y3 + (25.0 / 3.0) * y3 * y3 +
                  (11.0 / 3.0) * y2 * y4 - (19.0 / 3.0) * y3 * y4 + (4.0 / 3.0) * y4 * y4) +
                 eps2 * (1.0 + fabs(y2) + fabs(y3) + fabs(y4));
  const S b1 = beta1 * beta1, b2 = beta2 * beta2, b3 = beta3 * beta3;
  const S p23 = b2 * b3, p13 = b1 * b3, p12 = b1 * b2;
  // w1 ~ 1/b1 -> p23, w2 ~ 1/b2 -> p13, w3 ~ 1/b3 -> p12
  const S w1r = 0.0625 * p23, w2r = 0.625 * p13, w3r = 0.3125 * p12;
  const S w1l = 0.3125 * p23, w2l = 0.625 * p13, w3l = 0.0625 * p12;
  S u1r = 0.375 * y0 - 1.25 * y1 + 1.875 * y2;
  S u2r = -0.125 * y1 + 0.75 * y2 + 0.375 * y3;
  S u3r = 0.375 * y2 + 0.75 * y3 - 0.125 * y4;
  S u1l = -0.125 * y0 + 0.75 * y1 + 0.375 * y2;
  S u2l = 0.375 * y1 + 0.75 * y2 - 0.125 * y3;
  S u3l = 1.875 * y2 - 1.25 * y3 + 0.375 * y4;
  lo = (w1l * u1l + w2l * u2l + w3l * u3l) / (w1l + w2l + w3l);
  ro = (w1r * u1r + w2r * u2r + w3r * u3r) / (w1r + w2r + w3r);
}

// face values of zone i
template <class S>
GRIM_D void recon_faces(int scheme, double theta, S y0, S y1, S y2, S y3, S y4,
                        S& lo, S& ro) {
  switch (scheme) {
    case GRIM_WENO5: weno5_faces(y0, y1, y2, y3, y4, lo, ro); return;
    case GRIM_PPM: ppm_faces(y0, y1, y2, y3, y4, lo, ro); return;
    case GRIM_MP5:
      ro = mp5(y0, y1, y2, y3, y4);
      lo = mp5(y4, y3, y2, y1, y0);
      return;
    default: {
      // minmod.cpp:73-95 (dX = 1)
      S s = slope_mm(y1, y2, y3, 1., theta);
      lo = y2 - 0.5 * s;
      ro = y2 + 0.5 * s;
      return;
    }
  }
}
template <class S>
GRIM_D void recon_faces_fast(int scheme, double theta, S y0, S y1, S y2, S y3, S y4,
                             S& lo, S& ro) {
  if (scheme == GRIM_WENO5) {
    weno5_faces_fast(y0, y1, y2, y3, y4, lo, ro);
    return;
  }
  recon_faces(scheme, theta, y0, y1, y2, y3, y4, lo, ro);
}

// face values with the scheme fixed at compile time (RS >= 0: one scheme's
// code in the kernel) or read at run time (RS < 0); FAST selects the
// reassociated WENO5 weights
template <int RS, bool FAST, class S>
GRIM_D void recon_faces_rs(int scheme, double theta, S y0, S y1, S y2, S y3, S y4, S& lo, S& ro) {
  if constexpr (RS < 0) {
    if constexpr (FAST)
      recon_faces_fast(scheme, theta, y0, y1, y2, y3, y4, lo, ro);
    else
      recon_faces(scheme, theta, y0, y1, y2, y3, y4, lo, ro);
  } else if constexpr (RS == GRIM_WENO5) {
    if constexpr (FAST)
      weno5_faces_fast(y0, y1, y2, y3, y4, lo, ro);
    else
      weno5_faces(y0, y1, y2, y3, y4, lo, ro);
  } else {
    recon_faces(RS, theta, y0, y1, y2, y3, y4, lo, ro);  // a constant scheme folds the switch
  }
}

// the slope() used by the EMHD gradients (reconstruction.cpp:39-64); MP5
// uses the centred 5-point derivative
template <class S>
GRIM_D S recon_slope(int scheme, double theta, S y0, S y1, S y2, S y3,
                          S y4, double dX) {
  switch (scheme) {
    case GRIM_WENO5: return slope_5pt(y0, y1, y3, y4, dX);
    case GRIM_PPM: return slope_ppm(y0, y1, y2, y3, y4, dX);
    case GRIM_MP5: return slope_5pt(y0, y1, y3, y4, dX);
    default: return slope_mm(y1, y2, y3, dX, theta);
  }
}

}  // namespace grim
