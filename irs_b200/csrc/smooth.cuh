// Deflection by the smooth mass sheet that compensates the stars' convergence,
// and its derivatives. Restates include/alpha_smooth.cuh:
//   alpha_smooth           :62-127  (rectangular/circular x approximate/exact)
//   d_alpha_smooth_d_z     :141-170
//   d_alpha_smooth_d_zbar  :185-236
//   d2_alpha_smooth_d_zbar2 :251-300
// The rectangular approximate form is the degree-`taylor_smooth` series in
// conj(z)/corner of the exact four-logarithm expression.
#pragma once
#include "common.cuh"

namespace irsb {

template <typename T>
IRSB_HD T heaviside_(T x) {
  return x >= 0 ? T(1) : T(0);
}
template <typename T>
IRSB_HD T boxcar_(cplx<T> z, cplx<T> c) {
  return (-c.re <= z.re && z.re <= c.re && -c.im <= z.im && z.im <= c.im) ? T(1) : T(0);
}

template <typename T>
IRSB_HD cplx<T> alpha_smooth_(cplx<T> z, T ks, int rect, cplx<T> c, int approx, int ts, T inv_pi) {
  cplx<T> a;
  if (rect) {
    cplx<T> zb = cconj(z);
    if (approx) {
      cplx<T> s1 = mk<T>(0, 0), s2 = s1, s3 = s1, s4 = s1;
      cplx<T> r1 = cdiv(zb, c), r2 = cdiv(zb, cconj(c)), r3 = cdiv(zb, cneg(c)), r4 = cdiv(zb, cneg(cconj(c)));
      for (int i = ts; i >= 1; i--) {
        T inv = T(1) / T(i);
        s1.re += inv;
        s2.re += inv;
        s3.re += inv;
        s4.re += inv;
        s1 = cmul(s1, r1);
        s2 = cmul(s2, r2);
        s3 = cmul(s3, r3);
        s4 = cmul(s4, r4);
      }
      a = csub(cmul(csub(c, zb), csub(clog_(c), s1)), cmul(csub(cconj(c), zb), csub(clog_(cconj(c)), s2)));
      a = cadd(a, cmul(csub(cneg(c), zb), csub(clog_(cneg(c)), s3)));
      a = csub(a, cmul(csub(cneg(cconj(c)), zb), csub(clog_(cconj(cneg(c))), s4)));
      a = cmul(a, mk<T>(0, -ks * inv_pi));
      a.re -= ks * 2 * (c.re + z.re);
    } else {
      cplx<T> c1 = csub(c, zb), c2 = csub(cconj(c), zb), c3 = csub(cneg(c), zb), c4 = csub(cneg(cconj(c)), zb);
      a = csub(cadd(csub(cmul(c1, clog_(c1)), cmul(c2, clog_(c2))), cmul(c3, clog_(c3))), cmul(c4, clog_(c4)));
      a = cmul(a, mk<T>(0, -ks * inv_pi));
      a.re -= ks * 2 * (c.re + z.re) * boxcar_(z, c);
      a.re -= ks * 4 * c.re * heaviside_(c.im + z.im) * heaviside_(c.im - z.im) * heaviside_(z.re - c.re);
    }
  } else {
    if (approx) {
      a = cscale(z, -ks);
    } else {
      T ca = cabs_(c);
      if (cabs_(z) <= ca)
        a = cscale(z, -ks);
      else
        a = cdiv(mk<T>(-ks * ca * ca, 0), cconj(z));
    }
  }
  return a;
}

template <typename T>
IRSB_HD T d_alpha_smooth_dz_(cplx<T> z, T ks, int rect, cplx<T> c, int approx) {
  if (approx) return -ks;
  if (rect) return -ks * boxcar_(z, c);
  return -ks * heaviside_(cabs_(c) - cabs_(z));
}

template <typename T>
IRSB_HD cplx<T> d_alpha_smooth_dzbar_(cplx<T> z, T ks, int rect, cplx<T> c, int approx, int ts, T inv_pi) {
  cplx<T> d = mk<T>(0, 0);
  if (rect) {
    if (approx) {
      cplx<T> r = cdiv(cconj(z), c);
      cplx<T> r2 = cmul(r, r);
      T ph = carg(c);
      for (int i = ts - 1; i >= 2; i -= 2) {
        cplx<T> e = cexp_(mk<T>(0, 2 * ph * i));
        d = cadd(d, cdivr(mk<T>(1 - e.re, -e.im), T(i)));
        d = cmul(d, r2);
      }
      d = cscale(d, T(2));
      d = cmul(d, mk<T>(0, -ks * inv_pi));
      d.re += ks - 4 * ks * ph * inv_pi;
    } else {
      cplx<T> c1 = csub(cconj(c), cconj(z)), c2 = csub(c, cconj(z)), c3 = csub(cneg(c), cconj(z)),
              c4 = csub(cneg(cconj(c)), cconj(z));
      d = cadd(csub(csub(clog_(c1), clog_(c2)), clog_(c3)), clog_(c4));
      d = cmul(d, mk<T>(0, -ks * inv_pi));
      d.re -= ks * boxcar_(z, c);
    }
  } else if (!approx) {
    T ca = cabs_(c);
    cplx<T> zb = cconj(z);
    d = cdiv(mk<T>(ks * ca * ca, 0), cmul(zb, zb));
  }
  return d;
}

template <typename T>
IRSB_HD cplx<T> d2_alpha_smooth_dzbar2_(cplx<T> z, T ks, int rect, cplx<T> c, int approx, int ts, T inv_pi) {
  cplx<T> d = mk<T>(0, 0);
  cplx<T> zb = cconj(z);
  if (rect) {
    if (approx) {
      cplx<T> r = cdiv(zb, c);
      cplx<T> r2 = cmul(r, r);
      T ph = carg(c);
      for (int i = ts - 1; i >= 2; i -= 2) {
        cplx<T> e = cexp_(mk<T>(0, 2 * ph * i));
        d = cadd(d, mk<T>(1 - e.re, -e.im));
        d = cmul(d, r2);
      }
      d = cdiv(d, zb);
      d = cscale(d, T(2));
      d = cmul(d, mk<T>(0, -ks * inv_pi));
    } else {
      cplx<T> c1 = csub(cconj(c), zb), c2 = csub(c, zb), c3 = csub(cneg(c), zb), c4 = csub(cneg(cconj(c)), zb);
      cplx<T> one = mk<T>(1, 0);
      d = cadd(csub(cadd(cneg(cdiv(one, c1)), cdiv(one, c2)), cdiv(one, c4)), cdiv(one, c3));
      d = cmul(d, mk<T>(0, -ks * inv_pi));
    }
  } else if (!approx) {
    T ca = cabs_(c);
    d = cdiv(mk<T>(-2 * ks * ca * ca, 0), cmul(cmul(zb, zb), zb));
  }
  return d;
}

}  // namespace irsb
