// Stellar mass functions: inverse-CDF sampling and the moments <m>, <m^2>,
// <m^2 ln m> used by the derived parameters.
//
// Follows the reference's mass-function family (include/mass_functions.cuh:17-25):
//   equal          m = 1                                  (mass_functions/equal.cuh:11-74)
//   uniform        power law, slope 0                     (mass_functions/uniform.cuh:11-23)
//   salpeter       power law, slope -2.35                 (mass_functions/salpeter.cuh:22)
//   kroupa         broken power law, slopes -0.3/-1.3/-2.3,
//                  breaks at 0.08 and 0.5 solar masses    (mass_functions/kroupa.cuh:22-162)
//   optical_depth  two masses contributing equal kappa    (mass_functions/optical_depth.cuh:14-93)
// The power-law integrals are the closed forms of int b x^a dx and
// int b x^a ln x dx; the broken power law is normalised piecewise with
// continuity factors at the breaks. The segment bookkeeping keeps the same
// operation order as the reference so that single-precision moments round
// identically (they feed num_stars through a ceil()).
#pragma once
#include "common.cuh"
#include <cstring>

namespace irsb {

enum MassFunctionKind : int {
  kMFEqual = 0,
  kMFUniform = 1,
  kMFSalpeter = 2,
  kMFKroupa = 3,
  kMFOpticalDepth = 4,
  kMFInvalid = -1,
};

inline int mass_function_kind(const char* s) {
  if (!std::strcmp(s, "equal")) return kMFEqual;
  if (!std::strcmp(s, "uniform")) return kMFUniform;
  if (!std::strcmp(s, "salpeter")) return kMFSalpeter;
  if (!std::strcmp(s, "kroupa")) return kMFKroupa;
  if (!std::strcmp(s, "optical_depth")) return kMFOpticalDepth;
  return kMFInvalid;
}

// int_{x1}^{x2} b x^a dx
template <typename T>
IRSB_HD T pl_int(T x1, T x2, T a, T b = T(1)) {
  if (a != T(-1)) return b * (xpow(x2, a + 1) - xpow(x1, a + 1)) / (a + 1);
  return b * (xlog(x2) - xlog(x1));
}
// int_{x1}^{x2} b x^a ln(x) dx
template <typename T>
IRSB_HD T pl_log_int(T x1, T x2, T a, T b = T(1)) {
  if (a != T(-1))
    return b * (xpow(x2, a + 1) * ((a + 1) * xlog(x2) - 1) - xpow(x1, a + 1) * ((a + 1) * xlog(x1) - 1)) /
           ((a + 1) * (a + 1));
  return b * (xlog(x2) * xlog(x2) - xlog(x1) * xlog(x1)) / 2;
}
// x such that int_{x1}^{x} b t^a dt = p
template <typename T>
IRSB_HD T pl_inv(T p, T x1, T a, T b) {
  if (a != T(-1)) return xpow(p * (a + 1) / b + xpow(x1, a + 1), 1 / (a + 1));
  return x1 * xexp(p / b);
}

template <typename T>
IRSB_HD T mf_slope(int kind) {
  return kind == kMFSalpeter ? T(-2.35) : T(0);
}

// Broken power law with three segments: probabilities and normalisations of the
// segments that intersect [ml, mu].
template <typename T>
struct Kroupa3 {
  T s[3];
  T m0, m1;
  T probs[3];
  T b[3];
  IRSB_HD void setup(T ml, T mu, T msol) {
    s[0] = T(-0.3);
    s[1] = T(-1.3);
    s[2] = T(-2.3);
    m0 = T(0.08) * msol;
    m1 = T(0.5) * msol;
    for (int i = 0; i < 3; i++) {
      probs[i] = 0;
      b[i] = 0;
    }
    if (mu < m0) {
      probs[0] = pl_int(ml, mu, s[0]);
      b[0] = 1 / probs[0];
      probs[0] *= b[0];
    } else if (mu < m1) {
      if (ml < m0) {
        probs[0] = pl_int(ml, m0, s[0]);
        probs[1] = pl_int(m0, mu, s[1]) * xpow(m0, s[0] - s[1]);
        b[0] = 1 / (probs[0] + probs[1]);
        probs[0] *= b[0];
        probs[1] *= b[0];
        b[1] = b[0] * xpow(m0, s[0] - s[1]);
      } else {
        probs[1] = pl_int(ml, mu, s[1]);
        b[1] = 1 / probs[1];
        probs[1] *= b[1];
      }
    } else {
      if (ml < m0) {
        probs[0] = pl_int(ml, m0, s[0]);
        probs[1] = pl_int(m0, m1, s[1]) * xpow(m0, s[0] - s[1]);
        probs[2] = pl_int(m1, mu, s[2]) * xpow(m0, s[0] - s[1]) * xpow(m1, s[1] - s[2]);
        b[0] = 1 / (probs[0] + probs[1] + probs[2]);
        probs[0] *= b[0];
        probs[1] *= b[0];
        probs[2] *= b[0];
        b[1] = b[0] * xpow(m0, s[0] - s[1]);
        b[2] = b[1] * xpow(m1, s[1] - s[2]);
      } else if (ml < m1) {
        probs[1] = pl_int(ml, m1, s[1]);
        probs[2] = pl_int(m1, mu, s[2]) * xpow(m1, s[1] - s[2]);
        b[1] = 1 / (probs[1] + probs[2]);
        probs[1] *= b[1];
        probs[2] *= b[1];
        b[2] = b[1] * xpow(m1, s[1] - s[2]);
      } else {
        probs[2] = pl_int(ml, mu, s[2]);
        b[2] = 1 / probs[2];
        probs[2] *= b[2];
      }
    }
  }
  // moment: sum over segments of int b_k m^(s_k + e) [f] dm, f = 1 or ln m
  IRSB_HD T moment(T ml, T mu, int e, bool logm) const {
    auto seg = [&](T x1, T x2, int k) -> T {
      return logm ? pl_log_int(x1, x2, s[k] + e, b[k]) : pl_int(x1, x2, s[k] + e, b[k]);
    };
    if (mu < m0) return seg(ml, mu, 0);
    if (mu < m1) {
      if (ml < m0) return seg(ml, m0, 0) + seg(m0, mu, 1);
      return seg(ml, mu, 1);
    }
    if (ml < m0) return seg(ml, m0, 0) + seg(m0, m1, 1) + seg(m1, mu, 2);
    if (ml < m1) return seg(ml, m1, 1) + seg(m1, mu, 2);
    return seg(ml, mu, 2);
  }
  IRSB_HD T draw(T p, T ml) const {
    if (p < probs[0]) return pl_inv(p, ml, s[0], b[0]);
    if (p < probs[0] + probs[1]) {
      if (ml < m0) return pl_inv(p - probs[0], m0, s[1], b[1]);
      return pl_inv(p, ml, s[1], b[1]);
    }
    if (ml < m0) return pl_inv(p - probs[0] - probs[1], m1, s[2], b[2]);
    if (ml < m1) return pl_inv(p - probs[1], m1, s[2], b[2]);
    return pl_inv(p, ml, s[2], b[2]);
  }
};

// Mass for a uniform deviate p (ml, mu already in arbitrary units).
template <typename T>
IRSB_HD T mf_mass(int kind, T p, T ml, T mu, T msol) {
  switch (kind) {
    case kMFEqual:
      return T(1);
    case kMFUniform:
    case kMFSalpeter: {
      if (ml == mu) return ml;
      T a = mf_slope<T>(kind);
      T b = 1 / pl_int(ml, mu, a);
      return pl_inv(p, ml, a, b);
    }
    case kMFKroupa: {
      if (ml == mu) return ml;
      Kroupa3<T> k;
      k.setup(ml, mu, msol);
      return k.draw(p, ml);
    }
    case kMFOpticalDepth: {
      if (ml == mu) return ml;
      if (p <= mu / (ml + mu)) return ml;
      return mu;
    }
  }
  return T(0);
}

// <m^(1+e)> (e = 0 or 1) or <m^2 ln m> (logm) of the mass function.
template <typename T>
T mf_moment(int kind, T ml, T mu, T msol, int which) {
  // which: 0 -> <m>, 1 -> <m^2>, 2 -> <m^2 ln m>
  switch (kind) {
    case kMFEqual:
      return which == 2 ? T(0) : T(1);
    case kMFUniform:
    case kMFSalpeter: {
      if (ml == mu) return which == 0 ? ml : (which == 1 ? ml * ml : ml * ml * xlog(ml));
      T a = mf_slope<T>(kind);
      T b = 1 / pl_int(ml, mu, a);
      if (which == 0) return pl_int(ml, mu, a + 1, b);
      if (which == 1) return pl_int(ml, mu, a + 2, b);
      return pl_log_int(ml, mu, a + 2, b);
    }
    case kMFKroupa: {
      if (ml == mu) return which == 0 ? ml : (which == 1 ? ml * ml : ml * ml * xlog(ml));
      Kroupa3<T> k;
      k.setup(ml, mu, msol);
      if (which == 0) return k.moment(ml, mu, 1, false);
      if (which == 1) return k.moment(ml, mu, 2, false);
      return k.moment(ml, mu, 2, true);
    }
    case kMFOpticalDepth: {
      if (ml == mu) return which == 0 ? ml : (which == 1 ? ml * ml : ml * ml * xlog(ml));
      if (which == 0) return 2 * ml * mu / (ml + mu);
      if (which == 1) return ml * mu;
      return ml * mu * (ml * xlog(ml) + mu * xlog(mu)) / (ml + mu);
    }
  }
  return T(0);
}

}  // namespace irsb
