// ixb_bodies.cpp -- immersed solid bodies as Patankar penalty sources (host
// only, no GPU): the masks of definir_cuerpo (source/mod_front_inmersa.f90:
// 54-179), for general boxes and line-bounded regions as well as the
// reference's three fixed shapes.
//
// Inside a body the linear source is -1e51 and the constant source 1e51 *
// value, so the node's equation reads T = value to working precision; u and
// v get the constant source 1e40, which holds them at 1e-11.  The reference
// tests every p node (xp(ii), yp(jj)), ii = 1..mi+1, jj = 1..nj+1, and
// writes the u, v and T source arrays at the same (ii, jj):
// it writes fuente_*_u at ii = mi+1 past the end of the (mi, nj+1) u arrays
// and fuente_*_v at jj = nj+1 past the end of the (mi+1, nj) v arrays.  Here
// those out-of-range writes are dropped; every in-range entry is the
// reference's.  'chime' also stores 1e41 into au/av at the body's nodes
// (:156, :160); the first u- and v-sweep assemblies overwrite every interior
// au/av before anything reads them, so that store has no effect and is not
// reproduced.
#include <cstddef>

#include "../../include/ixb.h"

namespace {

// A body: yl <= y <= yh and sl*y + cl <= x <= sh*y + ch (a box has sl = sh = 0)
struct Body {
  double yl, yh, sl, cl, sh, ch;
  bool vel;      // penalty sources on u and v
  bool temp;     // hold T at t_value
  double t_value;
};

// The penalty values exactly as the reference forms them (10.0e50,
// 10.0e50*10.0e-12, 10e50*1.0; mod_front_inmersa.f90:89-95, 153-163).
constexpr double kLin = -10.0e50;
const double kConVel = 10.0e50 * 10.0e-12;

bool inside(const Body& b, double x, double y) {
  if (!(b.yl <= y && y <= b.yh)) return false;
  const double x0 = b.sl == 0.0 ? b.cl : y * b.sl + b.cl;
  const double x1 = b.sh == 0.0 ? b.ch : y * b.sh + b.ch;
  return x0 <= x && x <= x1;
}

bool preset(int shape, Body* b) {
  switch (shape) {
    case IXB_BODY_TRIAN: {  // :73-99: vertex (6, 0.1), height 0.1; x between recta_mxb1 and recta_mxb2 of y
      const double yv = 0.1, hh = 0.1;
      const double m1 = 1.0 / 2.0, b1 = -(0.1 - m1 * 6.0) / m1;  // recta_mxb1, :210-215
      const double m2 = -1.0 / 2.0, b2 = -(0.1 - m2 * 6.0) / m2;  // recta_mxb2, :226-231
      *b = Body{yv - hh, yv, 1.0 / m1, b1, 1.0 / m2, b2, true, false, 0.0};
      return true;
    }
    case IXB_BODY_CUADR: {  // :101-133: square of side 0.1 centred on (6, 0.05)
      const double yv = 0.05, xv = 6.0, hh = 0.1;
      *b = Body{yv - hh / 2.0, yv + hh / 2.0, 0.0, xv - hh / 2.0, 0.0, xv + hh / 2.0, true, false, 0.0};
      return true;
    }
    case IXB_BODY_CHIME: {  // :135-177: square of side 0.3 centred on (8.5, 0.5), T held at 1
      const double yv = 0.5, xv = 8.5, hh = 0.3;
      *b = Body{yv - hh / 2.0, yv + hh / 2.0, 0.0, xv - hh / 2.0, 0.0, xv + hh / 2.0, true, true, 1.0};
      return true;
    }
    default:
      return false;
  }
}

}  // namespace

extern "C" int ixb_body_sources(int mi, int nj, const double* xp, const double* yp, int shape, const double* prm,
                                int flags, double t_value, double* fcon_u, double* flin_u, double* fcon_v,
                                double* flin_v, double* fcon_t, double* flin_t) {
  if (mi < 2 || nj < 2 || !xp || !yp) return IXB_EINVAL;
  Body b{};
  if (shape == IXB_BODY_BOX || shape == IXB_BODY_REGION) {
    if (!prm) return IXB_EINVAL;
    if (shape == IXB_BODY_BOX) b = Body{prm[2], prm[3], 0.0, prm[0], 0.0, prm[1], false, false, 0.0};
    else b = Body{prm[0], prm[1], prm[2], prm[3], prm[4], prm[5], false, false, 0.0};
    b.vel = (flags & IXB_BODY_VEL) != 0;
    b.temp = (flags & IXB_BODY_TEMP) != 0;
    b.t_value = t_value;
  } else if (!preset(shape, &b)) {
    return IXB_EINVAL;
  }
  if (b.vel && (!fcon_u || !flin_u || !fcon_v || !flin_v)) return IXB_EINVAL;
  if (b.temp && (!fcon_t || !flin_t)) return IXB_EINVAL;
  const double con_t = 10e50 * b.t_value;
  for (int jj = 1; jj <= nj + 1; ++jj)
    for (int ii = 1; ii <= mi + 1; ++ii) {
      if (!inside(b, xp[ii - 1], yp[jj - 1])) continue;
      if (b.vel) {
        if (ii <= mi) {  // u arrays (mi, nj+1)
          const size_t k = (size_t)(jj - 1) * mi + (ii - 1);
          flin_u[k] = kLin;
          fcon_u[k] = kConVel;
        }
        if (jj <= nj) {  // v arrays (mi+1, nj)
          const size_t k = (size_t)(jj - 1) * (mi + 1) + (ii - 1);
          flin_v[k] = kLin;
          fcon_v[k] = kConVel;
        }
      }
      if (b.temp) {  // T arrays (mi+1, nj+1)
        const size_t k = (size_t)(jj - 1) * (mi + 1) + (ii - 1);
        flin_t[k] = kLin;
        fcon_t[k] = con_t;
      }
    }
  return IXB_OK;
}
