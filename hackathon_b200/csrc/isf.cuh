// Swimmer self-ISF kernels on the device, with the log-derivatives the fits'
// Jacobians need: g(x; Z), x dg/dx and Z dg/dZ, x = q vbar tau.
//
//   3D (isf3d, motility_fit.js:140-144): the Schulz average of sin(qv tau)/(qv tau)
//      in closed form, sin(Z atan L) / (Z L (1+L^2)^(Z/2)), L = x/(Z+1);
//   2D (isf2d, motility_fit.js:152-159): the Schulz average of J0(q v tau),
//      P_Z(cos th) cos^(Z+1) th with th = atan L, P_Z the Legendre function.
//
// The 2D kernel has no closed form cheap enough for a fit, so it is read from
// a table built once per device (isf2d.cu): rows at 96 values of ln Z spaced
// evenly over [ln 0.5, ln 100]; along each row, P_Z(cos th) and dP/dth at
// evenly spaced th from 0 to the angle where cos^(Z+1) th = e^-25 (beyond it
// g = 0, the reference's cut-off), with a step that keeps the phase advance
// (Z + 1/2) h <= 0.08 rad. Within a row: cubic Hermite interpolation in th of
// P (exact node derivatives), times the prefactor cos^(Z+1) th evaluated
// exactly -- P is smooth up to th = pi/2, the prefactor is not polynomial
// there. Across rows: cubic Lagrange interpolation in ln Z at fixed x (g is
// smooth in Z at fixed x). Deviation from the exact Schulz average: < 5e-8
// over Z in [0.5, 100], x in [1e-3, 3e3]. Below L = 1e-4 both kernels use the
// reference's small-argument series.
#pragma once

#include <cuda_runtime.h>

namespace ddm {

constexpr int ISF2D_ROWS = 96;
constexpr int ISF2D_MAX_NODES = 32768;
constexpr double ISF2D_ZMIN = 0.5, ISF2D_ZMAX = 100.0;

struct Isf2dTable {
  const double2* node;  // (P_Z(cos th), dP/dth) at th = j h of each row
  const double4* row;   // per row: Z, h, th_end (last node), index of the row's first node
  double lz0, dlz;      // ln Z of row 0, row spacing in ln Z
};

// g, x dg/dx, Z dg/dZ of the 3D kernel (R = float or double).
template <typename R>
__device__ __forceinline__ void isf3d_d(R x, R Z, R& g, R& gx, R& gz);

template <>
__device__ __forceinline__ void isf3d_d<double>(double x, double Z, double& g, double& gx, double& gz) {
  const double Z1 = Z + 1.0;
  const double L = x / Z1;
  if (L < 1e-4) {
    const double x2 = x * x;
    g = 1.0 - x2 * (Z + 2.0) / (6.0 * Z1);
    gx = -2.0 * x2 * (Z + 2.0) / (6.0 * Z1);
    gz = x2 * Z / (6.0 * Z1 * Z1);
    return;
  }
  const double a = atan(L), u = 1.0 + L * L, lu = log1p(L * L);
  const double U = exp(0.5 * Z * lu);
  double s, c;
  sincos(Z * a, &s, &c);
  const double G = s / (Z * L * U);
  const double LgL = c / (u * U) - G * (1.0 + Z * L * L / u);
  g = G;
  gx = LgL;
  gz = a * c / (L * U) - G - 0.5 * Z * G * lu - (Z / Z1) * LgL;
}

template <>
__device__ __forceinline__ void isf3d_d<float>(float x, float Z, float& g, float& gx, float& gz) {
  const float Z1 = Z + 1.f;
  const float L = x / Z1;
  if (L < 1e-4f) {
    const float x2 = x * x;
    g = 1.f - x2 * (Z + 2.f) / (6.f * Z1);
    gx = -2.f * x2 * (Z + 2.f) / (6.f * Z1);
    gz = x2 * Z / (6.f * Z1 * Z1);
    return;
  }
  const float a = atanf(L), u = 1.f + L * L, lu = log1pf(L * L);
  const float U = expf(0.5f * Z * lu);
  float s, c;
  sincosf(Z * a, &s, &c);
  const float G = s / (Z * L * U);
  const float LgL = c / (u * U) - G * (1.f + Z * L * L / u);
  g = G;
  gx = LgL;
  gz = a * c / (L * U) - G - 0.5f * Z * G * lu - (Z / Z1) * LgL;
}

// One row of the 2D table at x: g and dg/dx.
__device__ __forceinline__ void isf2d_row(const Isf2dTable& t, int i, double x, double& g, double& dgdx) {
  const double4 r = t.row[i];
  const double Z = r.x, h = r.y, th_end = r.z, Z1 = Z + 1.0;
  const double L = x / Z1;
  if (L < 1e-4) {  // the reference's series, 1 - x^2 (Z+2) / (4 (Z+1))
    g = 1.0 - x * x * (Z + 2.0) / (4.0 * Z1);
    dgdx = -x * (Z + 2.0) / (2.0 * Z1);
    return;
  }
  const double th = atan(L);
  if (th >= th_end) {  // cos^(Z+1) th < e^-25
    g = 0.0;
    dgdx = 0.0;
    return;
  }
  const double u = th / h;
  const int m = (int)(th_end / h + 0.5);  // intervals in the row
  int j = (int)u;
  if (j > m - 1) j = m - 1;
  const double s = u - j;
  const int base = (int)r.w;
  const double2 a = t.node[base + j], b = t.node[base + j + 1];
  const double s2 = s * s, s3 = s2 * s;
  const double h00 = 2 * s3 - 3 * s2 + 1, h10 = s3 - 2 * s2 + s, h01 = -2 * s3 + 3 * s2, h11 = s3 - s2;
  const double d00 = 6 * s2 - 6 * s, d10 = 3 * s2 - 4 * s + 1, d01 = -6 * s2 + 6 * s, d11 = 3 * s2 - 2 * s;
  const double P = h00 * a.x + h10 * h * a.y + h01 * b.x + h11 * h * b.y;
  const double dP = (d00 * a.x + d10 * h * a.y + d01 * b.x + d11 * h * b.y) / h;
  const double pre = exp(-0.5 * Z1 * log1p(L * L));  // cos^(Z+1) th
  // d/dth [P pre] = dP pre - (Z+1) tan(th) P pre; dth/dx = 1 / ((Z+1) (1 + L^2))
  g = P * pre;
  dgdx = (dP - Z1 * L * P) * pre / (Z1 * (1.0 + L * L));
}

// g, x dg/dx, Z dg/dZ of the 2D kernel; Z is clamped to [0.5, 100] like the
// reference's tabulated kernel (isf2dFast, motility_fit.js:212-220).
__device__ __forceinline__ void isf2d_d(const Isf2dTable& t, double x, double Z, double& g, double& gx, double& gz) {
  const double Zc = fmin(ISF2D_ZMAX, fmax(ISF2D_ZMIN, Z));
  const double zf = (log(Zc) - t.lz0) / t.dlz;
  int i0 = (int)floor(zf) - 1;
  i0 = i0 < 0 ? 0 : (i0 > ISF2D_ROWS - 4 ? ISF2D_ROWS - 4 : i0);
  const double s = zf - i0;
  // cubic Lagrange weights on rows i0..i0+3 at s, and their s-derivatives
  const double w0 = -(s - 1) * (s - 2) * (s - 3) / 6, w1 = s * (s - 2) * (s - 3) / 2;
  const double w2 = -s * (s - 1) * (s - 3) / 2, w3 = s * (s - 1) * (s - 2) / 6;
  const double v0 = -((s - 2) * (s - 3) + (s - 1) * (s - 3) + (s - 1) * (s - 2)) / 6;
  const double v1 = ((s - 2) * (s - 3) + s * (s - 3) + s * (s - 2)) / 2;
  const double v2 = -((s - 1) * (s - 3) + s * (s - 3) + s * (s - 1)) / 2;
  const double v3 = ((s - 1) * (s - 2) + s * (s - 2) + s * (s - 1)) / 6;
  double g0, g1, g2, g3, x0, x1, x2, x3;
  isf2d_row(t, i0, x, g0, x0);
  isf2d_row(t, i0 + 1, x, g1, x1);
  isf2d_row(t, i0 + 2, x, g2, x2);
  isf2d_row(t, i0 + 3, x, g3, x3);
  g = w0 * g0 + w1 * g1 + w2 * g2 + w3 * g3;
  gx = x * (w0 * x0 + w1 * x1 + w2 * x2 + w3 * x3);
  const bool clamped = Z < ISF2D_ZMIN || Z > ISF2D_ZMAX;
  gz = clamped ? 0.0 : (v0 * g0 + v1 * g1 + v2 * g2 + v3 * g3) / t.dlz;
}

// Host: the table on the current device, built on first use (one kernel
// launch and a synchronisation; call it before any stream capture).
// Returns cudaSuccess and fills *out, or the error of the set-up.
cudaError_t isf2d_table(Isf2dTable* out);

}  // namespace ddm
