// Per-node formulas of FDMAP's body initialisation, shared by the host
// restatement of init_domain (host_init.cpp) and the device body builder
// (body_init.cu).  Both sides evaluate exactly these expressions, in this
// order and without fused multiply-adds (the device file is compiled with
// -fmad=false, the host with no FMA target), so a body built on the device is
// bit-identical to the host's: + - * / and sqrt are correctly rounded on both.
// The one exception is exp() in the 'smooth' and 'gaussian' perturbation
// shapes, whose host and device implementations may differ in the last bit.
#pragma once

#include <cmath>

#include "sbp_tables.h"

#ifdef __CUDACC__
#define FDMAP_HD __host__ __device__
#else
#define FDMAP_HD
#endif

namespace fdmap {

// transfinite_interp (geometry.f90:153-200): one coordinate of the node at
// index coordinates (q, r) from the four edge curves' values cL(r), cR(r),
// cB(q), cT(q) and the four corners.
FDMAP_HD inline double transfinite(double q, double r, double qmin, double qmax, double rmin, double rmax, double Wq,
                                   double Wr, double cL, double cR, double cB, double cT, double LB, double LT,
                                   double RB, double RT) {
  return (qmax - q) * cL / Wq + (q - qmin) * cR / Wq + (rmax - r) * cB / Wr + (r - rmin) * cT / Wr -
         (qmax - q) * (rmax - r) * LB / (Wq * Wr) - (qmax - q) * (r - rmin) * LT / (Wq * Wr) -
         (q - qmin) * (rmax - r) * RB / (Wq * Wr) - (q - qmin) * (r - rmin) * RT / (Wq * Wr);
}

// SBP first derivative with unit spacing (fd.f90:42-80) at point i of a line
// of n >= 2*nbst values f(0..n-1): DL rows at the two ends (DR = -DL mirrored),
// the interior stencil DI summed from s = -pI upward including its zero centre.
template <class DLT, class Get>
FDMAP_HD inline double sbp_diff_at(int nbst, int nbnd, int pI, const double* DI, const DLT& DL, int n, int i,
                                   const Get& f) {
  double s = 0.0;
  if (i < nbst) {
    for (int k = 0; k < nbnd; ++k) s = s + DL[i][k] * f(k);
  } else if (i > n - 1 - nbst) {
    const int r = n - 1 - i;
    for (int k = 0; k < nbnd; ++k) {
      double w = -DL[r][nbnd - 1 - k];
      s = s + w * f(n - nbnd + k);
    }
  } else {
    for (int q = -pI; q <= pI; ++q) {
      double w = q < 0 ? -DI[-q] : (q == 0 ? 0.0 : DI[q]);
      s = s + w * f(i + q);
    }
  }
  return s;
}

// grid spacing at a node (set_dt, domain.f90:1481-1495): the distances
// |J| / |x_r| and |J| / |x_q| whose minimum and maximum are hmin and hmax
FDMAP_HD inline double spacing_q(double J, double xr, double yr) { return fabs(J / sqrt(xr * xr + yr * yr)); }
FDMAP_HD inline double spacing_r(double J, double xq, double yq) { return fabs(J / sqrt(xq * xq + yq * yq)); }

// utilities.f90 shape functions (utilities.f90:303-420)
constexpr double kShapeTol = 100.0 * 2.220446049250313e-16;  // 100d0*epsilon(r)

FDMAP_HD inline double shape_boxcar(double r, double w, double fin, double fout) {
  if (-w + kShapeTol < r && r < w - kShapeTol) return fin;
  if (fabs(-w - r) <= kShapeTol || fabs(r - w) <= kShapeTol) return 0.5 * (fin + fout);
  return fout;
}
FDMAP_HD inline double shape_gaussian(double r, double w, double fin, double fout) {
  return fout + (fin - fout) * exp(-0.5 * ((r / w) * (r / w)));
}
FDMAP_HD inline double shape_smooth(double r, double w, double fin, double fout) {
  if (r >= w - kShapeTol) return fout;
  return fout + (fin - fout) * exp((r * r) / ((r * r) - (w * w)));
}
FDMAP_HD inline double shape_triangle(double r, double w, double fin, double fout) {
  if (-w < r && r < w) return fout + (fin - fout) * (1.0 - r / w);
  return fout;
}

// amplitude of one fields_perturb item at (x, y) (perturb_fields, fields.f90:900-934)
FDMAP_HD inline double perturb_amp(int shape, double x, double y, double x0, double y0, double Lx, double Ly) {
  double a = (x - x0) / Lx, b = (y - y0) / Ly;
  double r = sqrt(a * a + b * b);
  switch (shape) {
    case 1: return (x - x0) / Lx + (y - y0) / Ly;  // FDMAP_PERTURB_LINEAR
    case 2: return shape_boxcar(r, 1.0, 1.0, 0.0);
    case 3: return shape_triangle(r, 1.0, 1.0, 0.0);
    case 4: return shape_smooth(r, 1.0, 1.0, 0.0);
    case 5: return shape_gaussian(r, 1.0, 1.0, 0.0);
    default: return 0.0;
  }
}

// edge impedances of one side node (init_edges, domain.f90:1349-1459):
// M = (Zs, Zp, gamma, Ks, Kp) from the material and |grad| of the metric
// along the side and the Jacobian at the node
FDMAP_HD inline void edge_impedances(double rho, double cs, double cp, double mag, double J, double H00i, double* M,
                                     long long stride) {
  M[0] = rho * cs;
  M[stride] = rho * cp;
  M[2 * stride] = 1.0 - 2.0 * ((cs / cp) * (cs / cp));
  M[3 * stride] = H00i * cs * mag / J;
  M[4 * stride] = H00i * cp * mag / J;
}

// set_dt (domain.f90:1462-1535) with the refinement of main.f90:92-116, from
// the input dt, CFL, refine, tend and nt, the fastest wave speed
// c = sqrt(cs^2 + cp^2) and the minimum grid spacing.
inline void finish_time_step(double dt_in, double CFL_in, double refine, double tend, int nt_in, double c, double hmin,
                             double* dt_out, double* CFL_out, int* nt_out) {
  double dt = dt_in / refine, CFL = CFL_in;
  if (CFL == 0.0) {
    if (dt == 0.0) { CFL = 0.5; dt = CFL * hmin / c; }
    else CFL = c * dt / hmin;
  } else {
    if (dt == 0.0) dt = CFL * hmin / c;
    else CFL = c * dt / hmin;
  }
  int nt;
  if (nt_in == 0) nt = (int)std::ceil(tend / dt);
  else nt = (int)std::ceil((double)(nt_in - 1) * refine) + 1;
  *dt_out = dt; *CFL_out = CFL; *nt_out = nt;
}

}  // namespace fdmap
