// Summation-by-parts first-derivative operators and Runge-Kutta tables.
//
// The coefficient values are FDMAP's own literals (fd_coeff.f90:83-246 for
// SBP2/SBP4/SBP6, time_step.f90:36-63 for the low-storage RK tables).  They are
// kept digit-for-digit -- including the 15-decimal truncation of fd_coeff.f90 --
// because bitwise agreement with FDMAP's operators is the point: replacing them
// with exact rationals would change every rate in the last few bits.
//
// Layout (0-based, C order):
//   sbp_DI[s]         interior weight of point i+s, s = 1..pI (antisymmetric:
//                     weight of i-s is -DI[s]); DI[0] = 0
//   sbp_DL[r][s]      left-boundary weight of point mgx+s (s = 0..nbnd-1) for the
//                     derivative at node mgx+r (r = 0..nbst-1)  == DL(s,r)
//   right boundary by symmetry: weight of point pgx-s at node pgx-r is -DL[r][s]
//                     (fd_coeff.f90:242-246, DR(-s,-r) = -DL(s,r))
#pragma once

#include "fdmap_desc.h"

namespace fdmap {

constexpr int SBP_MAX_NBND = 9;
constexpr int SBP_MAX_NBST = 6;
constexpr int SBP_MAX_PI = 3;

struct SbpOperator {
  int nI, nbnd, nbst, pI;
  double H00i;
  double DI[SBP_MAX_PI + 1];                    // DI[s] for s = 0..pI
  double DL[SBP_MAX_NBST][SBP_MAX_NBND];        // DL[r][s]
  double HL[SBP_MAX_NBST];
};

// Fills `op` for FDMAP_SBP2/4/6; returns false for an unknown method.
inline bool sbp_operator(int method, SbpOperator* op) {
  *op = SbpOperator{};
  switch (method) {
    case FDMAP_SBP2: {
      op->nI = 3; op->nbnd = 2; op->nbst = 1; op->H00i = 2.0;
      op->DI[1] = 0.5;
      op->DL[0][0] = -1.0; op->DL[0][1] = 1.0;
      op->HL[0] = 0.5;
      break;
    }
    case FDMAP_SBP4: {
      op->nI = 5; op->nbnd = 6; op->nbst = 4; op->H00i = 2.823529411764706;
      op->DI[1] = 0.666666666666667; op->DI[2] = -0.083333333333333;
      const double dl[4][6] = {
          {-1.411764705882353, 1.735294117647059, -0.235294117647059, -0.088235294117647, 0.0, 0.0},
          {-0.500000000000000, 0.000000000000000, 0.500000000000000, 0.000000000000000, 0.0, 0.0},
          {0.093023255813953, -0.686046511627907, 0.000000000000000, 0.686046511627907, -0.093023255813953, 0.0},
          {0.030612244897959, 0.000000000000000, -0.602040816326531, 0.000000000000000, 0.653061224489796, -0.081632653061224}};
      for (int r = 0; r < 4; ++r)
        for (int s = 0; s < 6; ++s) op->DL[r][s] = dl[r][s];
      const double hl[4] = {0.354166666666667, 1.229166666666667, 0.895833333333333, 1.020833333333333};
      for (int r = 0; r < 4; ++r) op->HL[r] = hl[r];
      break;
    }
    case FDMAP_SBP6: {
      op->nI = 7; op->nbnd = 9; op->nbst = 6; op->H00i = 3.165067037878233;
      op->DI[1] = 0.750000000000000; op->DI[2] = -0.150000000000000; op->DI[3] = 0.016666666666667;
      const double dl[6][9] = {
          {-1.582533518939116, 2.033378678700676, -0.141512858744873, -0.450398306578272, 0.104488069284042, 0.036577936277544, 0.0, 0.0, 0.0},
          {-0.462059195631158, 0.000000000000000, 0.287258622978251, 0.258816087376832, -0.069112065532624, -0.014903449191300, 0.0, 0.0, 0.0},
          {0.071247104721830, -0.636451095137907, 0.000000000000000, 0.606235523609147, -0.022902190275815, -0.018129342917256, 0.0, 0.0, 0.0},
          {0.114713313798970, -0.290087484386815, -0.306681191361148, 0.000000000000000, 0.520262285050482, -0.051642265516119, 0.013435342414630, 0.0, 0.0},
          {-0.036210680656541, 0.105400944933782, 0.015764336127392, -0.707905442575989, 0.000000000000000, 0.769199413962647, -0.164529643265203, 0.018281071473911, 0.0},
          {-0.011398193015050, 0.020437334208704, 0.011220896474665, 0.063183694641876, -0.691649024426814, 0.000000000000000, 0.739709139060752, -0.147941827812150, 0.016437980868017}};
      for (int r = 0; r < 6; ++r)
        for (int s = 0; s < 9; ++s) op->DL[r][s] = dl[r][s];
      const double hl[6] = {0.315949074074074, 1.390393518518518, 0.627546296296296,
                            1.240509259259259, 0.911689814814815, 1.013912037037037};
      for (int r = 0; r < 6; ++r) op->HL[r] = hl[r];
      break;
    }
    default:
      return false;
  }
  op->pI = (op->nI - 1) / 2;
  return true;
}

struct RkTable {
  int nstage;
  double A[5], B[5], C[6];
};

// Low-storage RK coefficients of order 1..4 (time_step.f90:36-63); the
// rationals are evaluated in double exactly as the Fortran literals are.
inline bool rk_table(int order, RkTable* rk) {
  *rk = RkTable{};
  switch (order) {
    case 1:
      rk->nstage = 1; rk->A[0] = 0.0; rk->B[0] = 1.0; rk->C[0] = 0.0; rk->C[1] = 1.0;
      return true;
    case 2:
      rk->nstage = 2; rk->A[0] = 0.0; rk->A[1] = -1.0; rk->B[0] = 1.0; rk->B[1] = 1.0 / 2.0;
      rk->C[0] = 0.0; rk->C[1] = 1.0; rk->C[2] = 1.0;
      return true;
    case 3:
      rk->nstage = 3;
      rk->A[0] = 0.0; rk->A[1] = -5.0 / 9.0; rk->A[2] = -153.0 / 128.0;
      rk->B[0] = 1.0 / 3.0; rk->B[1] = 15.0 / 16.0; rk->B[2] = 8.0 / 15.0;
      rk->C[0] = 0.0; rk->C[1] = 1.0 / 3.0; rk->C[2] = 3.0 / 4.0; rk->C[3] = 1.0;
      return true;
    case 4:
      rk->nstage = 5;
      rk->A[0] = 0.0;
      rk->A[1] = -567301805773.0 / 1357537059087.0;
      rk->A[2] = -2404267990393.0 / 2016746695238.0;
      rk->A[3] = -3550918686646.0 / 2091501179385.0;
      rk->A[4] = -1275806237668.0 / 842570457699.0;
      rk->B[0] = 1432997174477.0 / 9575080441755.0;
      rk->B[1] = 5161836677717.0 / 13612068292357.0;
      rk->B[2] = 1720146321549.0 / 2090206949498.0;
      rk->B[3] = 3134564353537.0 / 4481467310338.0;
      rk->B[4] = 2277821191437.0 / 14882151754819.0;
      rk->C[0] = 0.0;
      rk->C[1] = 1432997174477.0 / 9575080441755.0;
      rk->C[2] = 2526269341429.0 / 6820363962896.0;
      rk->C[3] = 2006345519317.0 / 3224310063776.0;
      rk->C[4] = 2802321613138.0 / 2924317926251.0;
      rk->C[5] = 1.0;
      return true;
    default:
      return false;
  }
}

}  // namespace fdmap
