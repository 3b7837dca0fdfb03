// Fused stage kernel: for every node of every block, in one pass over HBM,
//   DF <- A*DF                                   (scale_rates_interior, fields.f90:1061)
//   DF += SAT penalty (sides L, R, B, T)         (set_rates_SAT, time_step.f90:754-851)
//   DF += SBP split-form rates                   (rates.f90 / rates_heterogeneous.f90)
//   DF6 <- nu*(DF3+DF5)  (mode II, plane strain) (rates_szz, rates.f90:920-936)
//   DF += point source / gravity                 (set_source, source.f90:147-252)
//   F_out <- F_in + (B*dt)*DF                    (update_fields_interior, fields.f90:1167)
// Interior nodes read their cross-shaped neighbourhood from a shared-memory
// tile loaded once per CTA; nodes inside the SBP boundary closures (within
// nbst of a block edge) take a slower path through L1/L2 that applies the
// one-sided DL/DR rows exactly like rates_boundary_mode2/3.
#pragma once

#include "edge_kernel.cuh"

namespace fdmap {

// Rate components as flat sums of metric-average x field products
// (rates.f90:30-49, 407-444): the Y-metric term uses field fa, the X-metric
// term field fb, optionally times gamma; coef 0: DI/rho, 1: DI*G, 2: DI*M.
template <int MODE> struct RDef;
template <> struct RDef<2> {
  static constexpr int NR = 5;
  __host__ __device__ static constexpr int fa(int r) { return r == 0 ? 2 : r == 1 ? 3 : r == 2 ? 0 : r == 3 ? 1 : 0; }
  __host__ __device__ static constexpr int fb(int r) { return r == 0 ? 3 : r == 1 ? 4 : r == 2 ? 1 : r == 3 ? 0 : 1; }
  __host__ __device__ static constexpr bool ga(int r) { return r == 4; }
  __host__ __device__ static constexpr bool gb(int r) { return r == 2; }
  __host__ __device__ static constexpr int coef(int r) { return r < 2 ? 0 : (r == 3 ? 1 : 2); }
};
template <> struct RDef<3> {
  static constexpr int NR = 3;
  __host__ __device__ static constexpr int fa(int r) { return r == 0 ? 1 : r == 1 ? 0 : -1; }
  __host__ __device__ static constexpr int fb(int r) { return r == 0 ? 2 : r == 1 ? -1 : 0; }
  __host__ __device__ static constexpr bool ga(int) { return false; }
  __host__ __device__ static constexpr bool gb(int) { return false; }
  __host__ __device__ static constexpr int coef(int r) { return r == 0 ? 0 : 1; }
};

constexpr int TX = 32;
constexpr int TY = 8;

struct NodeMat {
  double rho, G, M, gamma, nu;
  double rinv;  // 1/rho
};

__device__ __forceinline__ double mat_coef(const NodeMat& m, int kind, double w) {
  // w/rho, w*G, w*M (the division is taken once per node through rinv)
  return kind == 0 ? w * m.rinv : (kind == 1 ? w * m.G : w * m.M);
}

// Split-form rates of one interior node (rates_interior_mode2/3,
// rates.f90:8-56, 384-450; heterogeneous media rates_heterogeneous.f90), added
// to acc.  Every interior kernel that reads its neighbourhood from a
// shared-memory ring or from global memory calls this one routine, so the
// same inputs give the same bits whichever kernel computes the node.
// Accessors (s = +-1 .. +-PI, 0 the node itself):
//   fq(l, s) field l at column offset s,   fr(l, s) field l at row offset s;
//   mq(0, s) yr, mq(1, s) xr at column offset s;
//   mr(0, s) yq, mr(1, s) xq at row offset s.
template <int MODE, int PI_, bool HET, class FQ, class FR, class MQ, class MRr>
__device__ __forceinline__ void split_rates(double* acc, const NodeMat& m, const double (&cf)[PI_ + 1][3],
                                            const double* DI, double Ji, FQ&& fq, FR&& fr, MQ&& mq, MRr&& mr) {
  using RD = RDef<MODE>;
  const double yrc = mq(0, 0), xrc = mq(1, 0);
  const double yqc = mr(0, 0), xqc = mr(1, 0);
#pragma unroll
  for (int s = 1; s <= PI_; ++s) {
    const double Yrp = 0.5 * (mq(0, s) + yrc), Xrp = 0.5 * (mq(1, s) + xrc);
    const double Yrm = 0.5 * (mq(0, -s) + yrc), Xrm = 0.5 * (mq(1, -s) + xrc);
    const double Yqp = 0.5 * (mr(0, s) + yqc), Xqp = 0.5 * (mr(1, s) + xqc);
    const double Yqm = 0.5 * (mr(0, -s) + yqc), Xqm = 0.5 * (mr(1, -s) + xqc);
    const double w = HET ? DI[s] : 0.0;
#pragma unroll
    for (int r = 0; r < RD::NR; ++r) {
      double sum = 0.0;
      if (RD::fa(r) >= 0) {
        const int f = RD::fa(r);
        double t = Yrp * fq(f, s) - Yrm * fq(f, -s) - Yqp * fr(f, s) + Yqm * fr(f, -s);
        if (RD::ga(r)) t *= m.gamma;
        sum += t;
      }
      if (RD::fb(r) >= 0) {
        const int f = RD::fb(r);
        double t = -Xrp * fq(f, s) + Xrm * fq(f, -s) + Xqp * fr(f, s) - Xqm * fr(f, -s);
        if (RD::gb(r)) t *= m.gamma;
        sum += t;
      }
      const double cfr = HET ? mat_coef(m, RD::coef(r), w) : cf[s][RD::coef(r)];
      acc[r] += sum * cfr * Ji;
    }
  }
}

// flux of rate r at point k: q direction +t1 - t2 (Yr, Xr), r direction -t1 + t2 (Yq, Xq);
// r is a compile-time constant after unrolling, so the table lookups fold away
template <int MODE>
__device__ __forceinline__ double flux(int r, double Ym, double Xm, const double* Fk, double g, bool qdir) {
  using RD = RDef<MODE>;
  double v = 0.0;
  if (RD::fa(r) >= 0) {
    double t = Ym * Fk[RD::fa(r)];
    if (RD::ga(r)) t *= g;
    v = qdir ? t : -t;
  }
  if (RD::fb(r) >= 0) {
    double t = Xm * Fk[RD::fb(r)];
    if (RD::gb(r)) t *= g;
    v = qdir ? v - t : v + t;
  }
  return v;
}

// Closure-region rates for node (i, j) read through the cache hierarchy
// (rates_boundary_mode2/3 and the heterogeneous variants).
__host__ __device__ constexpr int nbnd_of(int pI) { return pI == 1 ? 2 : (pI == 2 ? 6 : 9); }

template <int MODE, int PI_, bool PLAIN = false>
__device__ __forceinline__ void closure_rates(const DevDomain& D, const DevBlock& B, const double* __restrict__ Fin, int i, int j,
                              const NodeMat& m, double Ji, double* acc) {
  using RD = RDef<MODE>;
  constexpr int NR = RD::NR;
  constexpr int nbnd = nbnd_of(PI_);  // one-sided stencil width (fd_coeff.f90:57-70)
  const int nx = B.nx, ny = B.ny, nbst = D.nbst;
  const long long pitch = B.pitch, plane = B.plane;
  const long long c = (long long)j * pitch + i;
  const int qreg = i < nbst ? 0 : (i > nx - 1 - nbst ? 1 : -1);
  const int rreg = j < nbst ? 0 : (j > ny - 1 - nbst ? 1 : -1);
  const double yrc = B.yr[c], xrc = B.xr[c], yqc = B.yq[c], xqc = B.xq[c];
  auto loadF = [&](long long k, double* Fk) {
#pragma unroll
    for (int l = 0; l < (MODE == 2 ? 5 : 3); ++l) Fk[l] = Fin[l * plane + k];
  };
  auto qterm = [&](long long k, double w, int sgn) {
    double Fk[5];
    loadF(k, Fk);
    double Y = 0.5 * (B.yr[k] + yrc), X = 0.5 * (B.xr[k] + xrc);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      double f = flux<MODE>(r, Y, X, Fk, m.gamma, true);
      acc[r] += (sgn * f) * mat_coef(m, RD::coef(r), w) * Ji;
    }
  };
  auto rterm = [&](long long k, double w, int sgn) {
    double Fk[5];
    loadF(k, Fk);
    double Y = 0.5 * (B.yq[k] + yqc), X = 0.5 * (B.xq[k] + xqc);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      double f = flux<MODE>(r, Y, X, Fk, m.gamma, false);
      acc[r] += (sgn * f) * mat_coef(m, RD::coef(r), w) * Ji;
    }
  };
  auto qone = [&](int s, double& w, long long& k) {
    if (qreg == 0) { w = D.DL[i][s]; k = (long long)j * pitch + s; }
    else { w = -D.DL[nx - 1 - i][s]; k = (long long)j * pitch + (nx - 1 - s); }
  };
  auto rone = [&](int s, double& w, long long& k) {
    if (rreg == 0) { w = D.DL[j][s]; k = (long long)s * pitch + i; }
    else { w = -D.DL[ny - 1 - j][s]; k = (long long)(ny - 1 - s) * pitch + i; }
  };
  if (qreg >= 0 && rreg >= 0) {
#pragma unroll
    for (int s = 0; s < nbnd; ++s) {
      double w; long long k;
      qone(s, w, k);
      qterm(k, w, 1);
      rone(s, w, k);
      rterm(k, w, 1);
    }
  } else if (qreg >= 0) {
#pragma unroll
    for (int s = 0; s < nbnd; ++s) {
      double w; long long k;
      qone(s, w, k);
      qterm(k, w, 1);
    }
#pragma unroll
    for (int s = 1; s <= PI_; ++s) {
      rterm(c + s * pitch, D.DI[s], 1);
      rterm(c - s * pitch, D.DI[s], -1);
    }
  } else {
#pragma unroll
    for (int s = 0; s < nbnd; ++s) {
      double w; long long k;
      rone(s, w, k);
      rterm(k, w, 1);
    }
#pragma unroll
    for (int s = 1; s <= PI_; ++s) {
      qterm(c + s, D.DI[s], 1);
      qterm(c - s, D.DI[s], -1);
    }
  }
  if (!PLAIN && B.Cdiss > 0.0) {
    // artificial dissipation (rates_dissipation_boundary_mode2/3, rates.f90:1002-1394,
    // 1485-2021): J-weighted AL rows (AR mirrors AL without a sign change) in a
    // one-sided direction, AI in a central one, and AI(0)*F once per central direction
    const double Cd = B.Cdiss;
    auto diss = [&](long long k, double wa) {
      const double Jk = B.J[k];
#pragma unroll
      for (int l = 0; l < NR; ++l) acc[l] += Jk * Fin[l * plane + k] * wa * Ji * Cd;
    };
    if (qreg >= 0) {
#pragma unroll
      for (int s = 0; s < nbnd; ++s)
        diss((long long)j * pitch + (qreg == 0 ? s : nx - 1 - s), qreg == 0 ? D.AL[i][s] : D.AL[nx - 1 - i][s]);
    } else {
#pragma unroll
      for (int s = 1; s <= PI_; ++s) { diss(c + s, D.AI[s]); diss(c - s, D.AI[s]); }
    }
    if (rreg >= 0) {
#pragma unroll
      for (int s = 0; s < nbnd; ++s)
        diss((long long)(rreg == 0 ? s : ny - 1 - s) * pitch + i, rreg == 0 ? D.AL[j][s] : D.AL[ny - 1 - j][s]);
    } else {
#pragma unroll
      for (int s = 1; s <= PI_; ++s) { diss(c + s * pitch, D.AI[s]); diss(c - s * pitch, D.AI[s]); }
    }
    const double ncentral = (qreg < 0 ? 1.0 : 0.0) + (rreg < 0 ? 1.0 : 0.0);
#pragma unroll
    for (int l = 0; l < NR; ++l) acc[l] += ncentral * D.AI[0] * Cd * Fin[l * plane + c];
  }
}

// Hat variables of an outer-boundary node depend only on the node's own fields
// (set_bc, boundaries.f90:132-377), so they are evaluated where they are used
// and stored for inspection.
template <int MODE>
__device__ __forceinline__ void bc_hat(const DevSide& S, int k, const double* F, double* Fh) {
  constexpr int NF = MODE == 2 ? 6 : 3;
  double F0[6];
#pragma unroll
  for (int l = 0; l < NF; ++l) F0[l] = S.F0[k + S.n * l];
  d_set_bc<MODE>(Fh, F, F0, S.nrm[k], S.nrm[k + S.n], S.bc, S.M[k], S.M[k + S.n], S.M[k + 2 * S.n]);
#pragma unroll
  for (int l = 0; l < NF; ++l) S.Fhat[k + S.n * l] = Fh[l];
}

// SAT penalty (SAT_term / split_sp, time_step.f90:813-851) with hat variables Fh
template <int MODE>
__device__ __forceinline__ void sat_apply(const DevSide& S, int k, const double* F, const double* Fh, double* acc) {
  constexpr int NF = MODE == 2 ? 6 : 3;
  double Ks = S.M[k + 3 * S.n], Kp = S.M[k + 4 * S.n];
  double d[6];
#pragma unroll
  for (int l = 0; l < NF; ++l) d[l] = Fh[l] - F[l];
  if (MODE == 3) {
#pragma unroll
    for (int l = 0; l < 3; ++l) acc[l] += Ks * d[l];
  } else {
    double n0 = S.nrm[k], n1 = S.nrm[k + S.n];
    double r[6], Fs[6], Fp[6];
    rot2_xy2nt(d, n0, n1, r);
    rot2_nt2xy(Fs, n0, n1, r[0], 0.0, 0.0, r[3], 0.0, 0.0);
    rot2_nt2xy(Fp, n0, n1, 0.0, r[1], r[2], 0.0, r[4], r[5]);
#pragma unroll
    for (int l = 0; l < 6; ++l) acc[l] += Ks * Fs[l];
#pragma unroll
    for (int l = 0; l < 6; ++l) acc[l] += Kp * Fp[l];
  }
}

// SAT of side s for the node with fields F: hat variables from `Fh_given` when
// s == iside (an interface solve done by the caller), evaluated in place on
// an outer boundary, or read back from the interface kernel's output.
template <int MODE>
__device__ __forceinline__ void sat_term(const DevSide& S, int s, int k, const double* F, double* acc, int iside,
                                         const double* Fh_given, const StageArgs& a) {
  constexpr int NF = MODE == 2 ? 6 : 3;
  double Fh[6];
  if (s == iside) {
#pragma unroll
    for (int l = 0; l < NF; ++l) Fh[l] = Fh_given[l];
  } else if (S.bc != FDMAP_BC_NONE && !(k >= S.cov_lo && k < S.cov_hi)) {
    bc_hat<MODE>(S, k, F, Fh);
  } else {
#pragma unroll
    for (int l = 0; l < NF; ++l) Fh[l] = S.Fhat[k + S.n * l];
  }
  sat_apply<MODE>(S, k, F, Fh, acc);
  if (S.U) {
    // boundary displacement: DU <- A*DU + Fhat(:, 1:nU), U <- U + Bdt*DU
    // (scale_rates_boundary / set_rates_boundary / update_fields_boundary,
    // fields.f90:1083-1276); the stage-1 U is kept for the output
    constexpr int NU = MODE == 2 ? 2 : 1;
#pragma unroll
    for (int c = 0; c < NU; ++c) {
      const long long q = k + (long long)S.n * c;
      const double u = S.U[q];
      double du = a.scale ? (a.A != 0.0 ? a.A * S.DU[q] : 0.0) : S.DU[q];
      du = du + Fh[c];
      S.DU[q] = du;
      if (a.tap && S.Utap) S.Utap[q] = u;
      if (a.update) S.U[q] = u + a.Bdt * du;
    }
  }
}

// singular source amplitude (source.f90:208-223)
__device__ __forceinline__ double stf_amp(const fdmap_source& S, double t) {
  const double pi = 3.14159265358979323846264338327950288;
  double tc = t - S.t_center;
  switch (S.stf) {
    case FDMAP_STF_RAMP: return fmax(fmin(tc / S.t_duration, 1.0), 0.0);
    case FDMAP_STF_SINUSOID: return sin(2.0 * pi * tc / S.t_duration);
    case FDMAP_STF_GAUSSIAN: return exp(-0.5 * (tc * tc) / (S.t_duration * S.t_duration));
    default:
      return (1.0 - 2.0 * (pi * pi) * (tc * tc) / (S.t_duration * S.t_duration)) *
             exp(-(pi * pi) * (tc * tc) / (S.t_duration * S.t_duration));
  }
}

// body forces (set_source, source.f90:147-324) at block-local node (i, j):
// gravity, the point source, tsunami forcing and forcing from file, in that order
// PLAIN: the domain has no long-wave forcing and no forcing file, so only
// gravity and the point source are compiled in.
template <int MODE, bool PLAIN = false>
__device__ __forceinline__ void body_forces(const DevDomain& D, const DevBlock& B, int i, int j, double t,
                                            const StageArgs& a, double* acc) {
  if (D.src.use_gravity) {
    if (MODE == 2) { acc[0] += D.src.gx; acc[1] += D.src.gy; }
    else acc[0] += D.src.gz;
  }
  if (D.src.use_singular) {
    // a point source outside the block ends set_source for it (source.f90:200-206)
    if (!B.src_ok) return;
    int di = i - B.src_i0, dj = j - B.src_j0;
    if (di >= -2 && di <= 2 && dj >= -2 && dj <= 2) {
      double A = stf_amp(D.src, t);
      double dx = B.src_wx[di + 2], dy = B.src_wy[dj + 2];
      if (MODE == 2) {
        acc[0] += A * D.src.Fx * dx * dy / B.rho_b;
        acc[1] += A * D.src.Fy * dx * dy / B.rho_b;
        acc[2] -= A * D.src.Mxx * dx * dy;
        acc[3] -= A * D.src.Mxy * dx * dy;
        acc[4] -= A * D.src.Myy * dx * dy;
      } else {
        acc[0] += A * D.src.Fz * dx * dy / B.rho_b;
        acc[1] -= A * D.src.Mzx * dx * dy;
        acc[2] -= A * D.src.Mzy * dx * dy;
      }
    }
  }
  if constexpr (PLAIN) return;
  const long long c = (long long)j * B.pitch + i;
  if (MODE == 3 && B.gforce) {
    // problem = 'Forcing' (source.f90:299-312); the spatial factor is per node
    const double pi = 3.14159265358979323846264338327950288;
    const double u = (t - 4.0 * D.src.gauss_sigmat) / D.src.gauss_sigmat;
    acc[0] = acc[0] + B.gforce[c] * exp(-0.5 * (u * u)) / (D.src.gauss_sigmat * sqrt(2.0 * pi));
  }
  if (B.frc_new) {
    // forcing from file, interpolated linearly in time (source.f90:315-322)
    double t_old, t_new;
    step_window(a, t_old, t_new);
    const double w_old = (t_new - t) / (t_new - t_old), w_new = 1.0 - w_old;
    constexpr int NF = MODE == 2 ? 6 : 3;
#pragma unroll
    for (int l = 0; l < NF; ++l)
      acc[l] = acc[l] + w_old * B.frc_old[l * B.plane + c] + w_new * B.frc_new[l * B.plane + c];
  }
}

// body displacement and peak motion of one node, after its rates are complete:
// DU <- A*DU + F(1:nU), U <- U + Bdt*DU (scale_rates_interior,
// set_rates_displacement, update_fields_interior, fields.f90:1060-1258), the
// stage-1 U kept for the output; in stage 1 pgv <- max(pgv, |v|),
// pga <- max(pga, |dv/dt|) (update_fields_peak, fields.f90:1136-1164)
template <int MODE>
__device__ __forceinline__ void body_extras(const DevBlock& B, long long c, const double* Fc, const double* acc,
                                            const StageArgs& a) {
  if (B.DU) {
    constexpr int NU = MODE == 2 ? 2 : 1;
#pragma unroll
    for (int l = 0; l < NU; ++l) {
      const long long q = l * B.plane + c;
      const double u = B.U[q];
      double du = a.A != 0.0 ? a.A * B.DU[q] : 0.0;
      du = du + Fc[l];
      B.DU[q] = du;
      if (a.tap && B.Utap) B.Utap[q] = u;
      if (a.update) B.U[q] = u + a.Bdt * du;
    }
  }
  if (B.pgv && a.first) {
    double v, dv;
    if (MODE == 2) {
      v = sqrt(Fc[0] * Fc[0] + Fc[1] * Fc[1]);
      dv = sqrt(acc[0] * acc[0] + acc[1] * acc[1]);
    } else {
      v = fabs(Fc[0]);
      dv = fabs(acc[0]);
    }
    B.pgv[c] = fmax(B.pgv[c], v);
    B.pga[c] = fmax(B.pga[c], dv);
  }
}

__device__ __forceinline__ bool interior_node(const DevDomain& D, const DevBlock& B, int i, int j) {
  return i >= D.nbst && i <= B.nx - 1 - D.nbst && j >= D.nbst && j <= B.ny - 1 - D.nbst;
}


// Perfectly matched layer, mode II (rates_interior_mode2_pml and
// rates_boundary_mode2_pml, rates.f90:2024-2619): the rates of a PML block at
// node (i, j), added to acc (the scaled rates plus SAT) in place of the
// curvilinear split form.  Cartesian differences are scaled by hxi = Ji*yr,
// hyi = Ji*xq taken at the first node of the node's region; the auxiliary
// fields Wx, Wy of the node are read, their rates scaled by A, formed here and
// written back, and on update stages W += Bdt*DW (scale_rates_interior /
// update_fields_interior, fields.f90:1060-1186).  The reference's interior
// loop runs to s = 3 with DI(s) = 0 beyond pI; those exact zeros are left out.
template <int PI_>
__device__ __forceinline__ void pml_rates(const DevDomain& D, const DevBlock& B, const double* __restrict__ Fin, int i,
                                          int j, const StageArgs& a, double* acc) {
  constexpr int NBND = nbnd_of(PI_);
  constexpr int NF = 6;
  const int nbst = D.nbst, nx = B.nx, ny = B.ny;
  const long long pitch = B.pitch, plane = B.plane;
  const long long c = (long long)j * pitch + i;
  const int qreg = i < nbst ? 0 : (i > nx - 1 - nbst ? 1 : 2);
  const int rreg = j < nbst ? 0 : (j > ny - 1 - nbst ? 1 : 2);
  const double hxi = B.pml_h[(qreg * 3 + rreg) * 2], hyi = B.pml_h[(qreg * 3 + rreg) * 2 + 1];
  const double sx = B.pml_s[c], sy = B.pml_s[plane + c];
  const double rho = B.rho_b, G = B.G_b, M = B.M_b, gamma = B.gamma_b;
  const bool onx = B.pml & 1, ony = (B.pml >> 1) & 1;
  const bool load = a.scale && a.A != 0.0;
  double dwx[NF], dwy[NF];
  if (onx) {
    double w[NF];
#pragma unroll
    for (int l = 0; l < NF; ++l) {
      w[l] = B.Wx[l * plane + c];
      dwx[l] = load ? a.A * B.DWx[l * plane + c] : 0.0;
    }
    acc[0] = acc[0] - w[2] / rho;
    acc[1] = acc[1] - w[3] / rho;
    acc[2] = acc[2] - w[0] * M;
    acc[3] = acc[3] - w[1] * G;
    acc[4] = acc[4] - w[0] * gamma * M;
#pragma unroll
    for (int l = 0; l < NF; ++l) dwx[l] = dwx[l] - (sx + B.pml_kappa) * w[l];
  }
  if (ony) {
    double w[NF];
#pragma unroll
    for (int l = 0; l < NF; ++l) {
      w[l] = B.Wy[l * plane + c];
      dwy[l] = load ? a.A * B.DWy[l * plane + c] : 0.0;
    }
    acc[0] = acc[0] - w[3] / rho;
    acc[1] = acc[1] - w[4] / rho;
    acc[2] = acc[2] - w[1] * gamma * M;
    acc[3] = acc[3] - w[0] * G;
    acc[4] = acc[4] - w[1] * M;
#pragma unroll
    for (int l = 0; l < NF; ++l) dwy[l] = dwy[l] - (sy + B.pml_kappa) * w[l];
  }
  double f[NF];
  auto at = [&](int ii, int jj) {
    const long long k = (long long)jj * pitch + ii;
#pragma unroll
    for (int l = 0; l < NF; ++l) f[l] = Fin[l * plane + k];
  };
  auto diff = [&](int ip, int jp, int im, int jm) {
    const long long kp = (long long)jp * pitch + ip, km = (long long)jm * pitch + im;
#pragma unroll
    for (int l = 0; l < NF; ++l) f[l] = Fin[l * plane + kp] - Fin[l * plane + km];
  };
  // q- and r-direction contributions of the point values (or differences) f with weight w
  auto qterm = [&](double w) {
    if (onx) {
#pragma unroll
      for (int l = 0; l < NF; ++l) dwx[l] = dwx[l] + sx * hxi * f[l] * w;
    }
    acc[0] = acc[0] + hxi * f[2] * w / rho;
    acc[1] = acc[1] + hxi * f[3] * w / rho;
    acc[2] = acc[2] + hxi * f[0] * w * M;
    acc[3] = acc[3] + hxi * f[1] * w * G;
    acc[4] = acc[4] + hxi * f[0] * w * M * gamma;
  };
  auto rterm = [&](double w) {
    if (ony) {
#pragma unroll
      for (int l = 0; l < NF; ++l) dwy[l] = dwy[l] + sy * hyi * f[l] * w;
    }
    acc[0] = acc[0] + hyi * f[3] * w / rho;
    acc[1] = acc[1] + hyi * f[4] * w / rho;
    acc[2] = acc[2] + hyi * f[1] * w * M * gamma;
    acc[3] = acc[3] + hyi * f[0] * w * G;
    acc[4] = acc[4] + hyi * f[1] * w * M;
  };
  if (qreg == 2 && rreg == 2) {
    // interior (rates.f90:2089-2126)
#pragma unroll
    for (int s = 1; s <= PI_; ++s) {
      double dq[NF], dr[NF];
      const long long kqp = c + s, kqm = c - s, krp = c + s * pitch, krm = c - s * pitch;
#pragma unroll
      for (int l = 0; l < NF; ++l) {
        dq[l] = Fin[l * plane + kqp] - Fin[l * plane + kqm];
        dr[l] = Fin[l * plane + krp] - Fin[l * plane + krm];
      }
      const double DIs = D.DI[s];
      if (onx) {
#pragma unroll
        for (int l = 0; l < NF; ++l) dwx[l] = dwx[l] + sx * hxi * dq[l] * DIs;
      }
      if (ony) {
#pragma unroll
        for (int l = 0; l < NF; ++l) dwy[l] = dwy[l] + sy * hyi * dr[l] * DIs;
      }
      const double as = DIs / rho, bs = DIs * G, cs = DIs * M;
      acc[0] = acc[0] + (hxi * dq[2] + hyi * dr[3]) * as;
      acc[1] = acc[1] + (hxi * dq[3] + hyi * dr[4]) * as;
      acc[2] = acc[2] + (hxi * dq[0] + hyi * dr[1] * gamma) * cs;
      acc[3] = acc[3] + (hxi * dq[1] + hyi * dr[0]) * bs;
      acc[4] = acc[4] + (hxi * dq[0] * gamma + hyi * dr[1]) * cs;
    }
  } else if (qreg < 2 && rreg < 2) {
    // corners: one-sided in both directions, q then r for each point
#pragma unroll
    for (int s = 0; s < NBND; ++s) {
      const double wq = qreg == 0 ? D.DL[i][s] : -D.DL[nx - 1 - i][s];
      const double wr = rreg == 0 ? D.DL[j][s] : -D.DL[ny - 1 - j][s];
      at(qreg == 0 ? s : nx - 1 - s, j);
      qterm(wq);
      at(i, rreg == 0 ? s : ny - 1 - s);
      rterm(wr);
    }
  } else if (qreg < 2) {
    // L / R strips: one-sided in q, then central in r
#pragma unroll
    for (int s = 0; s < NBND; ++s) {
      at(qreg == 0 ? s : nx - 1 - s, j);
      qterm(qreg == 0 ? D.DL[i][s] : -D.DL[nx - 1 - i][s]);
    }
#pragma unroll
    for (int s = 1; s <= PI_; ++s) {
      diff(i, j + s, i, j - s);
      rterm(D.DI[s]);
    }
  } else {
    // B / T strips: central in q, then one-sided in r
#pragma unroll
    for (int s = 1; s <= PI_; ++s) {
      diff(i + s, j, i - s, j);
      qterm(D.DI[s]);
    }
#pragma unroll
    for (int s = 0; s < NBND; ++s) {
      at(i, rreg == 0 ? s : ny - 1 - s);
      rterm(rreg == 0 ? D.DL[j][s] : -D.DL[ny - 1 - j][s]);
    }
  }
  if (onx) {
#pragma unroll
    for (int l = 0; l < NF; ++l) {
      B.DWx[l * plane + c] = dwx[l];
      if (a.update) B.Wx[l * plane + c] = B.Wx[l * plane + c] + a.Bdt * dwx[l];
    }
  }
  if (ony) {
#pragma unroll
    for (int l = 0; l < NF; ++l) {
      B.DWy[l * plane + c] = dwy[l];
      if (a.update) B.Wy[l * plane + c] = B.Wy[l * plane + c] + a.Bdt * dwy[l];
    }
  }
}

// Per-block constants of the PML interior, read once per march segment
// instead of once per node.
struct PmlSeg {
  double hxi, hyi, kappa, rho, G, M, gamma;
  double DI[4], as[4], bs[4], cs[4];  // DI(s), DI(s)/rho, DI(s)*G, DI(s)*M
  bool onx, ony;
};

template <int PI_>
__device__ __forceinline__ PmlSeg pml_segment(const DevDomain& D, const DevBlock& B) {
  PmlSeg P;
  P.hxi = B.pml_h[(2 * 3 + 2) * 2];
  P.hyi = B.pml_h[(2 * 3 + 2) * 2 + 1];
  P.kappa = B.pml_kappa;
  P.rho = B.rho_b; P.G = B.G_b; P.M = B.M_b; P.gamma = B.gamma_b;
  P.onx = B.pml & 1;
  P.ony = (B.pml >> 1) & 1;
#pragma unroll
  for (int s = 1; s <= PI_; ++s) {
    P.DI[s] = D.DI[s];
    P.as[s] = P.DI[s] / P.rho;
    P.bs[s] = P.DI[s] * P.G;
    P.cs[s] = P.DI[s] * P.M;
  }
  return P;
}

// The interior branch of pml_rates (rates.f90:2089-2126) for a node whose
// neighbour values come from elsewhere (the march kernel's shared-memory
// ring): F(l, dq, dr) is field l at (i + dq, j + dr).  Same arithmetic, in the
// same order, as pml_rates for an interior node; the block constants come
// from pml_segment.
template <int PI_, typename FieldAt>
__device__ __forceinline__ void march_pml_interior(const PmlSeg& P, const DevBlock& B, long long c,
                                                   const StageArgs& a, double* acc, FieldAt F) {
  constexpr int NF = 6;
  const long long plane = B.plane;
  const double hxi = P.hxi, hyi = P.hyi;
  const double sx = B.pml_s[c], sy = B.pml_s[plane + c];
  const double rho = P.rho, G = P.G, M = P.M, gamma = P.gamma;
  const bool onx = P.onx, ony = P.ony;
  const bool load = a.scale && a.A != 0.0;
  double dwx[NF], dwy[NF];
  if (onx) {
    double w[NF];
#pragma unroll
    for (int l = 0; l < NF; ++l) {
      w[l] = B.Wx[l * plane + c];
      dwx[l] = load ? a.A * B.DWx[l * plane + c] : 0.0;
    }
    acc[0] = acc[0] - w[2] / rho;
    acc[1] = acc[1] - w[3] / rho;
    acc[2] = acc[2] - w[0] * M;
    acc[3] = acc[3] - w[1] * G;
    acc[4] = acc[4] - w[0] * gamma * M;
#pragma unroll
    for (int l = 0; l < NF; ++l) dwx[l] = dwx[l] - (sx + P.kappa) * w[l];
  }
  if (ony) {
    double w[NF];
#pragma unroll
    for (int l = 0; l < NF; ++l) {
      w[l] = B.Wy[l * plane + c];
      dwy[l] = load ? a.A * B.DWy[l * plane + c] : 0.0;
    }
    acc[0] = acc[0] - w[3] / rho;
    acc[1] = acc[1] - w[4] / rho;
    acc[2] = acc[2] - w[1] * gamma * M;
    acc[3] = acc[3] - w[0] * G;
    acc[4] = acc[4] - w[1] * M;
#pragma unroll
    for (int l = 0; l < NF; ++l) dwy[l] = dwy[l] - (sy + P.kappa) * w[l];
  }
#pragma unroll
  for (int s = 1; s <= PI_; ++s) {
    double dq[NF], dr[NF];
#pragma unroll
    for (int l = 0; l < NF; ++l) {
      dq[l] = F(l, s, 0) - F(l, -s, 0);
      dr[l] = F(l, 0, s) - F(l, 0, -s);
    }
    const double DIs = P.DI[s];
    if (onx) {
#pragma unroll
      for (int l = 0; l < NF; ++l) dwx[l] = dwx[l] + sx * hxi * dq[l] * DIs;
    }
    if (ony) {
#pragma unroll
      for (int l = 0; l < NF; ++l) dwy[l] = dwy[l] + sy * hyi * dr[l] * DIs;
    }
    const double as = P.as[s], bs = P.bs[s], cs = P.cs[s];
    acc[0] = acc[0] + (hxi * dq[2] + hyi * dr[3]) * as;
    acc[1] = acc[1] + (hxi * dq[3] + hyi * dr[4]) * as;
    acc[2] = acc[2] + (hxi * dq[0] + hyi * dr[1] * gamma) * cs;
    acc[3] = acc[3] + (hxi * dq[1] + hyi * dr[0]) * bs;
    acc[4] = acc[4] + (hxi * dq[0] * gamma + hyi * dr[1]) * cs;
  }
  if (onx) {
#pragma unroll
    for (int l = 0; l < NF; ++l) {
      B.DWx[l * plane + c] = dwx[l];
      if (a.update) B.Wx[l * plane + c] = B.Wx[l * plane + c] + a.Bdt * dwx[l];
    }
  }
  if (ony) {
#pragma unroll
    for (int l = 0; l < NF; ++l) {
      B.DWy[l * plane + c] = dwy[l];
      if (a.update) B.Wy[l * plane + c] = B.Wy[l * plane + c] + a.Bdt * dwy[l];
    }
  }
}

// Whole stage for one node of the SBP closure strips: scale, SAT (sides in the
// reference's order L, R, B, T), one-sided closure rates (rates_boundary_mode2/3),
// szz, sources, update.  Side `iside` takes the caller's hat variables.
// PLAIN: a domain without PML, dissipation, forcing, body displacement and
// peak motion; those branches are compiled out (a smaller kernel, fewer
// instruction-cache misses), the arithmetic is the same.
template <int MODE, int PI_, bool HET, bool PLAIN = false>
__device__ __forceinline__ void closure_node(const DevDomain& D, const DevBlock& B, int i, int j, const StageArgs& a,
                                             int iside, const double* Fh_given) {
  constexpr int NF = MODE == 2 ? 6 : 3;
  const int nx = B.nx, ny = B.ny;
  const long long pitch = B.pitch, plane = B.plane;
  const long long c = (long long)j * pitch + i;
  const double* __restrict__ Fin = B.F[a.in];
  const double* __restrict__ DFr = a.dfr ? B.DFalt : B.DF;
  double acc[NF];
  const bool load_df = a.scale && a.A != 0.0;
#pragma unroll
  for (int l = 0; l < NF; ++l) acc[l] = load_df ? a.A * DFr[l * plane + c] : 0.0;
  if (MODE == 2) acc[5] = 0.0;
  double Fc[NF];
#pragma unroll
  for (int l = 0; l < NF; ++l) Fc[l] = Fin[l * plane + c];
  if (i == 0) sat_term<MODE>(B.side[0], 0, j, Fc, acc, iside, Fh_given, a);
  if (i == nx - 1) sat_term<MODE>(B.side[1], 1, j, Fc, acc, iside, Fh_given, a);
  if (j == 0) sat_term<MODE>(B.side[2], 2, i, Fc, acc, iside, Fh_given, a);
  if (j == ny - 1) sat_term<MODE>(B.side[3], 3, i, Fc, acc, iside, Fh_given, a);
  NodeMat m;
  if (HET) {
    m.rho = B.rho[c]; m.G = B.G[c];
    if (MODE == 2) { m.M = B.M[c]; m.gamma = B.gamma[c]; m.nu = B.nu[c]; }
    else { m.M = 0.0; m.gamma = 0.0; m.nu = 0.0; }
  } else {
    m.rho = B.rho_b; m.G = B.G_b; m.M = B.M_b; m.gamma = B.gamma_b; m.nu = B.nu_b;
  }
  m.rinv = HET ? 1.0 / m.rho : B.rinv_b;
  bool pml = false;
  if constexpr (MODE == 2 && !PLAIN) {
    if (B.pml) { pml_rates<PI_>(D, B, Fin, i, j, a, acc); pml = true; }
  }
  if (!pml) closure_rates<MODE, PI_, PLAIN>(D, B, Fin, i, j, m, B.Ji[c], acc);
  if (MODE == 2) acc[5] = m.nu * (acc[2] + acc[4]);
  if (!PLAIN || D.src.use_gravity || D.src.use_singular)
    body_forces<MODE, PLAIN>(D, B, i, j, stage_time(a), a, acc);
  if constexpr (!PLAIN) body_extras<MODE>(B, c, Fc, acc, a);
  double* __restrict__ DFw = a.dfw ? B.DFalt : B.DF;
#pragma unroll
  for (int l = 0; l < NF; ++l) DFw[l * plane + c] = acc[l];
  if (a.update) {
    double* __restrict__ Fout = B.F[a.out];
#pragma unroll
    for (int l = 0; l < NF; ++l) Fout[l * plane + c] = Fc[l] + a.Bdt * acc[l];
  }
}

// closure strip item -> block-local node; returns the block
__device__ __forceinline__ int closure_item(const DevDomain& D, long long tid, int& i, int& j) {
  int sg = 0;
  while (tid >= D.cstart[sg + 1]) ++sg;
  const int b = sg >> 2, strip = sg & 3;
  const DevBlock& B = D.blk[b];
  const int nbst = D.nbst, nx = B.nx, ny = B.ny;
  long long k = tid - D.cstart[sg];
  if (strip == 0) { j = (int)(k / nx); i = (int)(k % nx); }                      // bottom rows
  else if (strip == 1) { j = ny - nbst + (int)(k / nx); i = (int)(k % nx); }     // top rows
  else if (strip == 2) { j = nbst + (int)(k / nbst); i = (int)(k % nbst); }       // left columns
  else { j = nbst + (int)(k / nbst); i = nx - nbst + (int)(k % nbst); }           // right columns
  return b;
}

// true if node (i, j) lies on a block side whose hat variables come from an interface
__device__ __forceinline__ bool on_interface_side(const DevBlock& B, int i, int j) {
  if (i == 0 && j >= B.side[0].cov_lo && j < B.side[0].cov_hi) return true;
  if (i == B.nx - 1 && j >= B.side[1].cov_lo && j < B.side[1].cov_hi) return true;
  if (j == 0 && i >= B.side[2].cov_lo && i < B.side[2].cov_hi) return true;
  if (j == B.ny - 1 && i >= B.side[3].cov_lo && i < B.side[3].cov_hi) return true;
  return false;
}

// Boundary kernel: every node within nbst of a block edge (the SBP closure strips).
template <int MODE, int PI_, bool HET, bool PLAIN = false>
__global__ void __maxnreg__(BOUNDARY_REGS) closure_kernel(const __grid_constant__ DevDomain D, StageArgs a) {
  const unsigned long long t_in = (threadIdx.x == 0 && D.trace.rec) ? globaltimer_ns() : 0ull;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= D.cstart[4 * D.nblocks]) return;
  int i, j;
  const int b = closure_item(D, tid, i, j);
  closure_node<MODE, PI_, HET, PLAIN>(D, D.blk[b], i, j, a, -1, nullptr);
  if (threadIdx.x == 0) trace_record(D.trace, TRACE_CLOSURE, t_in);
}

// Closure strips of a batch of independent instances in one launch.
template <int MODE, int PI_, bool HET, bool PLAIN = false>
__global__ void __maxnreg__(BOUNDARY_REGS)
    closure_kernel_batch(const DevDomain* __restrict__ doms, const int* __restrict__ cta_begin, int ninst, StageArgs a) {
  const int k = batch_instance(cta_begin, ninst, blockIdx.x);
  const DevDomain& D = doms[k];
  const long long tid = (long long)(blockIdx.x - cta_begin[k]) * blockDim.x + threadIdx.x;
  if (tid >= D.cstart[4 * D.nblocks]) return;
  int i, j;
  const int b = closure_item(D, tid, i, j);
  closure_node<MODE, PI_, HET, PLAIN>(D, D.blk[b], i, j, a, -1, nullptr);
}

template <int MODE, int PI_, bool HET>
__global__ void __launch_bounds__(TX* TY) stencil_kernel(const DevDomain* __restrict__ Dp, StageArgs a) {
  using RD = RDef<MODE>;
  constexpr int NR = RD::NR;
  constexpr int NF = MODE == 2 ? 6 : 3;
  constexpr int H = PI_;
  constexpr int WX = TX + 2 * H, WY = TY + 2 * H;
  __shared__ double sF[NR][WY][WX];
  __shared__ double s_yr[TY][WX], s_xr[TY][WX];
  __shared__ double s_yq[WY][TX], s_xq[WY][TX];
  __shared__ double s_Jr[TY][WX], s_Jq[WY][TX];  // Jacobian halos (dissipative blocks)

  const DevDomain& D = *Dp;
  int b = 0;
  while (b + 1 < D.nblocks && (int)blockIdx.x >= D.blk[b + 1].tile_begin) ++b;
  const DevBlock& B = D.blk[b];
  const int tile = blockIdx.x - B.tile_begin;
  const int i0 = (tile % B.tiles_x) * TX, j0 = (tile / B.tiles_x) * TY;
  const int nx = B.nx, ny = B.ny;
  const long long pitch = B.pitch, plane = B.plane;
  const double* __restrict__ Fin = B.F[a.in];
  const int tid = threadIdx.x;

  // cooperative tile loads (cross-shaped halo; corners loaded but unused)
  for (int idx = tid; idx < WX * WY; idx += TX * TY) {
    int ty = idx / WX, tx = idx % WX;
    int gi = i0 + tx - H, gj = j0 + ty - H;
    if (gi >= 0 && gi < nx && gj >= 0 && gj < ny) {
      long long g = (long long)gj * pitch + gi;
#pragma unroll
      for (int l = 0; l < NR; ++l) sF[l][ty][tx] = Fin[l * plane + g];
    }
  }
  for (int idx = tid; idx < WX * TY; idx += TX * TY) {
    int ty = idx / WX, tx = idx % WX;
    int gi = i0 + tx - H, gj = j0 + ty;
    if (gi >= 0 && gi < nx && gj < ny) {
      long long g = (long long)gj * pitch + gi;
      s_yr[ty][tx] = B.yr[g];
      s_xr[ty][tx] = B.xr[g];
    }
  }
  for (int idx = tid; idx < TX * WY; idx += TX * TY) {
    int ty = idx / TX, tx = idx % TX;
    int gi = i0 + tx, gj = j0 + ty - H;
    if (gi < nx && gj >= 0 && gj < ny) {
      long long g = (long long)gj * pitch + gi;
      s_yq[ty][tx] = B.yq[g];
      s_xq[ty][tx] = B.xq[g];
    }
  }
  const bool diss = B.Cdiss > 0.0;
  if (diss) {
    for (int idx = tid; idx < WX * TY; idx += TX * TY) {
      int ty = idx / WX, tx = idx % WX;
      int gi = i0 + tx - H, gj = j0 + ty;
      if (gi >= 0 && gi < nx && gj < ny) s_Jr[ty][tx] = B.J[(long long)gj * pitch + gi];
    }
    for (int idx = tid; idx < TX * WY; idx += TX * TY) {
      int ty = idx / TX, tx = idx % TX;
      int gi = i0 + tx, gj = j0 + ty - H;
      if (gi < nx && gj >= 0 && gj < ny) s_Jq[ty][tx] = B.J[(long long)gj * pitch + gi];
    }
  }
  __syncthreads();

  const int tx = tid % TX, ty = tid / TX;
  const int i = i0 + tx, j = j0 + ty;
  if (i >= nx || j >= ny) return;
  const long long c = (long long)j * pitch + i;

  if (!interior_node(D, B, i, j)) return;  // closure strips: closure_kernel
  double acc[NF];
  const bool load_df = a.scale && a.A != 0.0;
#pragma unroll
  for (int l = 0; l < NF; ++l) acc[l] = load_df ? a.A * B.DF[l * plane + c] : 0.0;
  if (MODE == 2) acc[5] = 0.0;

  double Fc[NF];
#pragma unroll
  for (int l = 0; l < NR; ++l) Fc[l] = sF[l][ty + H][tx + H];
  if (MODE == 2) Fc[5] = Fin[5 * plane + c];

  NodeMat m;
  if (HET) {
    m.rho = B.rho[c]; m.G = B.G[c];
    if (MODE == 2) { m.M = B.M[c]; m.gamma = B.gamma[c]; m.nu = B.nu[c]; }
    else { m.M = 0.0; m.gamma = 0.0; m.nu = 0.0; }
  } else {
    m.rho = B.rho_b; m.G = B.G_b; m.M = B.M_b; m.gamma = B.gamma_b; m.nu = B.nu_b;
  }
  m.rinv = HET ? 1.0 / m.rho : B.rinv_b;
  const double Ji = B.Ji[c];
  bool pml = false;
  if constexpr (MODE == 2) {
    if (B.pml) { pml_rates<PI_>(D, B, Fin, i, j, a, acc); pml = true; }
  }
  if (!pml) {
    const int cx = tx + H, cy = ty + H;
    const double yrc = s_yr[ty][cx], xrc = s_xr[ty][cx];
    const double yqc = s_yq[cy][tx], xqc = s_xq[cy][tx];
#pragma unroll
    for (int s = 1; s <= PI_; ++s) {
      const double Yrp = 0.5 * (s_yr[ty][cx + s] + yrc), Xrp = 0.5 * (s_xr[ty][cx + s] + xrc);
      const double Yrm = 0.5 * (s_yr[ty][cx - s] + yrc), Xrm = 0.5 * (s_xr[ty][cx - s] + xrc);
      const double Yqp = 0.5 * (s_yq[cy + s][tx] + yqc), Xqp = 0.5 * (s_xq[cy + s][tx] + xqc);
      const double Yqm = 0.5 * (s_yq[cy - s][tx] + yqc), Xqm = 0.5 * (s_xq[cy - s][tx] + xqc);
      const double w = HET ? D.DI[s] : 0.0;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        double sum = 0.0;
        if (RD::fa(r) >= 0) {
          const int f = RD::fa(r);
          double t = Yrp * sF[f][cy][cx + s] - Yrm * sF[f][cy][cx - s] - Yqp * sF[f][cy + s][cx] +
                     Yqm * sF[f][cy - s][cx];
          if (RD::ga(r)) t *= m.gamma;
          sum += t;
        }
        if (RD::fb(r) >= 0) {
          const int f = RD::fb(r);
          double t = -Xrp * sF[f][cy][cx + s] + Xrm * sF[f][cy][cx - s] + Xqp * sF[f][cy + s][cx] -
                     Xqm * sF[f][cy - s][cx];
          if (RD::gb(r)) t *= m.gamma;
          sum += t;
        }
        const double cf = HET ? mat_coef(m, RD::coef(r), w) : B.coef[s][RD::coef(r)];
        acc[r] += sum * cf * Ji;
      }
    }
    if (diss) {
      // artificial dissipation (rates_dissipation_interior_mode2/3, rates.f90:939-999,
      // 1397-1482): 2*AI(0)*F + sum_s AI(s)*Ji*(J F at the four neighbours at distance s)
      const double Cd = B.Cdiss;
#pragma unroll
      for (int l = 0; l < NR; ++l) {
        double sum = 2.0 * D.AI[0] * Cd * sF[l][cy][cx];
#pragma unroll
        for (int s = 1; s <= PI_; ++s)
          sum += D.AI[s] * Cd * Ji *
                 (s_Jr[ty][cx + s] * sF[l][cy][cx + s] + s_Jr[ty][cx - s] * sF[l][cy][cx - s] +
                  s_Jq[cy + s][tx] * sF[l][cy + s][cx] + s_Jq[cy - s][tx] * sF[l][cy - s][cx]);
        acc[l] += sum;
      }
    }
  }

  if (MODE == 2) acc[5] = m.nu * (acc[2] + acc[4]);
  body_forces<MODE>(D, B, i, j, stage_time(a), a, acc);
  body_extras<MODE>(B, c, Fc, acc, a);

  double* __restrict__ DF = B.DF;
#pragma unroll
  for (int l = 0; l < NF; ++l) DF[l * plane + c] = acc[l];
  if (a.update) {
    double* __restrict__ Fout = B.F[a.out];
#pragma unroll
    for (int l = 0; l < NF; ++l) Fout[l * plane + c] = Fc[l] + a.Bdt * acc[l];
  }
}

}  // namespace fdmap
