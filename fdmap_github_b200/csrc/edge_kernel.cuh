// Interface kernel: one thread per interface node.
//
// Replaces, for one RK stage, prepare_edges (domain.f90:420-439; the edge rows
// are read straight from the block's field array -- on one GPU the MPI edge
// exchange of domain.f90:1179-1212 becomes a neighbour read), the outer
// boundary conditions (boundaries.f90:74-377), the locked / frictional
// interface solves (interfaces.f90:520-1012) and, per fault node, the whole
// low-storage life cycle of the fault registers inside that stage:
//   scale_rates_friction (friction.f90:555-573)
//   -> solve_friction (friction.f90:593-828, bracketed Newton 909-1038)
//   -> set_rates_friction (friction.f90:1101-1124)
//   -> update_fields_friction (friction.f90:576-590).
// These four are fused because each touches only its own node's registers
// and nothing else reads those registers in between.
#pragma once

#include "device_common.cuh"

namespace fdmap {

enum { ST_D = FDMAP_FAULT_D, ST_PSI = FDMAP_FAULT_PSI, ST_DPSI = FDMAP_FAULT_DPSI, ST_TRUP = FDMAP_FAULT_TRUP,
       ST_V = FDMAP_FAULT_V, ST_O = FDMAP_FAULT_O, ST_S = FDMAP_FAULT_S, ST_N = FDMAP_FAULT_N,
       ST_S0 = FDMAP_FAULT_S0, ST_N0 = FDMAP_FAULT_N0, ST_DS = FDMAP_FAULT_DS, ST_DN = FDMAP_FAULT_DN,
       ST_DDS = FDMAP_FAULT_DDS, ST_DDN = FDMAP_FAULT_DDN, ST_W = FDMAP_FAULT_W, ST_DW = FDMAP_FAULT_DW,
       ST_NREG = FDMAP_FAULT_NREG, ST_DNREG = FDMAP_FAULT_DNREG };

constexpr double kShapeTol = 100.0 * 2.220446049250313e-16;

__device__ __forceinline__ double d_boxcar(double r, double w, double fin, double fout) {
  if (-w + kShapeTol < r && r < w - kShapeTol) return fin;
  if (fabs(-w - r) <= kShapeTol || fabs(r - w) <= kShapeTol) return 0.5 * (fin + fout);
  return fout;
}

// load_stress default branch + load_ramp (friction.f90:1317-1374, 1455-1484)
static __device__ void d_load_stress(const DevFriction& FR, int n, int k, double x, double y, double t, double& S0,
                              double& N0) {
  double xx = x * FR.cos_angle + y * FR.sin_angle;
  double r = fabs((xx - FR.ld_x0) / FR.ld_R);
  S0 = FR.has_bsS0 ? FR.par[PAR_BSS0 * n + k] : 0.0;
  N0 = FR.has_bsN0 ? FR.par[PAR_BSN0 * n + k] : 0.0;
  double A = 0.0;
  switch (FR.ld_shape) {
    case FDMAP_LD_UNIFORM: A = 1.0; break;
    case FDMAP_LD_LINEAR: A = (xx - FR.ld_x0) / FR.ld_R; break;
    case FDMAP_LD_BOXCAR: A = d_boxcar(r, 1.0, 1.0, 0.0); break;
    case FDMAP_LD_SMOOTH_BOXCAR: {
      double f;
      if (r <= 1.0) f = 1.0;
      else if (r < 1.1) f = 0.5 * (1.0 + tanh(0.1 / (r - 1.0 - 0.1) + 0.1 / (r - 1.0)));
      else f = 0.0;
      A = f;
      break;
    }
    case FDMAP_LD_TRIANGLE: A = (-1.0 < r && r < 1.0) ? (1.0 - r) : 0.0; break;
    case FDMAP_LD_SMOOTH: A = (r >= 1.0 - kShapeTol) ? 0.0 : exp((r * r) / ((r * r) - 1.0)); break;
    case FDMAP_LD_GAUSSIAN: A = exp(-0.5 * (r * r)); break;
    default: A = 0.0; break;
  }
  double B;
  if (FR.ld_T <= 0.0) B = t < 0.0 ? 0.0 : 1.0;
  else B = t < 0.0 ? 0.0 : 1.0 - exp(-t / FR.ld_T);
  S0 = S0 + FR.ld_S * A * B;
  N0 = N0 + FR.ld_N * A * B;
}

__device__ __forceinline__ double d_arcsinh(double x) {
  double y = fabs(x);
  return fsign(log(y + sqrt(y * y + 1.0)), x);
}

struct DRS { double a, b, V0, f0, L, fw, Vw; };

__device__ __forceinline__ void d_strength(int law, const DRS& rs, double V, double Psi, double N, double& S,
                                           double& dSdV) {
  if (law == FDMAP_FR_SL || law == FDMAP_FR_FL) {
    if (V == 0.0) { S = 0.0; dSdV = 1e10; }
    else {
      double absV = fabs(V);
      double f = rs.a * log(absV / rs.V0) + Psi;
      S = N * fsign(f, V);
      dSdV = N * rs.a / absV;
    }
  } else {
    double O = 0.5 / rs.V0 * exp(Psi / rs.a);
    S = rs.a * N * d_arcsinh(O * V);
    dSdV = rs.a * N * O / sqrt(1.0 + (V * O) * (V * O));
  }
}

// newton_solver (friction.f90:909-1038): bracketed Newton with log-bisection.
// Returns true on failure (imax iterations without meeting atolR).  imax is
// the reference's 99 (friction.f90:924) unless the host lowered it.
static __device__ bool d_newton(int law, const DRS& rs, double& V, double& S, double Slock, double N, double eta, double Psi,
                                int imax = 99) {
  const double atolR = 2.220446049250313e-16 * 1e4;
  double Vmin = fmin(0.0, Slock / eta);
  double Vmax = fmax(0.0, Slock / eta);
  // estimate_V (friction.f90:1077-1098)
  double SaN = Slock / (rs.a * N);
  if (!(fabs(SaN) > 10.0)) {
    if (law == FDMAP_FR_SL || law == FDMAP_FR_FL) V = fsign(rs.V0 * exp(-Psi / rs.a) * exp(fabs(SaN)), SaN);
    else if (law != FDMAP_FR_RSF) V = 2.0 * rs.V0 * exp(-Psi / rs.a) * sinh(SaN);
  }
  if (V <= Vmin || Vmax <= V) V = 0.5 * (Vmin + Vmax);
  int i;
  for (i = 1; i <= imax; ++i) {
    S = Slock - eta * V;
    double Sf, dSfdV;
    d_strength(law, rs, V, Psi, N, Sf, dSfdV);
    double R = -S + Sf;
    if (R > 0.0) Vmax = V;
    if (R < 0.0) Vmin = V;
    double dRdV = eta + dSfdV;
    double dV = -R / dRdV;
    if (fabs(R) <= atolR) break;
    if (i == imax) break;
    V = V + dV;
    if (V <= Vmin || Vmax <= V) {
      if (Vmin == 0.0) V = 0.1 * Vmax;
      else if (Vmax == 0.0) V = 0.1 * Vmin;
      else V = fsign(sqrt(Vmin * Vmax), Slock);
      dV = Vmax - Vmin;
    }
    if (fabs(dV) <= 0.0) break;
  }
  return i == imax;
}

__device__ __forceinline__ double pow8(double x) {
  double x2 = x * x, x4 = x2 * x2;
  return x4 * x4;
}

// state_rate (friction.f90:1147-1264)
static __device__ double d_state_rate(int law, const DRS& rs, double V, double Psi) {
  if (law == FDMAP_FR_FRICTIONLESS || law == FDMAP_FR_SW || law == FDMAP_FR_LOCKED) return 0.0;
  if (V == 0.0) return 0.0;
  double absV = fabs(V);
  double frs, fss, fLV;
  switch (law) {
    case FDMAP_FR_SL:
      frs = rs.a * log(absV / rs.V0) + Psi;
      fss = rs.f0 - (rs.b - rs.a) * log(absV / rs.V0);
      return -(absV / rs.L) * (frs - fss);
    case FDMAP_FR_FL:
      frs = rs.a * log(absV / rs.V0) + Psi;
      fLV = rs.f0 - (rs.b - rs.a) * log(absV / rs.V0);
      fss = rs.fw + (fLV - rs.fw) / pow(1.0 + pow8(V / rs.Vw), 0.125);
      return -(absV / rs.L) * (frs - fss);
    case FDMAP_FR_RSL:
      fss = rs.f0 - (rs.b - rs.a) * log(absV / rs.V0);
      frs = rs.a * d_arcsinh(0.5 * absV / rs.V0 * exp(Psi / rs.a));
      return -(absV / rs.L) * (frs - fss);
    case FDMAP_FR_RFL:
      fLV = rs.f0 - (rs.b - rs.a) * log(absV / rs.V0);
      fss = rs.fw + (fLV - rs.fw) / pow(1.0 + pow8(V / rs.Vw), 0.125);
      frs = rs.a * d_arcsinh(0.5 * absV / rs.V0 * exp(Psi / rs.a));
      return (absV / rs.L) * (fss - frs);
    case FDMAP_FR_RSF: {
      fLV = rs.f0 - (rs.b - rs.a) * log(absV / rs.V0);
      fss = rs.fw + (fLV - rs.fw) / pow(1.0 + pow8(V / rs.Vw), 0.125);
      double Psiss = rs.a * log(2.0 * rs.V0 / absV * sinh(fss / rs.a));
      return (absV / rs.L) * (Psiss - Psi);
    }
    case FDMAP_FR_RAL:
      return (rs.b * rs.V0 / rs.L) * (exp((rs.f0 - Psi) / rs.b) - absV / rs.V0);
  }
  return 0.0;
}

// solve_friction (friction.f90:593-828) for node k; the state is read from and
// written to registers passed by reference (loaded from HBM by the caller).
struct NodeState {
  double V, O, S, N, S0, N0, Nreg, D, Psi;
};

static __device__ void d_solve_friction(const DevFriction& FR, int n, int k, NodeState& st, double S0, double N0, double phip,
                                 double phis, double eta, double x, double y, double t, double dt,
                                 unsigned long long* status, int imax) {
  d_load_stress(FR, n, k, x, y, t, st.S0, st.N0);
  st.S0 = st.S0 + S0;
  st.N0 = st.N0 + N0;
  double Slock = st.S0 + phis;
  double Nlock = st.N0 - (1.0 - FR.skempton) * phip;
  st.O = 0.0;
  st.N = Nlock;
  if (Nlock <= 0.0) {
    st.S = 0.0;
    st.V = Slock / eta;
    return;
  }
  if (dt == 0.0) st.Nreg = st.N;
  if (!FR.reg) st.Nreg = st.N;
  double xx = x * FR.cos_angle + y * FR.sin_angle;
  if (xx < FR.xlockm || xx > FR.xlockp) {
    st.S = FR.flock * st.Nreg;
    if (fabs(Slock) >= st.S) { st.S = fsign(st.S, Slock); st.V = (Slock - st.S) / eta; }
    else { st.V = 0.0; st.S = Slock; }
    return;
  }
  if (FR.law == FDMAP_FR_FRICTIONLESS) { st.S = 0.0; st.V = Slock / eta; return; }
  if (FR.law == FDMAP_FR_LOCKED) { st.V = 0.0; st.S = Slock; return; }
  double Sk = 0.0;
  if (FR.force) {
    double xm = FR.kn_xL + FR.kn_vL * fmin(t, FR.kn_tmax);
    double fkm = (xx < xm) ? FR.kn_fd + FR.kn_dfdx * (xm - xx) : FR.kn_fd;
    double xp = FR.kn_xR + FR.kn_vR * fmin(t, FR.kn_tmax);
    double fkp = (xx > xp) ? FR.kn_fd + FR.kn_dfdx * (xx - xp) : FR.kn_fd;
    Sk = FR.kn_c0 + st.Nreg * fmax(fkm, fkp);
  }
  if (FR.law == FDMAP_FR_SW) {
    double c0 = FR.par[PAR_C0 * n + k], fs = FR.par[PAR_FS * n + k];
    double fd = FR.par[PAR_FD * n + k], Dc = FR.par[PAR_DC * n + k];
    double S = c0 + fmax(st.Nreg, 0.0) * ((fs - (fs - fd) * fmin(st.D, Dc) / Dc));
    if (FR.force) S = fmin(S, Sk);
    if (fabs(Slock) >= S) { st.S = fsign(S, Slock); st.V = (Slock - st.S) / eta; }
    else { st.V = 0.0; st.S = Slock; }
    return;
  }
  DRS rs{FR.par[PAR_A * n + k], FR.par[PAR_B * n + k], FR.par[PAR_V0 * n + k], FR.par[PAR_F0 * n + k],
         FR.par[PAR_L * n + k], FR.par[PAR_FW * n + k], FR.par[PAR_VW * n + k]};
  if (d_newton(FR.law, rs, st.V, st.S, Slock, st.Nreg, eta, st.Psi, imax)) {
    // the reference warns and retries from the failed iterate V, S
    // (friction.f90:789-790); a second failure is where it stops (friction.f90:1014)
    atomicAdd(&status[0], 1ull);
    if (d_newton(FR.law, rs, st.V, st.S, Slock, st.Nreg, eta, st.Psi, imax)) atomicAdd(&status[3], 1ull);
  }
  if (FR.force) {
    if (Sk < fabs(st.S)) { st.S = fsign(Sk, Slock); st.V = (Slock - st.S) / eta; }
  }
}

// ---------------------------------------------------------------------------
// outer boundary (set_bc_mode2/3, boundaries.f90:155-377)
// ---------------------------------------------------------------------------
template <int MODE>
__device__ void d_set_bc(double* Fh, const double* F, const double* F0, double n0, double n1, int bc, double Zs,
                         double Zp, double gamma) {
  if (MODE == 3) {
    if (Zs == 0.0) { for (int l = 0; l < 3; ++l) Fh[l] = F[l]; return; }
    double Zsi = 1.0 / Zs;
    double d[3] = {F[0] - F0[0], F[1] - F0[1], F[2] - F0[2]};
    double r[3];
    rot3_xy2nt(d, n0, n1, r);
    double vz, snz;
    if (bc == FDMAP_BC_ABSORBING) { vz = 0.5 * (r[0] - Zsi * r[2]); snz = 0.5 * (r[2] - Zs * r[0]); }
    else if (bc == FDMAP_BC_FREE) { vz = r[0] - Zsi * r[2]; snz = 0.0; }
    else { vz = 0.0; snz = r[2] - Zs * r[0]; }
    rot3_nt2xy(Fh, n0, n1, vz, r[1], snz);
    for (int l = 0; l < 3; ++l) Fh[l] = Fh[l] + F0[l];
  } else {
    double Zsi = (Zs == 0.0) ? 0.0 : 1.0 / Zs;
    double Zpi = 1.0 / Zp;
    bool zero_variant = (bc == FDMAP_BC_ABSORBING_0 || bc == FDMAP_BC_FREE_0 || bc == FDMAP_BC_RIGID_0);
    double d[6], r[6];
    for (int l = 0; l < 6; ++l) d[l] = zero_variant ? F[l] : F[l] - F0[l];
    rot2_xy2nt(d, n0, n1, r);
    double vtFD = r[0], vnFD = r[1], sntFD = r[3], snnFD = r[4];
    double vt, vn, snt, snn;
    switch (bc) {
      case FDMAP_BC_ABSORBING:
      case FDMAP_BC_ABSORBING_0:
        vt = 0.5 * (vtFD - Zsi * sntFD); snt = 0.5 * (sntFD - Zs * vtFD);
        vn = 0.5 * (vnFD - Zpi * snnFD); snn = 0.5 * (snnFD - Zp * vnFD);
        break;
      case FDMAP_BC_FREE:
      case FDMAP_BC_FREE_0:
        vt = vtFD - Zsi * sntFD; snt = 0.0; vn = vnFD - Zpi * snnFD; snn = 0.0;
        break;
      case FDMAP_BC_RIGID:
      case FDMAP_BC_RIGID_0:
        vt = 0.0; snt = sntFD - Zs * vtFD; vn = 0.0; snn = snnFD - Zp * vnFD;
        break;
      case FDMAP_BC_ABSORBING_VELOCITY:
        vt = -Zsi * sntFD; snt = sntFD; vn = -Zpi * snnFD; snn = snnFD;
        break;
      default:  // FDMAP_BC_FREE_VELOCITY
        vt = vtFD - Zsi * sntFD; snt = sntFD; vn = vnFD - Zpi * snnFD; snn = snnFD;
        break;
    }
    double stt = r[2] - gamma * (snnFD - snn);
    double szz = r[5] - gamma * (snnFD - snn);
    rot2_nt2xy(Fh, n0, n1, vt, vn, stt, snt, snn, szz);
    if (!zero_variant)
      for (int l = 0; l < 6; ++l) Fh[l] = Fh[l] + F0[l];
  }
}

__device__ __forceinline__ void side_node_local(int s, int k, int nx, int ny, int& i, int& j) {
  if (s == 0) { i = 0; j = k; }
  else if (s == 1) { i = nx - 1; j = k; }
  else if (s == 2) { i = k; j = 0; }
  else { i = k; j = ny - 1; }
}

// ---------------------------------------------------------------------------
// interface node (interfaces.f90:676-1012 + friction register life cycle)
// ---------------------------------------------------------------------------
template <int MODE>
__device__ void d_iface_node(const DevDomain& D, const DevIface& I, int k, const StageArgs& a, double* Fhm_out = nullptr,
                             double* Fhp_out = nullptr) {
  constexpr int NF = MODE == 2 ? 6 : 3;
  const DevBlock& Bm = D.blk[I.im];
  const DevBlock& Bp = D.blk[I.ip];
  const DevSide& Sm = Bm.side[I.direction == 0 ? 1 : 3];
  const DevSide& Sp = Bp.side[I.direction == 0 ? 0 : 2];
  int km = I.offm + k, kp = I.offp + k;
  int im_, jm_, ip_, jp_;
  side_node_local(I.direction == 0 ? 1 : 3, km, Bm.nx, Bm.ny, im_, jm_);
  side_node_local(I.direction == 0 ? 0 : 2, kp, Bp.nx, Bp.ny, ip_, jp_);
  double Fm[6], Fp[6], F0m[6], F0p[6];
  // edge values: the block's own row, or (partitioned domain) the values
  // the peer GPU sent for this stage
  if (I.rem_m) {
#pragma unroll
    for (int l = 0; l < NF; ++l) Fm[l] = I.rem_m[l * I.n + k];
  } else {
    const double* fm = Bm.F[a.in] + (long long)jm_ * Bm.pitch + im_;
#pragma unroll
    for (int l = 0; l < NF; ++l) Fm[l] = fm[l * Bm.plane];
  }
  if (I.rem_p) {
#pragma unroll
    for (int l = 0; l < NF; ++l) Fp[l] = I.rem_p[l * I.n + k];
  } else {
    const double* fp = Bp.F[a.in] + (long long)jp_ * Bp.pitch + ip_;
#pragma unroll
    for (int l = 0; l < NF; ++l) Fp[l] = fp[l * Bp.plane];
  }
#pragma unroll
  for (int l = 0; l < NF; ++l) {
    F0m[l] = Sm.F0[km + Sm.n * l];
    F0p[l] = Sp.F0[kp + Sp.n * l];
  }
  double n0 = I.nhat[k], n1 = I.nhat[k + I.n];
  double Fhm[6], Fhp[6];
  if (I.coupling == FDMAP_COUPLING_LOCKED) {
    if (MODE == 2) {
      double gm = Sm.M[km + 2 * Sm.n], gp = Sp.M[kp + 2 * Sp.n];
      double rp[6], rm[6];
      rot2_xy2nt(Fp, n0, n1, rp);
      rot2_xy2nt(Fm, n0, n1, rm);
      const double Zsip = I.icoef[IC_ZSIP * I.n + k], Zsim = I.icoef[IC_ZSIM * I.n + k];
      const double Zpip = I.icoef[IC_ZPIP * I.n + k], Zpim = I.icoef[IC_ZPIM * I.n + k];
      double etap = I.icoef[IC_ETAP * I.n + k];
      double phip = etap * (rp[4] * Zpip + rm[4] * Zpim + rp[1] - rm[1]);
      double vnp = rp[1] + Zpip * (rp[4] - phip);
      double vnm = rm[1] - Zpim * (rm[4] - phip);
      double sttp = rp[2] - gp * (rp[4] - phip), sttm = rm[2] - gm * (rm[4] - phip);
      double szzp = rp[5] - gp * (rp[4] - phip), szzm = rm[5] - gm * (rm[4] - phip);
      double etas = I.icoef[IC_ETAS * I.n + k];
      double phis = etas * (rp[3] * Zsip + rm[3] * Zsim + rp[0] - rm[0]);
      double vtp = rp[0] + Zsip * (rp[3] - phis);
      double vtm = rm[0] - Zsim * (rm[3] - phis);
      rot2_nt2xy(Fhp, n0, n1, vtp, vnp, sttp, phis, phip, szzp);
      rot2_nt2xy(Fhm, n0, n1, vtm, vnm, sttm, phis, phip, szzm);
    } else {
      double rp[3], rm[3];
      rot3_xy2nt(Fp, n0, n1, rp);
      rot3_xy2nt(Fm, n0, n1, rm);
      const double Zsip = I.icoef[IC_ZSIP * I.n + k], Zsim = I.icoef[IC_ZSIM * I.n + k];
      double etas = I.icoef[IC_ETAS * I.n + k];
      double phis = etas * (rp[2] * Zsip + rm[2] * Zsim + rp[0] - rm[0]);
      double vzp = rp[0] + Zsip * (rp[2] - phis);
      double vzm = rm[0] - Zsim * (rm[2] - phis);
      rot3_nt2xy(Fhp, n0, n1, vzp, rp[1], phis);
      rot3_nt2xy(Fhm, n0, n1, vzm, rm[1], phis);
    }
  } else {
    const DevFriction& FR = I.fr;
    const int n = I.n;
    double* st = FR.st;
    // scale_rates_friction: registers times A at the start of the stage
    double DDs = st[ST_DDS * n + k], DDn = st[ST_DDN * n + k], DPsi = st[ST_DPSI * n + k];
    double DW = st[ST_DW * n + k], DNreg = st[ST_DNREG * n + k];
    if (a.scale) { DDs = a.A * DDs; DDn = a.A * DDn; DPsi = a.A * DPsi; DW = a.A * DW; DNreg = a.A * DNreg; }
    NodeState ns;
    ns.V = st[ST_V * n + k]; ns.O = st[ST_O * n + k]; ns.S = st[ST_S * n + k]; ns.N = st[ST_N * n + k];
    ns.S0 = st[ST_S0 * n + k]; ns.N0 = st[ST_N0 * n + k]; ns.Nreg = st[ST_NREG * n + k];
    ns.D = st[ST_D * n + k]; ns.Psi = st[ST_PSI * n + k];
    double x = I.x[k], y = I.y[k];
    double p = 0.0;
    if (FR.tp_use) p = p + FR.tp_p0;
    if (MODE == 2) {
      // interfaces.f90:795 hands (F0m, F0p) to dummies declared (F0p, F0m)
      const double* dF0p = F0m;
      const double* dF0m = F0p;
      double gm = Sm.M[km + 2 * Sm.n], gp = Sp.M[kp + 2 * Sp.n];
      double r0p[6];
      rot2_xy2nt(dF0p, n0, n1, r0p);
      double dp[6], dm[6], rp[6], rm[6];
      for (int l = 0; l < 6; ++l) { dp[l] = Fp[l] - dF0p[l]; dm[l] = Fm[l] - dF0m[l]; }
      rot2_xy2nt(dp, n0, n1, rp);
      rot2_xy2nt(dm, n0, n1, rm);
      const double Zsip = I.icoef[IC_ZSIP * I.n + k], Zsim = I.icoef[IC_ZSIM * I.n + k];
      const double Zpip = I.icoef[IC_ZPIP * I.n + k], Zpim = I.icoef[IC_ZPIM * I.n + k];
      double etas = I.icoef[IC_ETAS * I.n + k];
      double phis = etas * (rp[3] * Zsip + rm[3] * Zsim + rp[0] - rm[0]);
      double etap = I.icoef[IC_ETAP * I.n + k];
      double phip = etap * (rp[4] * Zpip + rm[4] * Zpim + rp[1] - rm[1]);
      double S0 = r0p[3];
      double N0 = -r0p[4] - p;
      d_solve_friction(FR, n, k, ns, S0, N0, phip, phis, etas, x, y, stage_time(a), a.Bdt, D.status, D.newton_imax);
      double snn = -(ns.N - ns.N0) / (1.0 - FR.skempton);
      double vnp = rp[1] + Zpip * (rp[4] - snn);
      double vnm = rm[1] - Zpim * (rm[4] - snn);
      double sttp = rp[2] - gp * (rp[4] - snn), sttm = rm[2] - gm * (rm[4] - snn);
      double szzp = rp[5] - gp * (rp[4] - snn), szzm = rm[5] - gm * (rm[4] - snn);
      double snt = ns.S - ns.S0;
      double vtp = rp[0] + Zsip * (rp[3] - snt);
      double vtm = rm[0] - Zsim * (rm[3] - snt);
      rot2_nt2xy(Fhp, n0, n1, vtp, vnp, sttp, snt, snn, szzp);
      rot2_nt2xy(Fhm, n0, n1, vtm, vnm, sttm, snt, snn, szzm);
      for (int l = 0; l < 6; ++l) { Fhp[l] = Fhp[l] + dF0p[l]; Fhm[l] = Fhm[l] + dF0m[l]; }
    } else {
      double r0p[3];
      rot3_xy2nt(F0p, n0, n1, r0p);
      double dp[3] = {Fp[0] - F0p[0], Fp[1] - F0p[1], Fp[2] - F0p[2]};
      double dm[3] = {Fm[0] - F0m[0], Fm[1] - F0m[1], Fm[2] - F0m[2]};
      double rp[3], rm[3];
      rot3_xy2nt(dp, n0, n1, rp);
      rot3_xy2nt(dm, n0, n1, rm);
      const double Zsip = I.icoef[IC_ZSIP * I.n + k], Zsim = I.icoef[IC_ZSIM * I.n + k];
      double etas = I.icoef[IC_ETAS * I.n + k];
      double phis = etas * (rp[2] * Zsip + rm[2] * Zsim + rp[0] - rm[0]);
      double S0 = r0p[2];
      double stt, snt, snn;
      xy2nt_mat(Bp.F0v[3], Bp.F0v[4], Bp.F0v[6], stt, snt, snn, n0, n1);
      double N0 = -snn - p;
      d_solve_friction(FR, n, k, ns, S0, N0, 0.0, phis, etas, x, y, stage_time(a), a.Bdt, D.status, D.newton_imax);
      double snz = ns.S - ns.S0;
      double vzp = rp[0] + Zsip * (rp[2] - snz);
      double vzm = rm[0] - Zsim * (rm[2] - snz);
      rot3_nt2xy(Fhp, n0, n1, vzp, rp[1], snz);
      rot3_nt2xy(Fhm, n0, n1, vzm, rm[1], snz);
      for (int l = 0; l < 3; ++l) { Fhp[l] = Fhp[l] + F0p[l]; Fhm[l] = Fhm[l] + F0m[l]; }
    }
    // set_rates_friction + rupture_front (friction.f90:1101-1124, 1267-1290)
    DRS rs{};
    if (FR.law >= FDMAP_FR_SL)
      rs = DRS{FR.par[PAR_A * n + k], FR.par[PAR_B * n + k], FR.par[PAR_V0 * n + k], FR.par[PAR_F0 * n + k],
               FR.par[PAR_L * n + k], FR.par[PAR_FW * n + k], FR.par[PAR_VW * n + k]};
    DDs = DDs + ns.V;
    DDn = DDn + ns.O;
    DPsi = DPsi + d_state_rate(FR.law, rs, ns.V, ns.Psi);
    if (FR.reg) DNreg = DNreg + (-(fabs(ns.V) / FR.par[PAR_L * n + k]) * (ns.Nreg - fmax(ns.N, 0.0)));
    DW = DW + ns.S * ns.V;
    double trup = st[ST_TRUP * n + k];
    bool rup = FR.rup_field == 1 ? (ns.D > FR.rup_threshold) : (fabs(ns.V) > FR.rup_threshold);
    if (rup) trup = fmin(trup, stage_time(a));
    st[ST_TRUP * n + k] = trup;
    st[ST_V * n + k] = ns.V; st[ST_O * n + k] = ns.O; st[ST_S * n + k] = ns.S; st[ST_N * n + k] = ns.N;
    st[ST_S0 * n + k] = ns.S0; st[ST_N0 * n + k] = ns.N0;
    if (a.tap && FR.st_out) {
      // the fields as write_output sees them in stage 1: solved and rates set, not yet updated
      double* so = FR.st_out;
      so[ST_D * n + k] = ns.D; so[ST_PSI * n + k] = ns.Psi; so[ST_DPSI * n + k] = DPsi; so[ST_TRUP * n + k] = trup;
      so[ST_V * n + k] = ns.V; so[ST_O * n + k] = ns.O; so[ST_S * n + k] = ns.S; so[ST_N * n + k] = ns.N;
      so[ST_S0 * n + k] = ns.S0; so[ST_N0 * n + k] = ns.N0; so[ST_DS * n + k] = st[ST_DS * n + k];
      so[ST_DN * n + k] = st[ST_DN * n + k]; so[ST_DDS * n + k] = DDs; so[ST_DDN * n + k] = DDn;
      so[ST_W * n + k] = st[ST_W * n + k]; so[ST_DW * n + k] = DW; so[ST_NREG * n + k] = ns.Nreg;
      so[ST_DNREG * n + k] = DNreg;
    }
    double Nreg = ns.Nreg;
    if (a.update) {
      // update_fields_friction (friction.f90:576-590)
      st[ST_DS * n + k] = st[ST_DS * n + k] + a.Bdt * DDs;
      st[ST_DN * n + k] = st[ST_DN * n + k] + a.Bdt * DDn;
      st[ST_D * n + k] = ns.D + a.Bdt * fabs(DDs);
      st[ST_PSI * n + k] = ns.Psi + a.Bdt * DPsi;
      st[ST_W * n + k] = st[ST_W * n + k] + a.Bdt * DW;
      Nreg = Nreg + a.Bdt * DNreg;
    }
    st[ST_NREG * n + k] = Nreg;
    st[ST_DDS * n + k] = DDs; st[ST_DDN * n + k] = DDn; st[ST_DPSI * n + k] = DPsi;
    st[ST_DW * n + k] = DW; st[ST_DNREG * n + k] = DNreg;
  }
#pragma unroll
  for (int l = 0; l < NF; ++l) {
    Sm.Fhat[km + Sm.n * l] = Fhm[l];
    Sp.Fhat[kp + Sp.n * l] = Fhp[l];
  }
  if (Fhm_out) {
#pragma unroll
    for (int l = 0; l < NF; ++l) { Fhm_out[l] = Fhm[l]; Fhp_out[l] = Fhp[l]; }
  }
}

// Partitioned domain: the local side's edge values of every interface whose
// other side lives on another GPU, packed as [l*n + k] for the peer.
template <int MODE>
__global__ void __launch_bounds__(128) pack_edges(const __grid_constant__ DevDomain D, int in, int iface) {
  constexpr int NF = MODE == 2 ? 6 : 3;
  const DevIface& I = D.ifc[iface];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n || !I.send) return;
  const bool local_m = I.rem_p != nullptr;  // the minus side is this GPU's
  const DevBlock& B = D.blk[local_m ? I.im : I.ip];
  const int side = local_m ? (I.direction == 0 ? 1 : 3) : (I.direction == 0 ? 0 : 2);
  int i, j;
  side_node_local(side, (local_m ? I.offm : I.offp) + k, B.nx, B.ny, i, j);
  const double* f = B.F[in] + (long long)j * B.pitch + i;
#pragma unroll
  for (int l = 0; l < NF; ++l) I.send[l * I.n + k] = f[l * B.plane];
}

// One thread per interface node: the locked / frictional solve of this stage,
// hat variables of both sides, and the fault register life cycle.
template <int MODE>
__global__ void __maxnreg__(BOUNDARY_REGS) edge_kernel(const __grid_constant__ DevDomain D, StageArgs a) {
  const unsigned long long t_in = (threadIdx.x == 0 && D.trace.rec) ? globaltimer_ns() : 0ull;
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= D.seg_start[D.nseg]) return;
  int sg = 0;
  while (tid >= D.seg_start[sg + 1]) ++sg;
  d_iface_node<MODE>(D, D.ifc[D.seg_a[sg]], tid - D.seg_start[sg], a);
  if (threadIdx.x == 0) trace_record(D.trace, TRACE_EDGE, t_in);
}

// Interface nodes of a batch of independent instances in one launch.
template <int MODE>
__global__ void __maxnreg__(BOUNDARY_REGS)
    edge_kernel_batch(const DevDomain* __restrict__ doms, const int* __restrict__ cta_begin, int ninst, StageArgs a) {
  const int k = batch_instance(cta_begin, ninst, blockIdx.x);
  const DevDomain& D = doms[k];
  const int tid = (blockIdx.x - cta_begin[k]) * blockDim.x + threadIdx.x;
  if (tid >= D.seg_start[D.nseg]) return;
  int sg = 0;
  while (tid >= D.seg_start[sg + 1]) ++sg;
  d_iface_node<MODE>(D, D.ifc[D.seg_a[sg]], tid - D.seg_start[sg], a);
}

}  // namespace fdmap
