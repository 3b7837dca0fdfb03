// Discrete adjoint of the mode III block coupling: every block's SBP-SAT
// stage (adj_node_part on any block) and the interface solve of each fault
// node (interfaces.f90:676-1012, friction.f90:593-828, 909-1038, 1147-1264),
// locked or frictional with a smooth rate-and-state law.
//
// Per forward stage s an interface node maps
//   x = (u-[3], u+[3], Psi, S0, rho-, G-, rho+, G+)
// to its SAT rates and its state rate
//   y = (Ks- (Fh- - u-), Ks+ (Fh+ - u+), dPsi/dt),
// where Fh are the hat variables of the solve (slip velocity V from the
// bracketed Newton iteration) and S0 is the node's total shear load (the
// background shear stress plus the load shape plus the traction of the side
// prestress).  The stage adjoint needs ybar . dy/dx.  It is formed in forward
// mode: one evaluation of the node's map on dual numbers per input, with V
// carried through one Newton step from the converged root V*,
//   V = V* - R(V*, x) / R_V(V*, x),
// whose tangent is the implicit derivative -R_x / R_V of the friction
// equation R(V, x) = Sf(V, Psi) - (S0 + phi - eta V) = 0 (R(V*) = 0 to the
// solver's tolerance).  The state variable has its own low-storage RK adjoint:
//   qs_Psi = qbar'_Psi + B dt Psibar,  Psibar += dy/dPsi^T (qs, qs_Psi),
//   qbar'_Psi = A qs_Psi.
#pragma once

#include "adjoint_kernel.cuh"
#include "edge_kernel.cuh"

namespace fdmap {

// value and one tangent
struct Dn {
  double v, d;
};
__device__ __forceinline__ Dn dn(double v) { return Dn{v, 0.0}; }
__device__ __forceinline__ Dn operator+(Dn a, Dn b) { return Dn{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dn operator-(Dn a, Dn b) { return Dn{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dn operator-(Dn a) { return Dn{-a.v, -a.d}; }
__device__ __forceinline__ Dn operator*(Dn a, Dn b) { return Dn{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dn operator/(Dn a, Dn b) { return Dn{a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
__device__ __forceinline__ Dn operator+(Dn a, double b) { return Dn{a.v + b, a.d}; }
__device__ __forceinline__ Dn operator+(double a, Dn b) { return Dn{a + b.v, b.d}; }
__device__ __forceinline__ Dn operator-(Dn a, double b) { return Dn{a.v - b, a.d}; }
__device__ __forceinline__ Dn operator-(double a, Dn b) { return Dn{a - b.v, -b.d}; }
__device__ __forceinline__ Dn operator*(Dn a, double b) { return Dn{a.v * b, a.d * b}; }
__device__ __forceinline__ Dn operator*(double a, Dn b) { return Dn{a * b.v, a * b.d}; }
__device__ __forceinline__ Dn operator/(Dn a, double b) { return Dn{a.v / b, a.d / b}; }
__device__ __forceinline__ Dn operator/(double a, Dn b) { return Dn{a / b.v, -a * b.d / (b.v * b.v)}; }
__device__ __forceinline__ Dn dsqrt(Dn a) {
  const double s = sqrt(a.v);
  return Dn{s, 0.5 * a.d / s};
}
__device__ __forceinline__ Dn dexp(Dn a) {
  const double e = exp(a.v);
  return Dn{e, e * a.d};
}
__device__ __forceinline__ Dn dlog(Dn a) { return Dn{log(a.v), a.d / a.v}; }
__device__ __forceinline__ Dn dsinh(Dn a) { return Dn{sinh(a.v), cosh(a.v) * a.d}; }
__device__ __forceinline__ Dn dfabs(Dn a) { return a.v < 0.0 ? -a : a; }
// |a| with the sign of b (Fortran SIGN)
__device__ __forceinline__ Dn dsign(Dn a, Dn b) {
  const Dn m = dfabs(a);
  return signbit(b.v) ? -m : m;
}
__device__ __forceinline__ Dn dasinh(Dn a) { return Dn{d_arcsinh(a.v), a.d / sqrt(1.0 + a.v * a.v)}; }
__device__ __forceinline__ Dn dpow(Dn a, double p) {
  const double v = pow(a.v, p);
  return Dn{v, p * v / a.v * a.d};
}
__device__ __forceinline__ Dn dpow8(Dn a) {
  const Dn a2 = a * a, a4 = a2 * a2;
  return a4 * a4;
}

// d_strength on dual numbers: strength and its V derivative
__device__ __forceinline__ void dn_strength(int law, const DRS& rs, Dn V, Dn Psi, Dn N, Dn& S, Dn& dSdV) {
  if (law == FDMAP_FR_SL || law == FDMAP_FR_FL) {
    if (V.v == 0.0) {
      S = dn(0.0);
      dSdV = dn(1e10);
    } else {
      const Dn absV = dfabs(V);
      const Dn f = rs.a * dlog(absV / rs.V0) + Psi;
      S = N * dsign(f, V);
      dSdV = N * rs.a / absV;
    }
  } else {
    const Dn O = (0.5 / rs.V0) * dexp(Psi / rs.a);
    S = rs.a * N * dasinh(O * V);
    const Dn VO = V * O;
    dSdV = rs.a * N * O / dsqrt(1.0 + VO * VO);
  }
}

// d_state_rate on dual numbers
__device__ __forceinline__ Dn dn_state_rate(int law, const DRS& rs, Dn V, Dn Psi) {
  if (law == FDMAP_FR_FRICTIONLESS || law == FDMAP_FR_SW || law == FDMAP_FR_LOCKED) return dn(0.0);
  if (V.v == 0.0) return dn(0.0);
  const Dn absV = dfabs(V);
  const Dn lv = dlog(absV / rs.V0);
  switch (law) {
    case FDMAP_FR_SL: {
      const Dn frs = rs.a * lv + Psi, fss = rs.f0 - (rs.b - rs.a) * lv;
      return -(absV / rs.L) * (frs - fss);
    }
    case FDMAP_FR_FL: {
      const Dn frs = rs.a * lv + Psi, fLV = rs.f0 - (rs.b - rs.a) * lv;
      const Dn fss = rs.fw + (fLV - rs.fw) / dpow(1.0 + dpow8(V / rs.Vw), 0.125);
      return -(absV / rs.L) * (frs - fss);
    }
    case FDMAP_FR_RSL: {
      const Dn fss = rs.f0 - (rs.b - rs.a) * lv;
      const Dn frs = rs.a * dasinh((0.5 / rs.V0) * absV * dexp(Psi / rs.a));
      return -(absV / rs.L) * (frs - fss);
    }
    case FDMAP_FR_RFL: {
      const Dn fLV = rs.f0 - (rs.b - rs.a) * lv;
      const Dn fss = rs.fw + (fLV - rs.fw) / dpow(1.0 + dpow8(V / rs.Vw), 0.125);
      const Dn frs = rs.a * dasinh((0.5 / rs.V0) * absV * dexp(Psi / rs.a));
      return (absV / rs.L) * (fss - frs);
    }
    case FDMAP_FR_RSF: {
      const Dn fLV = rs.f0 - (rs.b - rs.a) * lv;
      const Dn fss = rs.fw + (fLV - rs.fw) / dpow(1.0 + dpow8(V / rs.Vw), 0.125);
      const Dn Psiss = rs.a * dlog((2.0 * rs.V0) / absV * dsinh(fss / rs.a));
      return (absV / rs.L) * (Psiss - Psi);
    }
    case FDMAP_FR_RAL:
      return (rs.b * rs.V0 / rs.L) * (dexp((rs.f0 - Psi) / rs.b) - absV / rs.V0);
  }
  return dn(0.0);
}

// Fault-node inputs of the interface map (index of each in x[])
enum { FX_UM = 0, FX_UP = 3, FX_PSI = 6, FX_S0 = 7, FX_RHOM = 8, FX_GM = 9, FX_RHOP = 10, FX_GP = 11, FX_N = 12 };
// outputs: SAT rates of the - and + edge nodes, state rate
enum { FY_RM = 0, FY_RP = 3, FY_PSI = 6, FY_N = 7 };

struct FaultConst {
  double n0, n1;            // fault normal
  double F0m[3], F0p[3];    // side prestress of both edge nodes
  double N0;                // normal load (constant in mode III)
  double geom, geop;        // edge geometry factors H00i |grad| / J of both edge nodes
  double xx;                // along-strike coordinate for the lock window
  bool friction;
};

// The interface map of one fault node on dual numbers.  With `solve` the
// Newton root is found first (d_newton from the values) and returned in V0;
// otherwise V0 is the root of an earlier call with the same values.
__device__ void fault_map3(const DevFriction& FR, int n, int k, const FaultConst& c, const Dn* x, bool solve,
                           double& V0, Dn* y) {
  const Dn csm = dsqrt(x[FX_GM] / x[FX_RHOM]), csp = dsqrt(x[FX_GP] / x[FX_RHOP]);
  const Dn Zsim = 1.0 / (x[FX_RHOM] * csm), Zsip = 1.0 / (x[FX_RHOP] * csp);
  const Dn Ksm = csm * c.geom, Ksp = csp * c.geop;
  const Dn etas = 1.0 / (Zsip + Zsim);
  const double n0 = c.n0, n1 = c.n1;
  Dn dm[3], dp[3];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    dm[l] = c.friction ? x[FX_UM + l] - c.F0m[l] : x[FX_UM + l];
    dp[l] = c.friction ? x[FX_UP + l] - c.F0p[l] : x[FX_UP + l];
  }
  // rot3_xy2nt: (vz, stz, snz)
  const Dn rm0 = dm[0], rm1 = n1 * dm[1] - n0 * dm[2], rm2 = n0 * dm[1] + n1 * dm[2];
  const Dn rp0 = dp[0], rp1 = n1 * dp[1] - n0 * dp[2], rp2 = n0 * dp[1] + n1 * dp[2];
  const Dn phis = etas * (rp2 * Zsip + rm2 * Zsim + rp0 - rm0);
  Dn snz, V = dn(0.0);
  y[FY_PSI] = dn(0.0);
  if (!c.friction) {
    snz = phis;
  } else {
    const Dn Slock = x[FX_S0] + phis;
    const double N = c.N0;
    const DRS rs{FR.par[PAR_A * n + k], FR.par[PAR_B * n + k], FR.par[PAR_V0 * n + k], FR.par[PAR_F0 * n + k],
                 FR.par[PAR_L * n + k], FR.par[PAR_FW * n + k], FR.par[PAR_VW * n + k]};
    Dn S;
    if (N <= 0.0) {
      S = dn(0.0);
      V = Slock / etas;
    } else if (c.xx < FR.xlockm || c.xx > FR.xlockp) {
      const double Sl = FR.flock * N;
      if (fabs(Slock.v) >= Sl) {
        S = dn(Slock.v < 0.0 ? -Sl : Sl);
        V = (Slock - S) / etas;
      } else {
        S = Slock;
      }
    } else if (FR.law == FDMAP_FR_FRICTIONLESS) {
      S = dn(0.0);
      V = Slock / etas;
    } else if (FR.law == FDMAP_FR_LOCKED) {
      S = Slock;
    } else {
      if (solve) {
        double Vs = 0.0, Ss = 0.0;
        d_newton(FR.law, rs, Vs, Ss, Slock.v, N, etas.v, x[FX_PSI].v);
        V0 = Vs;
      }
      // one Newton step from the root carries the implicit derivative
      Dn Sf, dSfdV;
      const Dn Vr = dn(V0);
      dn_strength(FR.law, rs, Vr, x[FX_PSI], dn(N), Sf, dSfdV);
      const Dn R = Sf - (Slock - etas * Vr);
      V = Vr - R / (etas + dSfdV);
      S = Slock - etas * V;
    }
    // set_rates_friction evaluates the state rate at the solved V in every branch
    y[FY_PSI] = dn_state_rate(FR.law, rs, V, x[FX_PSI]);
    snz = S - x[FX_S0];
  }
  const Dn vzp = rp0 + Zsip * (rp2 - snz);
  const Dn vzm = rm0 - Zsim * (rm2 - snz);
  // rot3_nt2xy (+ prestress on a frictional interface)
  Dn Fhp[3] = {vzp, n1 * rp1 + n0 * snz, -n0 * rp1 + n1 * snz};
  Dn Fhm[3] = {vzm, n1 * rm1 + n0 * snz, -n0 * rm1 + n1 * snz};
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    if (c.friction) {
      Fhp[l] = Fhp[l] + c.F0p[l];
      Fhm[l] = Fhm[l] + c.F0m[l];
    }
    y[FY_RM + l] = Ksm * (Fhm[l] - x[FX_UM + l]);
    y[FY_RP + l] = Ksp * (Fhp[l] - x[FX_UP + l]);
  }
}

// one interface of the adjoint: its fault nodes start at `start` in the
// concatenated fault arrays; geometry factors of its two edge sides
struct AdjIfaceInfo {
  int iface, start;
  const double* geom;
  const double* geop;
};

struct AdjFaultArgs {
  double A, Bdt, C;               // RK coefficients of the forward stage
  double t_start, dt;             // step clock: stage time t_start + (n-1) dt + C dt
  int s, nstage;
  const double* ub_in;            // ubar / qbar' of all blocks (concatenated 3-plane layout)
  const double* qp_in;
  double* ub_out;                 // written by the block kernels, the interface terms are added
  const double* store;            // stage inputs: slot (rel*nstage + s), slot_stride doubles each
  long long slot_stride, psi_off; // Psi of the fault nodes at psi_off within a slot
  long long v_off;                // the stage's converged slip rate at v_off
  const AdjClock* ck;
  const double* psib_in;          // Psibar, qbar'_Psi per fault node (ping-pong with the stage)
  const double* qpsib_in;
  double* psib_out;
  double* qpsib_out;
  double* grho;                   // gradient planes of all blocks (concatenated)
  double* gG;
  double* gS0;                    // dJ/dS0 per fault node
  const AdjIfaceInfo* info;
  int nifc, nfault;
  long long boff[MAX_BLOCKS];     // block offsets in the 3-plane layout
  long long goff[MAX_BLOCKS];     // block offsets in the gradient planes
};

// FAULT_LANES threads per fault node, lane j forms the adjoint of input j
// (lanes past FX_N idle); after the band kernels of every block, beside the
// interior tiles (fault nodes touch only edge nodes, which are band nodes)
constexpr int FAULT_LANES = 16;

__global__ void __launch_bounds__(128) adj_fault_kernel(const __grid_constant__ DevDomain D, AdjFaultArgs p) {
  const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int tid = (int)(gt / FAULT_LANES), lane = (int)(gt % FAULT_LANES);
  if (tid >= p.nfault || lane >= FX_N) return;
  int q = 0;
  while (q + 1 < p.nifc && tid >= p.info[q + 1].start) ++q;
  const AdjIfaceInfo& inf = p.info[q];
  const DevIface& I = D.ifc[inf.iface];
  const int k = tid - inf.start, n = I.n;
  const int im = I.im, ip = I.ip;
  const DevBlock& Bm = D.blk[im];
  const DevBlock& Bp = D.blk[ip];
  const int sm = I.direction == 0 ? 1 : 3, sp = I.direction == 0 ? 0 : 2;
  const DevSide& Sm = Bm.side[sm];
  const DevSide& Sp = Bp.side[sp];
  const int km = I.offm + k, kp = I.offp + k;
  int im_, jm_, ip_, jp_;
  side_node_local(sm, km, Bm.nx, Bm.ny, im_, jm_);
  side_node_local(sp, kp, Bp.nx, Bp.ny, ip_, jp_);
  const long long cm = (long long)jm_ * Bm.pitch + im_, cp = (long long)jp_ * Bp.pitch + ip_;
  const long long slot = ((p.ck->rel) * p.nstage + p.s) * p.slot_stride;
  const double* um = p.store + slot + p.boff[im] + cm;
  const double* up = p.store + slot + p.boff[ip] + cp;
  FaultConst c;
  c.n0 = I.nhat[k];
  c.n1 = I.nhat[k + n];
  c.friction = I.coupling != FDMAP_COUPLING_LOCKED;
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    c.F0m[l] = Sm.F0[km + Sm.n * l];
    c.F0p[l] = Sp.F0[kp + Sp.n * l];
  }
  c.geom = inf.geom[km];
  c.geop = inf.geop[kp];
  Dn x[FX_N];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    x[FX_UM + l] = dn(um[l * Bm.plane]);
    x[FX_UP + l] = dn(up[l * Bp.plane]);
  }
  x[FX_RHOM] = dn(Bm.rho[cm]);
  x[FX_GM] = dn(Bm.G[cm]);
  x[FX_RHOP] = dn(Bp.rho[cp]);
  x[FX_GP] = dn(Bp.G[cp]);
  x[FX_PSI] = dn(0.0);
  x[FX_S0] = dn(0.0);
  c.N0 = 0.0;
  c.xx = 0.0;
  if (c.friction) {
    const DevFriction& FR = I.fr;
    x[FX_PSI] = dn(p.store[slot + p.psi_off + tid]);
    // total shear load of the stage, as the forward's solve forms it
    const double t0 = __dadd_rn(p.t_start, __dmul_rn((double)(p.ck->n - 1), p.dt));
    const double t = __dadd_rn(t0, __dmul_rn(p.C, p.dt));
    double S0l, N0l;
    d_load_stress(FR, n, k, I.x[k], I.y[k], t, S0l, N0l);
    double r0p[3];
    rot3_xy2nt(c.F0p, c.n0, c.n1, r0p);
    x[FX_S0] = dn(S0l + r0p[2]);
    double stt, snt, snn;
    xy2nt_mat(Bp.F0v[3], Bp.F0v[4], Bp.F0v[6], stt, snt, snn, c.n0, c.n1);
    const double pp = FR.tp_use ? FR.tp_p0 : 0.0;
    c.N0 = N0l + (-snn - pp);
    c.xx = I.x[k] * FR.cos_angle + I.y[k] * FR.sin_angle;
  }
  // adjoint weights of the outputs
  double yb[FY_N];
  const long long om = p.boff[im] + cm, op = p.boff[ip] + cp;
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    yb[FY_RM + l] = p.qp_in[om + l * Bm.plane] + p.Bdt * p.ub_in[om + l * Bm.plane];
    yb[FY_RP + l] = p.qp_in[op + l * Bp.plane] + p.Bdt * p.ub_in[op + l * Bp.plane];
  }
  double psib = 0.0, qs_psi = 0.0;
  if (c.friction) {
    psib = p.psib_in[tid];
    qs_psi = p.qpsib_in[tid] + p.Bdt * psib;
  }
  yb[FY_PSI] = qs_psi;
  // the root the forward's Newton solve converged to in this stage, then this
  // lane's tangent through one Newton step from it
  double V0 = c.friction ? p.store[slot + p.v_off + tid] : 0.0;
  Dn y[FY_N];
  const bool active = c.friction || (lane != FX_PSI && lane != FX_S0);
  double xb = 0.0;
  if (active) {
    x[lane].d = 1.0;
    fault_map3(I.fr, n, k, c, x, false, V0, y);
#pragma unroll
    for (int o = 0; o < FY_N; ++o) xb += yb[o] * y[o].d;
  }
  // every lane owns the elements it writes
  if (lane < FX_UP) p.ub_out[om + (lane - FX_UM) * Bm.plane] += xb;
  else if (lane < FX_PSI) p.ub_out[op + (lane - FX_UP) * Bp.plane] += xb;
  else if (lane == FX_PSI) {
    p.psib_out[tid] = psib + xb;
    p.qpsib_out[tid] = p.A * qs_psi;
  } else if (lane == FX_S0) {
    if (c.friction) p.gS0[tid] += xb;
  } else if (lane == FX_RHOM) p.grho[p.goff[im] + cm] += xb;
  else if (lane == FX_GM) p.gG[p.goff[im] + cm] += xb;
  else if (lane == FX_RHOP) p.grho[p.goff[ip] + cp] += xb;
  else p.gG[p.goff[ip] + cp] += xb;
}

// Psi of every frictional fault node -> its place in stage slot (rel*nstage + s)
// With psi: Psi before stage s into slot (rel*nstage + s), and the slip rate
// the previous stage converged to into slot (rel*nstage + s - 1) when s > 0.
// Without psi (after the last stage): only that stage's slip rate, slot
// (rel*nstage + s).  Nodes of locked interfaces store 0.
__global__ void adj_stash_psi(const __grid_constant__ DevDomain D, const AdjIfaceInfo* info, int nifc, int nfault,
                              double* store, long long slot_stride, long long psi_off, long long v_off,
                              const long long* rel, int s, int nstage, int psi) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= nfault) return;
  int q = 0;
  while (q + 1 < nifc && tid >= info[q + 1].start) ++q;
  const DevIface& I = D.ifc[info[q].iface];
  const int k = tid - info[q].start;
  const bool locked = I.coupling == FDMAP_COUPLING_LOCKED;
  const long long base = (*rel) * nstage;
  if (psi) {
    store[(base + s) * slot_stride + psi_off + tid] = locked ? 0.0 : I.fr.st[ST_PSI * I.n + k];
    if (s > 0) store[(base + s - 1) * slot_stride + v_off + tid] = locked ? 0.0 : I.fr.st[ST_V * I.n + k];
  } else {
    store[(base + s) * slot_stride + v_off + tid] = locked ? 0.0 : I.fr.st[ST_V * I.n + k];
  }
}

// vz at the receivers (one pointer per receiver into the state) for sample ts->n
__global__ void adj_sample_ptr(const double* const* __restrict__ rec, int nrec, const TimeState* ts, double* traces,
                               int nsamples) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = ts->n;
  if (r >= nrec || n < 1 || n > nsamples) return;
  traces[(n - 1) * nrec + r] = *rec[r];
}

// end of a forward step: vz at the receivers of the new state (sample n+1),
// then n += 1 and, given the store clock, its step index += 1
__global__ void adj_sample_advance_ptr(const double* const* __restrict__ rec, int nrec, TimeState* ts,
                                       double* traces, int nsamples, AdjClock* ck) {
  const long long n = ts->n + 1;
  for (int r = threadIdx.x; r < nrec; r += blockDim.x)
    if (n >= 1 && n <= nsamples) traces[(n - 1) * nrec + r] = *rec[r];
  __syncthreads();
  if (threadIdx.x == 0) {
    ts->n = n;
    if (ck) ck->rel += 1;
  }
}

// interface impedances from the edge impedances of both sides (mode III)
__global__ void adj_iface_material(DevIface I, DevSide Sm, DevSide Sp) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= I.n) return;
  const double Zsim = 1.0 / Sm.M[I.offm + k], Zsip = 1.0 / Sp.M[I.offp + k];
  I.icoef[IC_ZSIM * I.n + k] = Zsim;
  I.icoef[IC_ZSIP * I.n + k] = Zsip;
  I.icoef[IC_ETAS * I.n + k] = 1.0 / (Zsip + Zsim);
}

}  // namespace fdmap
