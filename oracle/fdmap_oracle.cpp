// CPU restatement of FDMAP's explicit time step -- TEST INFRASTRUCTURE ONLY.
// See fdmap_oracle.h for scope and parity status.  Every routine cites the
// reference file:line it follows; expressions keep the Fortran evaluation
// order (left to right, parenthesised as in the source) and the build uses
// -ffp-contract=off so no fused multiply-adds are introduced.
#include "fdmap_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::vector<double> vec;

// ---------------------------------------------------------------------------
// Coefficient tables, restated from fd_coeff.f90:83-246 and time_step.f90:36-63.
// ---------------------------------------------------------------------------
struct Ops {
  int nbnd, nbst, pI;
  double DI[4];     // DI(s), s = 1..pI
  double DL[6][9];  // DL(s,r) at [r][s]
  double AI[4];     // AI(s), s = 0..pI (artificial dissipation, symmetric)
  double AL[6][9];  // AL(s,r) at [r][s]; AR(-s,-r) = AL(s,r) (fd_coeff.f90:244)
  double HL[6];     // diagonal norm near the boundary, HR(-i) = HL(i) (fd_coeff.f90:79-245)
};

bool make_ops(int method, Ops* o) {
  std::memset(o, 0, sizeof(*o));
  if (method == FDMAP_SBP2) {
    o->nbnd = 2; o->nbst = 1; o->pI = 1;
    o->DI[1] = 0.5;
    o->HL[0] = 0.5;
    o->DL[0][0] = -1.0; o->DL[0][1] = 1.0;
    o->AI[0] = -1.0; o->AI[1] = 0.5;
    o->AL[0][0] = -1.0; o->AL[0][1] = 1.0;
    return true;
  }
  if (method == FDMAP_SBP4) {
    o->nbnd = 6; o->nbst = 4; o->pI = 2;
    o->DI[1] = 0.666666666666667; o->DI[2] = -0.083333333333333;
    {
      const double hl[4] = {0.354166666666667, 1.229166666666667, 0.895833333333333, 1.020833333333333};
      for (int r = 0; r < 4; ++r) o->HL[r] = hl[r];
    }
    double t[4][6] = {{-1.411764705882353, 1.735294117647059, -0.235294117647059, -0.088235294117647, 0.0, 0.0},
                      {-0.5, 0.0, 0.5, 0.0, 0.0, 0.0},
                      {0.093023255813953, -0.686046511627907, 0.0, 0.686046511627907, -0.093023255813953, 0.0},
                      {0.030612244897959, 0.0, -0.602040816326531, 0.0, 0.653061224489796, -0.081632653061224}};
    for (int r = 0; r < 4; ++r) for (int s = 0; s < 6; ++s) o->DL[r][s] = t[r][s];
    o->AI[0] = -0.500000000000000; o->AI[1] = 0.333333333333333; o->AI[2] = -0.083333333333333;
    double a[4][6] = {{-0.470588235294118, 0.941176470588235, -0.470588235294118, 0.0, 0.0, 0.0},
                      {0.271186440677966, -0.610169491525424, 0.406779661016949, -0.067796610169492, 0.0, 0.0},
                      {-0.186046511627907, 0.558139534883721, -0.651162790697674, 0.372093023255814, -0.093023255813953, 0.0},
                      {0.0, -0.081632653061224, 0.326530612244898, -0.489795918367347, 0.326530612244898, -0.081632653061224}};
    for (int r = 0; r < 4; ++r) for (int s = 0; s < 6; ++s) o->AL[r][s] = a[r][s];
    return true;
  }
  if (method == FDMAP_SBP6) {
    o->nbnd = 9; o->nbst = 6; o->pI = 3;
    o->DI[1] = 0.75; o->DI[2] = -0.15; o->DI[3] = 0.016666666666667;
    {
      const double hl[6] = {0.315949074074074, 1.390393518518518, 0.627546296296296,
                            1.240509259259259, 0.911689814814815, 1.013912037037037};
      for (int r = 0; r < 6; ++r) o->HL[r] = hl[r];
    }
    double t[6][9] = {
        {-1.582533518939116, 2.033378678700676, -0.141512858744873, -0.450398306578272, 0.104488069284042, 0.036577936277544, 0, 0, 0},
        {-0.462059195631158, 0.0, 0.287258622978251, 0.258816087376832, -0.069112065532624, -0.014903449191300, 0, 0, 0},
        {0.071247104721830, -0.636451095137907, 0.0, 0.606235523609147, -0.022902190275815, -0.018129342917256, 0, 0, 0},
        {0.114713313798970, -0.290087484386815, -0.306681191361148, 0.0, 0.520262285050482, -0.051642265516119, 0.013435342414630, 0, 0},
        {-0.036210680656541, 0.105400944933782, 0.015764336127392, -0.707905442575989, 0.0, 0.769199413962647, -0.164529643265203, 0.018281071473911, 0},
        {-0.011398193015050, 0.020437334208704, 0.011220896474665, 0.063183694641876, -0.691649024426814, 0.0, 0.739709139060752, -0.147941827812150, 0.016437980868017}};
    for (int r = 0; r < 6; ++r) for (int s = 0; s < 9; ++s) o->DL[r][s] = t[r][s];
    o->AI[0] = -0.333333333333333; o->AI[1] = 0.25; o->AI[2] = -0.1; o->AI[3] = 0.016666666666667;
    double a[6][9] = {
        {-0.105502234595941, 0.316506703787823, -0.316506703787823, 0.105502234595941, 0, 0, 0, 0, 0},
        {0.071922084408557, -0.227753267293765, 0.251727295429951, -0.107883126612836, 0.011987014068093, 0, 0, 0, 0},
        {-0.159350793065290, 0.557727775728513, -0.743637034304685, 0.478052379195869, -0.159350793065290, 0.026558465510882, 0, 0, 0},
        {0.026870684829259, -0.120918081731666, 0.241836163463333, -0.282142190707221, 0.201530136219444, -0.080612054487778, 0.013435342414630, 0, 0},
        {0.0, 0.018281071473911, -0.109686428843468, 0.274216072108671, -0.365621429478228, 0.274216072108671, -0.109686428843468, 0.018281071473911, 0},
        {0.0, 0.0, 0.016437980868017, -0.098627885208100, 0.246569713020251, -0.328759617360334, 0.246569713020251, -0.098627885208100, 0.016437980868017}};
    for (int r = 0; r < 6; ++r) for (int s = 0; s < 9; ++s) o->AL[r][s] = a[r][s];
    return true;
  }
  return false;
}

struct RK {
  int nstage;
  double A[5], B[5], C[6];
};

bool make_rk(int order, RK* rk) {
  std::memset(rk, 0, sizeof(*rk));
  switch (order) {
    case 1: rk->nstage = 1; rk->A[0] = 0; rk->B[0] = 1; rk->C[1] = 1; return true;
    case 2: rk->nstage = 2; rk->A[1] = -1; rk->B[0] = 1; rk->B[1] = 1.0 / 2.0; rk->C[1] = 1; rk->C[2] = 1; return true;
    case 3:
      rk->nstage = 3; rk->A[1] = -5.0 / 9.0; rk->A[2] = -153.0 / 128.0;
      rk->B[0] = 1.0 / 3.0; rk->B[1] = 15.0 / 16.0; rk->B[2] = 8.0 / 15.0;
      rk->C[1] = 1.0 / 3.0; rk->C[2] = 3.0 / 4.0; rk->C[3] = 1.0;
      return true;
    case 4:
      rk->nstage = 5;
      rk->A[1] = -567301805773.0 / 1357537059087.0; rk->A[2] = -2404267990393.0 / 2016746695238.0;
      rk->A[3] = -3550918686646.0 / 2091501179385.0; rk->A[4] = -1275806237668.0 / 842570457699.0;
      rk->B[0] = 1432997174477.0 / 9575080441755.0; rk->B[1] = 5161836677717.0 / 13612068292357.0;
      rk->B[2] = 1720146321549.0 / 2090206949498.0; rk->B[3] = 3134564353537.0 / 4481467310338.0;
      rk->B[4] = 2277821191437.0 / 14882151754819.0;
      rk->C[1] = 1432997174477.0 / 9575080441755.0; rk->C[2] = 2526269341429.0 / 6820363962896.0;
      rk->C[3] = 2006345519317.0 / 3224310063776.0; rk->C[4] = 2802321613138.0 / 2924317926251.0; rk->C[5] = 1.0;
      return true;
  }
  return false;
}

// Fortran SIGN(a,b): |a| with the sign of b (b = -0 gives +|a| for gfortran
// only when -fno-sign-zero; the default honours the sign bit, as copysign).
inline double fsign(double a, double b) { return std::copysign(std::fabs(a), b); }

// ---------------------------------------------------------------------------
// Rate table (rates.f90 / rates_heterogeneous.f90).  Each rate component c is
// a flat sum of products of a metric average with one field:
//   q-flux at point k:  +t1 - t2,  t1 = (0.5*(yr(k)+yr(c)))*F(fa)[*gamma]
//                                   t2 = (0.5*(xr(k)+xr(c)))*F(fb)[*gamma]
//   r-flux at point k:  -t1 + t2   with yq, xq instead of yr, xr.
// ---------------------------------------------------------------------------
struct RateDef {
  int fa, fb;        // field of the Y-metric term, X-metric term (-1: absent)
  bool ga, gb;       // multiply that term by gamma
  int coef;          // 0: /rho, 1: *G, 2: *M
};

const RateDef kMode2[5] = {{2, 3, false, false, 0}, {3, 4, false, false, 0}, {0, 1, false, true, 2},
                           {1, 0, false, false, 1}, {0, 1, true, false, 2}};
const RateDef kMode3[3] = {{1, 2, false, false, 0}, {0, -1, false, false, 1}, {-1, 0, false, false, 1}};

}  // namespace

struct Side {
  int bc, n;
  vec M, F0, normal, x, y;
  vec F, Fhat;  // (n, nF)
  vec U, DU;    // (n, nU) boundary displacement and its rate (bnd_fields, fields.f90:14-15)
};

struct Blk {
  int mgx, pgx, mgy, pgy;
  double rho, G, M, gamma, nu;
  double F0[9];
  Side side[4];
  int src_ok, src_i0, src_j0;
  double src_hx, src_hy, src_ax, src_ay;
  double Cdiss;  // scaled artificial dissipation (0: set_rates, >0: set_rates_dissipation)
  bool pmlx, pmly;  // pml_list (material.f90:152-222)
  double pml_n, pml_sigma, pml_kappa, pml_mx, pml_px, pml_my, pml_py;
};

struct Fric {
  int law, reg, rup_field, force, ld_shape, tp_use;
  double rup_threshold, angle, xlockm, xlockp, flock, skempton;
  double kn_c0, kn_fd, kn_dfdx, kn_vL, kn_vR, kn_xL, kn_xR, kn_tmax;
  double ld_S, ld_N, ld_T, ld_R, ld_x0, ld_y0, tp_p0;
  vec a, b, V0, f0, L, fw, Vw, c0, fs, fd, Dc, bsS0, bsN0;
  vec st[FDMAP_FAULT_NFIELDS];
  vec tap[FDMAP_FAULT_NFIELDS];  // the fields at stage 1's output point of the last step (tap on)
};

struct Ifc {
  int direction, im, ip, m, p, coupling;
  vec nhat, x, y;
  Fric fr;
};

struct oracle_domain {
  int mode, nF, nx, ny, nblocks, nifaces, het;
  Ops op;
  RK rk;
  std::vector<Blk> blk;
  std::vector<Ifc> ifc;
  vec F, DF, x, y, xq, xr, yq, yr, J, Ji;
  vec rho, G, M, gamma, nu;
  vec Wx, DWx, Wy, DWy;  // PML fields (nx,ny,nF), allocated when some block has pmlx / pmly (fields.f90:203-210)
  vec U, DU;             // body displacement and its rate (nx,ny,nU), displacement = T (fields.f90:183-186)
  vec pgv, pga;          // peak ground velocity / acceleration (nx,ny), peak = T (fields.f90:187-190)
  bool energy = false;   // energy_balance = T: stage-1 mechanical energy of every block (energy.f90:9-96)
  std::vector<double> Etot;  // per block, then the sum over blocks
  fdmap_source src;
  // forcing from file (source.f90:12-14): the frames of the current step and its window
  std::FILE* frc = nullptr;
  vec frc_old, frc_new;
  double frc_t_old = 0.0, frc_t_new = 0.0;
  ~oracle_domain() {
    if (frc) std::fclose(frc);
  }
  double t;
  long long newton_fail;   // solves whose first Newton attempt failed (the reference's warning)
  long long newton_stop;   // solves whose retry failed too (the reference stops there)
  int newton_imax = 99;    // friction.f90:924 imax
  double newton_tol_scale = 1.0;  // atolR = 1e4*eps times this (a test of the result's sensitivity to atolR)
  bool tap = false;        // keep each step's stage-1 fault fields (write_output's view, time_step.f90:129)
  // block-aligned partition: blocks this rank steps (empty: all) and the
  // exchange of interface edge values, called after prepare_edges
  std::vector<char> owned;
  int (*exchange)(void*, long long) = nullptr;
  void* exchange_user = nullptr;
  long long xstage = 0;
};

namespace {

inline size_t G2(const oracle_domain& D, int i, int j) { return (size_t)(i - 1) + (size_t)D.nx * (size_t)(j - 1); }

vec copyv(const double* p, size_t n) { return p ? vec(p, p + n) : vec(); }

// ---------------------------------------------------------------------------
// geometry.f90:285-336 rotations and fields.f90:1297-1356 wrappers
// ---------------------------------------------------------------------------
inline void xy2nt_vec(double wx, double wy, double& wt, double& wn, const double n[2]) {
  wt = n[1] * wx - n[0] * wy;
  wn = n[0] * wx + n[1] * wy;
}
inline void nt2xy_vec(double& wx, double& wy, double wt, double wn, const double n[2]) {
  wx = n[1] * wt + n[0] * wn;
  wy = -n[0] * wt + n[1] * wn;
}
inline void xy2nt_mat(double wxx, double wxy, double wyy, double& wtt, double& wnt, double& wnn, const double n[2]) {
  wtt = -(2.0 * n[0] * n[1] * wxy) + (n[1] * n[1]) * wxx + (n[0] * n[0]) * wyy;
  wnt = n[0] * n[1] * (wxx - wyy) + ((n[1] * n[1]) - (n[0] * n[0])) * wxy;
  wnn = 2.0 * n[0] * n[1] * wxy + (n[0] * n[0]) * wxx + (n[1] * n[1]) * wyy;
}
inline void nt2xy_mat(double& wxx, double& wxy, double& wyy, double wtt, double wnt, double wnn, const double n[2]) {
  wxx = 2.0 * n[0] * n[1] * wnt + (n[1] * n[1]) * wtt + (n[0] * n[0]) * wnn;
  wxy = -(n[0] * n[1] * (wtt - wnn)) + ((n[1] * n[1]) - (n[0] * n[0])) * wnt;
  wyy = -(2.0 * n[0] * n[1] * wnt) + (n[0] * n[0]) * wtt + (n[1] * n[1]) * wnn;
}
// mode II: F(6) -> vt, vn, stt, snt, snn, szz
inline void rot2_xy2nt(const double* F, const double n[2], double* o) {
  xy2nt_vec(F[0], F[1], o[0], o[1], n);
  xy2nt_mat(F[2], F[3], F[4], o[2], o[3], o[4], n);
  o[5] = F[5];
}
inline void rot2_nt2xy(double* F, const double n[2], double vt, double vn, double stt, double snt, double snn, double szz) {
  nt2xy_vec(F[0], F[1], vt, vn, n);
  nt2xy_mat(F[2], F[3], F[4], stt, snt, snn, n);
  F[5] = szz;
}
// mode III: F(3) -> vz, stz, snz
inline void rot3_xy2nt(const double* F, const double n[2], double* o) {
  o[0] = F[0];
  xy2nt_vec(F[1], F[2], o[1], o[2], n);
}
inline void rot3_nt2xy(double* F, const double n[2], double vz, double stz, double snz) {
  F[0] = vz;
  nt2xy_vec(F[1], F[2], stz, snz, n);
}

// ---------------------------------------------------------------------------
// utilities.f90:303-420 shapes used by load_stress
// ---------------------------------------------------------------------------
const double kTol = 100.0 * 2.220446049250313e-16;
double boxcar(double r, double w, double fin, double fout) {
  if (-w + kTol < r && r < w - kTol) return fin;
  if (std::fabs(-w - r) <= kTol || std::fabs(r - w) <= kTol) return 0.5 * (fin + fout);
  return fout;
}
double gaussian(double r, double w, double fin, double fout) { return fout + (fin - fout) * std::exp(-0.5 * ((r / w) * (r / w))); }
double smooth(double r, double w, double fin, double fout) {
  if (r >= w - kTol) return fout;
  return fout + (fin - fout) * std::exp((r * r) / ((r * r) - (w * w)));
}
double triangle(double r, double w, double fin, double fout) {
  if (-w < r && r < w) return fout + (fin - fout) * (1.0 - r / w);
  return fout;
}
double smooth_boxcar(double r, double w, double l, double fin, double fout) {
  double f;
  if (r <= w) f = 1.0;
  else if (r < w + l) f = 0.5 * (1.0 + std::tanh(l / (r - w - l) + l / (r - w)));
  else f = 0.0;
  return fout + (fin - fout) * f;
}

// ---------------------------------------------------------------------------
// friction.f90
// ---------------------------------------------------------------------------
enum { D_ = FDMAP_FAULT_D, PSI_ = FDMAP_FAULT_PSI, DPSI_ = FDMAP_FAULT_DPSI, TRUP_ = FDMAP_FAULT_TRUP,
       V_ = FDMAP_FAULT_V, O_ = FDMAP_FAULT_O, S_ = FDMAP_FAULT_S, N_ = FDMAP_FAULT_N, S0_ = FDMAP_FAULT_S0,
       N0_ = FDMAP_FAULT_N0, DS_ = FDMAP_FAULT_DS, DN_ = FDMAP_FAULT_DN, DDS_ = FDMAP_FAULT_DDS,
       DDN_ = FDMAP_FAULT_DDN, W_ = FDMAP_FAULT_W, DW_ = FDMAP_FAULT_DW, NREG_ = FDMAP_FAULT_NREG,
       DNREG_ = FDMAP_FAULT_DNREG };

struct RS { double a, b, V0, f0, L, fw, Vw; };

// x**8 with an integer exponent: gfortran evaluates it by repeated squaring
inline double pow8(double x) {
  double x2 = x * x, x4 = x2 * x2;
  return x4 * x4;
}

// arcsinh (friction.f90:1293-1304)
double arcsinh(double x) {
  double y = std::fabs(x);
  double f = std::log(y + std::sqrt(y * y + 1.0));
  return fsign(f, x);
}

// load_ramp (friction.f90:1455-1484)
double load_ramp(double t, const Fric& FR) {
  if (FR.ld_T <= 0.0) return t < 0.0 ? 0.0 : 1.0;
  return t < 0.0 ? 0.0 : 1.0 - std::exp(-t / FR.ld_T);
}

// load_stress, default problem branch (friction.f90:1317-1374)
void load_stress(const Fric& FR, double x, double y, double t, int k, double& S0, double& N0) {
  double xx = x * std::cos(FR.angle) + y * std::sin(FR.angle);
  double r = std::fabs((xx - FR.ld_x0) / FR.ld_R);
  N0 = 0; S0 = 0;
  if (!FR.bsS0.empty()) S0 = FR.bsS0[k];
  if (!FR.bsN0.empty()) N0 = FR.bsN0[k];
  double A = 0.0;
  switch (FR.ld_shape) {
    case FDMAP_LD_NONE: A = 0.0; break;
    case FDMAP_LD_UNIFORM: A = 1.0; break;
    case FDMAP_LD_LINEAR: A = (xx - FR.ld_x0) / FR.ld_R; break;
    case FDMAP_LD_BOXCAR: A = boxcar(r, 1.0, 1.0, 0.0); break;
    case FDMAP_LD_SMOOTH_BOXCAR: A = smooth_boxcar(r, 1.0, 0.1, 1.0, 0.0); break;
    case FDMAP_LD_TRIANGLE: A = triangle(r, 1.0, 1.0, 0.0); break;
    case FDMAP_LD_SMOOTH: A = smooth(r, 1.0, 1.0, 0.0); break;
    case FDMAP_LD_GAUSSIAN: A = gaussian(r, 1.0, 1.0, 0.0); break;
  }
  double B = load_ramp(t, FR);
  S0 = S0 + FR.ld_S * A * B;
  N0 = N0 + FR.ld_N * A * B;
}

// strength (friction.f90:1041-1074)
void strength(int law, const RS& rs, double V, double Psi, double N, double& S, double& dSdV) {
  if (law == FDMAP_FR_SL || law == FDMAP_FR_FL) {
    if (V == 0.0) { S = 0.0; dSdV = 1e10; }
    else {
      double absV = std::fabs(V);
      double f = rs.a * std::log(absV / rs.V0) + Psi;
      S = N * fsign(f, V);
      dSdV = N * rs.a / absV;
    }
  } else {
    double O = 0.5 / rs.V0 * std::exp(Psi / rs.a);
    S = rs.a * N * arcsinh(O * V);
    dSdV = rs.a * N * O / std::sqrt(1.0 + (V * O) * (V * O));
  }
}

// estimate_V (friction.f90:1077-1098)
void estimate_V(int law, const RS& rs, double& V, double Slock, double N, double Psi) {
  double SaN = Slock / (rs.a * N);
  if (std::fabs(SaN) > 10.0) return;
  if (law == FDMAP_FR_SL || law == FDMAP_FR_FL) V = fsign(rs.V0 * std::exp(-Psi / rs.a) * std::exp(std::fabs(SaN)), SaN);
  else if (law != FDMAP_FR_RSF) V = 2.0 * rs.V0 * std::exp(-Psi / rs.a) * std::sinh(SaN);
}

// newton_solver (friction.f90:909-1038); returns fail.  imax is the
// reference's parameter 99 unless a test lowers it (oracle_set_newton_limit).
bool newton_solver(int law, const RS& rs, double& V, double& S, double Slock, double N, double eta, double Psi,
                   int imax, double tol_scale = 1.0) {
  const double rtolV = 0.0, atolV = 0.0, atolR = 2.220446049250313e-16 * 1e4 * tol_scale;
  double Vmin = std::min(0.0, Slock / eta);
  double Vmax = std::max(0.0, Slock / eta);
  estimate_V(law, rs, V, Slock, N, Psi);
  if (V <= Vmin || Vmax <= V) V = 0.5 * (Vmin + Vmax);
  int i;
  for (i = 1; i <= imax; ++i) {
    S = Slock - eta * V;
    double dSdV = -eta;
    double Sf, dSfdV;
    strength(law, rs, V, Psi, N, Sf, dSfdV);
    double R = -S + Sf;
    if (R > 0.0) Vmax = V;
    if (R < 0.0) Vmin = V;
    double dRdV = -dSdV + dSfdV;
    double dV = -R / dRdV;
    if (std::fabs(R) <= atolR) break;
    if (i == imax) break;
    V = V + dV;
    if (V <= Vmin || Vmax <= V) {
      if (Vmin == 0.0) V = 0.1 * Vmax;
      else if (Vmax == 0.0) V = 0.1 * Vmin;
      else V = fsign(std::sqrt(Vmin * Vmax), Slock);
      dV = Vmax - Vmin;
    }
    if (std::fabs(dV) <= atolV + rtolV * (std::fabs(V) + std::fabs(dV))) break;
  }
  return i == imax;
}

// solve_friction (friction.f90:593-828) for interface node k
void solve_friction(oracle_domain& Dm, Fric& FR, int k, double S0, double N0, double phip, double phis, double eta,
                    double x, double y, double t, double dt) {
  double& V = FR.st[V_][k];
  double& S = FR.st[S_][k];
  double& O = FR.st[O_][k];
  double& N = FR.st[N_][k];
  double& Nreg = FR.st[NREG_][k];
  const double D = FR.st[D_][k];
  const double Psi = FR.st[PSI_][k];
  load_stress(FR, x, y, t, k, FR.st[S0_][k], FR.st[N0_][k]);
  FR.st[S0_][k] = FR.st[S0_][k] + S0;
  FR.st[N0_][k] = FR.st[N0_][k] + N0;
  double Slock = FR.st[S0_][k] + phis;
  double Nlock = FR.st[N0_][k] - (1.0 - FR.skempton) * phip;
  O = 0.0;
  N = Nlock;
  if (Nlock <= 0.0) {
    S = 0.0;
    V = Slock / eta;
    return;
  }
  if (dt == 0.0) Nreg = N;
  if (!FR.reg) Nreg = N;
  double xx = x * std::cos(FR.angle) + y * std::sin(FR.angle);
  if (xx < FR.xlockm || xx > FR.xlockp) {
    S = FR.flock * Nreg;
    if (std::fabs(Slock) >= S) { S = fsign(S, Slock); V = (Slock - S) / eta; }
    else { V = 0.0; S = Slock; }
    return;
  }
  if (FR.law == FDMAP_FR_FRICTIONLESS) { S = 0.0; V = Slock / eta; return; }
  if (FR.law == FDMAP_FR_LOCKED) { V = 0.0; S = Slock; return; }
  double Sk = 0.0;
  if (FR.force) {
    xx = x * std::cos(FR.angle) + y * std::sin(FR.angle);
    double xm = FR.kn_xL + FR.kn_vL * std::min(t, FR.kn_tmax);
    double fkm = (xx < xm) ? FR.kn_fd + FR.kn_dfdx * (xm - xx) : FR.kn_fd;
    double xp = FR.kn_xR + FR.kn_vR * std::min(t, FR.kn_tmax);
    double fkp = (xx > xp) ? FR.kn_fd + FR.kn_dfdx * (xx - xp) : FR.kn_fd;
    Sk = FR.kn_c0 + Nreg * std::max(fkm, fkp);
  }
  if (FR.law == FDMAP_FR_SW) {
    double c0 = FR.c0[k], fs = FR.fs[k], fd = FR.fd[k], Dc = FR.Dc[k];
    S = c0 + std::max(Nreg, 0.0) * ((fs - (fs - fd) * std::min(D, Dc) / Dc));
    if (FR.force) S = std::min(S, Sk);
    if (std::fabs(Slock) >= S) { S = fsign(S, Slock); V = (Slock - S) / eta; }
    else { V = 0.0; S = Slock; }
    return;
  }
  RS rs{FR.a[k], FR.b[k], FR.V0[k], FR.f0[k], FR.L[k], FR.fw[k], FR.Vw[k]};
  bool fail = newton_solver(FR.law, rs, V, S, Slock, Nreg, eta, Psi, Dm.newton_imax, Dm.newton_tol_scale);
  if (fail) {
    // the reference warns, then retries from the failed iterate V, S
    // (friction.f90:789-790) and stops on a second failure (friction.f90:1014);
    // the oracle counts both events instead
    Dm.newton_fail++;
    if (newton_solver(FR.law, rs, V, S, Slock, Nreg, eta, Psi, Dm.newton_imax, Dm.newton_tol_scale)) Dm.newton_stop++;
  }
  if (FR.force) {
    if (Sk < std::fabs(S)) { S = fsign(Sk, Slock); V = (Slock - S) / eta; }
  }
}

// state_rate (friction.f90:1147-1264)
double state_rate(const Fric& FR, double V, double Psi, int k) {
  if (FR.law == FDMAP_FR_FRICTIONLESS || FR.law == FDMAP_FR_SW || FR.law == FDMAP_FR_LOCKED) return 0.0;
  if (V == 0.0) return 0.0;
  RS rs{FR.a[k], FR.b[k], FR.V0[k], FR.f0[k], FR.L[k], FR.fw[k], FR.Vw[k]};
  double absV = std::fabs(V);
  double frs, fss, fLV, Psiss;
  switch (FR.law) {
    case FDMAP_FR_SL:
      frs = rs.a * std::log(absV / rs.V0) + Psi;
      fss = rs.f0 - (rs.b - rs.a) * std::log(absV / rs.V0);
      return -(absV / rs.L) * (frs - fss);
    case FDMAP_FR_FL:
      frs = rs.a * std::log(absV / rs.V0) + Psi;
      fLV = rs.f0 - (rs.b - rs.a) * std::log(absV / rs.V0);
      fss = rs.fw + (fLV - rs.fw) / std::pow(1.0 + pow8(V / rs.Vw), 0.125);
      return -(absV / rs.L) * (frs - fss);
    case FDMAP_FR_RSL:
      fss = rs.f0 - (rs.b - rs.a) * std::log(absV / rs.V0);
      frs = rs.a * arcsinh(0.5 * absV / rs.V0 * std::exp(Psi / rs.a));
      return -(absV / rs.L) * (frs - fss);
    case FDMAP_FR_RFL:
      fLV = rs.f0 - (rs.b - rs.a) * std::log(absV / rs.V0);
      fss = rs.fw + (fLV - rs.fw) / std::pow(1.0 + pow8(V / rs.Vw), 0.125);
      frs = rs.a * arcsinh(0.5 * absV / rs.V0 * std::exp(Psi / rs.a));
      return (absV / rs.L) * (fss - frs);
    case FDMAP_FR_RSF:
      fLV = rs.f0 - (rs.b - rs.a) * std::log(absV / rs.V0);
      fss = rs.fw + (fLV - rs.fw) / std::pow(1.0 + pow8(V / rs.Vw), 0.125);
      Psiss = rs.a * std::log(2.0 * rs.V0 / absV * std::sinh(fss / rs.a));
      return (absV / rs.L) * (Psiss - Psi);
    case FDMAP_FR_RAL:
      return (rs.b * rs.V0 / rs.L) * (std::exp((rs.f0 - Psi) / rs.b) - absV / rs.V0);
  }
  return 0.0;
}

// set_rates_friction + rupture_front + regularize_N (friction.f90:1101-1144, 1267-1290)
void set_rates_friction(Fric& FR, int n, double t) {
  for (int k = 0; k < n; ++k) {
    FR.st[DDS_][k] = FR.st[DDS_][k] + FR.st[V_][k];
    FR.st[DDN_][k] = FR.st[DDN_][k] + FR.st[O_][k];
    FR.st[DPSI_][k] = FR.st[DPSI_][k] + state_rate(FR, FR.st[V_][k], FR.st[PSI_][k], k);
    if (FR.reg) {
      double absV = std::fabs(FR.st[V_][k]);
      double dn = -(absV / FR.L[k]) * (FR.st[NREG_][k] - std::max(FR.st[N_][k], 0.0));
      FR.st[DNREG_][k] = FR.st[DNREG_][k] + dn;
    }
    FR.st[DW_][k] = FR.st[DW_][k] + FR.st[S_][k] * FR.st[V_][k];
    bool rup = FR.rup_field == 1 ? (FR.st[D_][k] > FR.rup_threshold) : (std::fabs(FR.st[V_][k]) > FR.rup_threshold);
    if (rup) FR.st[TRUP_][k] = std::min(FR.st[TRUP_][k], t);
  }
}

// scale_rates_friction (friction.f90:555-573)
void scale_rates_friction(Fric& FR, double A) {
  const int regs[5] = {DDS_, DDN_, DPSI_, DW_, DNREG_};
  for (int r : regs)
    for (auto& v : FR.st[r]) v = A * v;
}

// update_fields_friction (friction.f90:576-590)
void update_fields_friction(Fric& FR, double dt) {
  size_t n = FR.st[V_].size();
  for (size_t k = 0; k < n; ++k) {
    FR.st[DS_][k] = FR.st[DS_][k] + dt * FR.st[DDS_][k];
    FR.st[DN_][k] = FR.st[DN_][k] + dt * FR.st[DDN_][k];
    FR.st[D_][k] = FR.st[D_][k] + dt * std::fabs(FR.st[DDS_][k]);
    FR.st[PSI_][k] = FR.st[PSI_][k] + dt * FR.st[DPSI_][k];
    FR.st[W_][k] = FR.st[W_][k] + dt * FR.st[DW_][k];
    FR.st[NREG_][k] = FR.st[NREG_][k] + dt * FR.st[DNREG_][k];
  }
}

// ---------------------------------------------------------------------------
// boundaries.f90:155-377
// ---------------------------------------------------------------------------
void set_bc_mode3(double* Fhat, const double* F, const double* F0, const double n[2], int bc, double Zs) {
  if (Zs == 0.0) { for (int l = 0; l < 3; ++l) Fhat[l] = F[l]; return; }
  double Zsi = 1.0 / Zs;
  double d[3] = {F[0] - F0[0], F[1] - F0[1], F[2] - F0[2]};
  double r[3];
  rot3_xy2nt(d, n, r);
  double vzFD = r[0], stzFD = r[1], snzFD = r[2], vz, snz;
  switch (bc) {
    case FDMAP_BC_ABSORBING: vz = 0.5 * (vzFD - Zsi * snzFD); snz = 0.5 * (snzFD - Zs * vzFD); break;
    case FDMAP_BC_FREE: vz = vzFD - Zsi * snzFD; snz = 0.0; break;
    case FDMAP_BC_RIGID: vz = 0.0; snz = snzFD - Zs * vzFD; break;
    default: vz = vzFD; snz = snzFD; break;  // other mode-II-only codes are rejected at create
  }
  rot3_nt2xy(Fhat, n, vz, stzFD, snz);
  for (int l = 0; l < 3; ++l) Fhat[l] = Fhat[l] + F0[l];
}

void set_bc_mode2(double* Fhat, const double* F, const double* F0, const double n[2], int bc, double Zs, double Zp,
                  double gamma) {
  double Zsi = (Zs == 0.0) ? 0.0 : 1.0 / Zs;
  double Zpi = 1.0 / Zp;
  bool zero_variant = (bc == FDMAP_BC_ABSORBING_0 || bc == FDMAP_BC_FREE_0 || bc == FDMAP_BC_RIGID_0);
  double d[6], r[6];
  for (int l = 0; l < 6; ++l) d[l] = zero_variant ? F[l] : F[l] - F0[l];
  rot2_xy2nt(d, n, r);
  double vtFD = r[0], vnFD = r[1], sttFD = r[2], sntFD = r[3], snnFD = r[4], szzFD = r[5];
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
    case FDMAP_BC_FREE_VELOCITY:
      vt = vtFD - Zsi * sntFD; snt = sntFD; vn = vnFD - Zpi * snnFD; snn = snnFD;
      break;
    default:
      vt = vtFD; snt = sntFD; vn = vnFD; snn = snnFD;
      break;
  }
  double stt = sttFD - gamma * (snnFD - snn);
  double szz = szzFD - gamma * (snnFD - snn);
  rot2_nt2xy(Fhat, n, vt, vn, stt, snt, snn, szz);
  if (!zero_variant)
    for (int l = 0; l < 6; ++l) Fhat[l] = Fhat[l] + F0[l];
}

// ---------------------------------------------------------------------------
// interfaces.f90:676-1012
// ---------------------------------------------------------------------------
void locked_mode3(double* Fhm, double* Fhp, const double* Fm, const double* Fp, const double n[2], double Zsm, double Zsp) {
  double rp[3], rm[3];
  rot3_xy2nt(Fp, n, rp);
  rot3_xy2nt(Fm, n, rm);
  double Zsip = 1.0 / Zsp, Zsim = 1.0 / Zsm;
  double etas = 1.0 / (Zsip + Zsim);
  double phis = etas * (rp[2] * Zsip + rm[2] * Zsim + rp[0] - rm[0]);
  double snzp = phis, snzm = phis;
  double vzp = rp[0] + Zsip * (rp[2] - snzp);
  double vzm = rm[0] - Zsim * (rm[2] - snzm);
  rot3_nt2xy(Fhp, n, vzp, rp[1], snzp);
  rot3_nt2xy(Fhm, n, vzm, rm[1], snzm);
}

void locked_mode2(double* Fhm, double* Fhp, const double* Fm, const double* Fp, const double n[2], double Zsm,
                  double Zsp, double Zpm, double Zpp, double gm, double gp) {
  double rp[6], rm[6];
  rot2_xy2nt(Fp, n, rp);
  rot2_xy2nt(Fm, n, rm);
  double Zsip = 1.0 / Zsp, Zsim = 1.0 / Zsm, Zpip = 1.0 / Zpp, Zpim = 1.0 / Zpm;
  double etap = 1.0 / (Zpip + Zpim);
  double phip = etap * (rp[4] * Zpip + rm[4] * Zpim + rp[1] - rm[1]);
  double snnp = phip, snnm = phip;
  double vnp = rp[1] + Zpip * (rp[4] - snnp);
  double vnm = rm[1] - Zpim * (rm[4] - snnm);
  double sttp = rp[2] - gp * (rp[4] - snnp);
  double sttm = rm[2] - gm * (rm[4] - snnm);
  double szzp = rp[5] - gp * (rp[4] - snnp);
  double szzm = rm[5] - gm * (rm[4] - snnm);
  double etas = 1.0 / (Zsip + Zsim);
  double phis = etas * (rp[3] * Zsip + rm[3] * Zsim + rp[0] - rm[0]);
  double sntp = phis, sntm = phis;
  double vtp = rp[0] + Zsip * (rp[3] - sntp);
  double vtm = rm[0] - Zsim * (rm[3] - sntm);
  rot2_nt2xy(Fhp, n, vtp, vnp, sttp, sntp, snnp, szzp);
  rot2_nt2xy(Fhm, n, vtm, vnm, sttm, sntm, snnm, szzm);
}

// frictional_interface_mode3 (interfaces.f90:806-897); F0blk is the plus
// block's 9-component F0 vector (vx0..szz0) used for the normal prestress.
void frictional_mode3(oracle_domain& Dm, Ifc& I, int k, double* Fhm, double* Fhp, const double* Fm, const double* Fp,
                      const double* F0m, const double* F0p, const double n[2], double Zsm, double Zsp, double t,
                      double dt, const double* F0blk) {
  Fric& FR = I.fr;
  double r0p[3], r0m[3];
  rot3_xy2nt(F0p, n, r0p);
  rot3_xy2nt(F0m, n, r0m);
  double dp[3] = {Fp[0] - F0p[0], Fp[1] - F0p[1], Fp[2] - F0p[2]};
  double dm[3] = {Fm[0] - F0m[0], Fm[1] - F0m[1], Fm[2] - F0m[2]};
  double rp[3], rm[3];
  rot3_xy2nt(dp, n, rp);
  rot3_xy2nt(dm, n, rm);
  double Zsip = 1.0 / Zsp, Zsim = 1.0 / Zsm;
  double etas = 1.0 / (Zsip + Zsim);
  double phis = etas * (rp[2] * Zsip + rm[2] * Zsim + rp[0] - rm[0]);
  double S0 = r0p[2];
  double stt, snt, snn;
  xy2nt_mat(F0blk[3], F0blk[4], F0blk[6], stt, snt, snn, n);
  double p = 0.0;
  if (FR.tp_use) p = p + FR.tp_p0;
  double N0 = -snn - p;
  double phip = 0.0;
  solve_friction(Dm, FR, k, S0, N0, phip, phis, etas, I.x[k], I.y[k], t, dt);
  double snzp = FR.st[S_][k] - FR.st[S0_][k];
  double snzm = FR.st[S_][k] - FR.st[S0_][k];
  double vzp = rp[0] + Zsip * (rp[2] - snzp);
  double vzm = rm[0] - Zsim * (rm[2] - snzm);
  rot3_nt2xy(Fhp, n, vzp, rp[1], snzp);
  rot3_nt2xy(Fhm, n, vzm, rm[1], snzm);
  for (int l = 0; l < 3; ++l) { Fhp[l] = Fhp[l] + F0p[l]; Fhm[l] = Fhm[l] + F0m[l]; }
}

// frictional_interface_mode2 (interfaces.f90:900-1012).  The caller
// (interfaces.f90:795) passes (F0m, F0p) into dummies declared (F0p, F0m);
// this routine is written with the dummy names, and the caller reproduces
// the swap.
void frictional_mode2(oracle_domain& Dm, Ifc& I, int k, double* Fhm, double* Fhp, const double* Fm, const double* Fp,
                      const double* F0p, const double* F0m, const double n[2], double Zsm, double Zsp, double Zpm,
                      double Zpp, double gm, double gp, double t, double dt) {
  Fric& FR = I.fr;
  double r0p[6], r0m[6];
  rot2_xy2nt(F0p, n, r0p);
  rot2_xy2nt(F0m, n, r0m);
  double dp[6], dm[6];
  for (int l = 0; l < 6; ++l) { dp[l] = Fp[l] - F0p[l]; dm[l] = Fm[l] - F0m[l]; }
  double rp[6], rm[6];
  rot2_xy2nt(dp, n, rp);
  rot2_xy2nt(dm, n, rm);
  double Zsip = 1.0 / Zsp, Zsim = 1.0 / Zsm, Zpip = 1.0 / Zpp, Zpim = 1.0 / Zpm;
  double etas = 1.0 / (Zsip + Zsim);
  double phis = etas * (rp[3] * Zsip + rm[3] * Zsim + rp[0] - rm[0]);
  double etap = 1.0 / (Zpip + Zpim);
  double phip = etap * (rp[4] * Zpip + rm[4] * Zpim + rp[1] - rm[1]);
  double S0 = r0p[3];
  double p = 0.0;
  if (FR.tp_use) p = p + FR.tp_p0;
  double N0 = -r0p[4] - p;
  solve_friction(Dm, FR, k, S0, N0, phip, phis, etas, I.x[k], I.y[k], t, dt);
  double snnp = -(FR.st[N_][k] - FR.st[N0_][k]) / (1.0 - FR.skempton);
  double snnm = -(FR.st[N_][k] - FR.st[N0_][k]) / (1.0 - FR.skempton);
  double vnp = rp[1] + Zpip * (rp[4] - snnp);
  double vnm = rm[1] - Zpim * (rm[4] - snnm);
  double sttp = rp[2] - gp * (rp[4] - snnp);
  double sttm = rm[2] - gm * (rm[4] - snnm);
  double szzp = rp[5] - gp * (rp[4] - snnp);
  double szzm = rm[5] - gm * (rm[4] - snnm);
  double sntp = FR.st[S_][k] - FR.st[S0_][k];
  double sntm = FR.st[S_][k] - FR.st[S0_][k];
  double vtp = rp[0] + Zsip * (rp[3] - sntp);
  double vtm = rm[0] - Zsim * (rm[3] - sntm);
  rot2_nt2xy(Fhp, n, vtp, vnp, sttp, sntp, snnp, szzp);
  rot2_nt2xy(Fhm, n, vtm, vnm, sttm, sntm, snnm, szzm);
  for (int l = 0; l < 6; ++l) { Fhp[l] = Fhp[l] + F0p[l]; Fhm[l] = Fhm[l] + F0m[l]; }
}

// ---------------------------------------------------------------------------
// domain.f90:420-471 edges
// ---------------------------------------------------------------------------
void side_node(const Blk& B, int s, int k, int& i, int& j) {
  if (s == 0) { i = B.mgx; j = B.mgy + k; }
  else if (s == 1) { i = B.pgx; j = B.mgy + k; }
  else if (s == 2) { i = B.mgx + k; j = B.mgy; }
  else { i = B.mgx + k; j = B.pgy; }
}

void prepare_edges(oracle_domain& D) {
  const size_t NN = (size_t)D.nx * D.ny;
  for (auto& B : D.blk)
    for (int s = 0; s < 4; ++s) {
      Side& S = B.side[s];
      for (int k = 0; k < S.n; ++k) {
        int i, j;
        side_node(B, s, k, i, j);
        for (int l = 0; l < D.nF; ++l) S.F[k + (size_t)S.n * l] = D.F[G2(D, i, j) + NN * l];
      }
    }
}

void enforce_edge_conditions(oracle_domain& D, double Bdt) {
  const int nF = D.nF;
  double Fh[6], F[6], F0[6], n[2];
  for (auto& B : D.blk)
    for (int s = 0; s < 4; ++s) {
      Side& S = B.side[s];
      if (S.bc == FDMAP_BC_NONE) continue;
      for (int k = 0; k < S.n; ++k) {
        for (int l = 0; l < nF; ++l) { F[l] = S.F[k + (size_t)S.n * l]; F0[l] = S.F0[k + (size_t)S.n * l]; }
        n[0] = S.normal[k]; n[1] = S.normal[k + S.n];
        if (D.mode == 3) set_bc_mode3(Fh, F, F0, n, S.bc, S.M[k]);
        else set_bc_mode2(Fh, F, F0, n, S.bc, S.M[k], S.M[k + S.n], S.M[k + 2 * (size_t)S.n]);
        for (int l = 0; l < nF; ++l) S.Fhat[k + (size_t)S.n * l] = Fh[l];
      }
    }
  for (auto& I : D.ifc) {
    Blk& Bm = D.blk[I.im];
    Blk& Bp = D.blk[I.ip];
    Side& Sm = Bm.side[I.direction == 0 ? 1 : 3];
    Side& Sp = Bp.side[I.direction == 0 ? 0 : 2];
    int offm = I.direction == 0 ? Bm.mgy : Bm.mgx;
    int offp = I.direction == 0 ? Bp.mgy : Bp.mgx;
    int nI = I.p - I.m + 1;
    double Fm[6], Fp[6], F0m[6], F0p[6], Fhm[6], Fhp[6];
    const double* F0blk = Bp.F0;  // Fp%F0 (interfaces.f90:576)
    for (int k = 0; k < nI; ++k) {
      int km = I.m + k - offm, kp = I.m + k - offp;
      for (int l = 0; l < nF; ++l) {
        Fm[l] = Sm.F[km + (size_t)Sm.n * l]; Fp[l] = Sp.F[kp + (size_t)Sp.n * l];
        F0m[l] = Sm.F0[km + (size_t)Sm.n * l]; F0p[l] = Sp.F0[kp + (size_t)Sp.n * l];
      }
      n[0] = I.nhat[k]; n[1] = I.nhat[k + nI];
      double Zsm = Sm.M[km], Zsp = Sp.M[kp];
      if (I.coupling == FDMAP_COUPLING_LOCKED) {
        if (D.mode == 2) locked_mode2(Fhm, Fhp, Fm, Fp, n, Zsm, Zsp, Sm.M[km + Sm.n], Sp.M[kp + Sp.n],
                                      Sm.M[km + 2 * (size_t)Sm.n], Sp.M[kp + 2 * (size_t)Sp.n]);
        else locked_mode3(Fhm, Fhp, Fm, Fp, n, Zsm, Zsp);
      } else {
        if (D.mode == 2)
          frictional_mode2(D, I, k, Fhm, Fhp, Fm, Fp, /*dummy F0p <-*/ F0m, /*dummy F0m <-*/ F0p, n, Zsm, Zsp,
                           Sm.M[km + Sm.n], Sp.M[kp + Sp.n], Sm.M[km + 2 * (size_t)Sm.n], Sp.M[kp + 2 * (size_t)Sp.n],
                           D.t, Bdt);
        else frictional_mode3(D, I, k, Fhm, Fhp, Fm, Fp, F0m, F0p, n, Zsm, Zsp, D.t, Bdt, F0blk);
      }
      for (int l = 0; l < nF; ++l) {
        Sm.Fhat[km + (size_t)Sm.n * l] = Fhm[l];
        Sp.Fhat[kp + (size_t)Sp.n * l] = Fhp[l];
      }
    }
    if (I.coupling == FDMAP_COUPLING_FRICTION) set_rates_friction(I.fr, nI, D.t);
  }
}

// ---------------------------------------------------------------------------
// set_rates_SAT, SAT_term, split_sp (time_step.f90:754-851)
// ---------------------------------------------------------------------------
void set_rates_SAT(oracle_domain& D, Blk& B) {
  const size_t NN = (size_t)D.nx * D.ny;
  const int nF = D.nF;
  for (int s = 0; s < 4; ++s) {
    Side& S = B.side[s];
    for (int k = 0; k < S.n; ++k) {
      int i, j;
      side_node(B, s, k, i, j);
      size_t g = G2(D, i, j);
      double Ks = S.M[k + 3 * (size_t)S.n], Kp = S.M[k + 4 * (size_t)S.n];
      double diff[6];
      for (int l = 0; l < nF; ++l) diff[l] = S.Fhat[k + (size_t)S.n * l] - S.F[k + (size_t)S.n * l];
      if (D.mode == 3) {
        for (int l = 0; l < 3; ++l) D.DF[g + NN * l] = D.DF[g + NN * l] + Ks * diff[l];
      } else {
        double n[2] = {S.normal[k], S.normal[k + S.n]};
        double r[6], Fs[6], Fp[6];
        rot2_xy2nt(diff, n, r);
        rot2_nt2xy(Fs, n, r[0], 0.0, 0.0, r[3], 0.0, 0.0);
        rot2_nt2xy(Fp, n, 0.0, r[1], r[2], 0.0, r[4], r[5]);
        for (int l = 0; l < 6; ++l) D.DF[g + NN * l] = D.DF[g + NN * l] + Ks * Fs[l];
        for (int l = 0; l < 6; ++l) D.DF[g + NN * l] = D.DF[g + NN * l] + Kp * Fp[l];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// SBP rates (rates.f90:8-936, rates_heterogeneous.f90:8-917)
// ---------------------------------------------------------------------------
struct Ctx {
  oracle_domain* D;
  const RateDef* defs;
  int nr;
  size_t NN;
};

// material of node g for coefficient kind
inline double mat(const Ctx& c, const Blk& B, size_t g, int kind) {
  const oracle_domain& D = *c.D;
  if (D.het) return kind == 0 ? D.rho[g] : (kind == 1 ? D.G[g] : D.M[g]);
  return kind == 0 ? B.rho : (kind == 1 ? B.G : B.M);
}
inline double gam(const Ctx& c, const Blk& B, size_t g) { return c.D->het ? c.D->gamma[g] : B.gamma; }

// term t1 or t2 of rate r at neighbour point k (q direction if qdir) for center g
inline double term(const Ctx& c, const RateDef& rd, bool second, bool qdir, size_t g, size_t k, double gmm) {
  const oracle_domain& D = *c.D;
  int f = second ? rd.fb : rd.fa;
  const vec& met = qdir ? (second ? D.xr : D.yr) : (second ? D.xq : D.yq);
  double v = 0.5 * (met[k] + met[g]) * D.F[k + c.NN * f];
  if (second ? rd.gb : rd.ga) v = v * gmm;
  return v;
}

// sum of the flux (q: +t1 -t2, r: -t1 +t2) at point k, multiplied by sgn = +1/-1,
// appended term by term to `acc` (acc starts "empty" when first = true)
inline void add_flux(const Ctx& c, const RateDef& rd, bool qdir, int sgn, size_t g, size_t k, double gmm, double& acc,
                     bool& first) {
  int s1 = qdir ? +1 : -1;  // sign of t1 in the flux
  s1 *= sgn;
  if (rd.fa >= 0) {
    double t = term(c, rd, false, qdir, g, k, gmm);
    if (first) { acc = s1 > 0 ? t : -t; first = false; }
    else acc = s1 > 0 ? acc + t : acc - t;
  }
  if (rd.fb >= 0) {
    double t = term(c, rd, true, qdir, g, k, gmm);
    int s2 = -s1;
    if (first) { acc = s2 > 0 ? t : -t; first = false; }
    else acc = s2 > 0 ? acc + t : acc - t;
  }
}

// boundary-type scaling: (sum)*w/rho*Ji or (sum)*w*G*Ji or (sum)*w*M*Ji
inline double bscale(const Ctx& c, const Blk& B, size_t g, int kind, double sum, double w) {
  double m = mat(c, B, g, kind);
  double Ji = c.D->Ji[g];
  if (kind == 0) return sum * w / m * Ji;
  return sum * w * m * Ji;
}

// interior scaling (rates.f90:24-28, 400-405; rates_heterogeneous.f90:31,36,398,412,419)
inline double iscale(const Ctx& c, const Blk& B, size_t g, int kind, double sum, double DIs) {
  const oracle_domain& D = *c.D;
  double Ji = D.Ji[g];
  if (!D.het) {
    double a = kind == 0 ? DIs / B.rho : (kind == 1 ? DIs * B.G : DIs * B.M);
    return sum * a * Ji;
  }
  if (kind == 0) return sum * DIs * Ji / D.rho[g];
  if (D.mode == 3) return sum * DIs * D.G[g] * Ji;  // rates_h_interior_mode3 DF2, DF3
  return sum * DIs * Ji * (kind == 1 ? D.G[g] : D.M[g]);
}

void rates_interior(Ctx& c, const Blk& B, int mx, int px, int my, int py) {
  oracle_domain& D = *c.D;
  const Ops& op = D.op;
#pragma omp parallel for schedule(static)
  for (int j = my; j <= py; ++j)
    for (int i = mx; i <= px; ++i) {
      size_t g = G2(D, i, j);
      double gmm = gam(c, B, g);
      for (int s = 1; s <= op.pI; ++s) {
        size_t qp = G2(D, i + s, j), qm = G2(D, i - s, j), rp = G2(D, i, j + s), rm = G2(D, i, j - s);
        for (int r = 0; r < c.nr; ++r) {
          const RateDef& rd = c.defs[r];
          double acc = 0;
          bool first = true;
          add_flux(c, rd, true, +1, g, qp, gmm, acc, first);
          add_flux(c, rd, true, -1, g, qm, gmm, acc, first);
          add_flux(c, rd, false, +1, g, rp, gmm, acc, first);
          add_flux(c, rd, false, -1, g, rm, gmm, acc, first);
          D.DF[g + c.NN * r] = D.DF[g + c.NN * r] + iscale(c, B, g, rd.coef, acc, op.DI[s]);
        }
      }
    }
}

// one-sided weight and point for the q (qdir) or r direction at node i (or j)
// side: 0 = minus end (DL), 1 = plus end (DR)
inline void onesided(const Ops& op, int side, int idx, int m, int p, int s, double& w, int& pt) {
  if (side == 0) { w = op.DL[idx - m][s]; pt = m + s; }
  else { w = -op.DL[p - idx][s]; pt = p - s; }
}

void rates_boundary(Ctx& c, const Blk& B, int mx, int px, int my, int py, int qside, int rside) {
  // qside/rside: -1 central, 0 minus end, 1 plus end
  oracle_domain& D = *c.D;
  const Ops& op = D.op;
#pragma omp parallel for schedule(static)
  for (int j = my; j <= py; ++j)
    for (int i = mx; i <= px; ++i) {
      size_t g = G2(D, i, j);
      double gmm = gam(c, B, g);
      if (qside >= 0 && rside >= 0) {
        // corners: per s, q term then r term (rates.f90:243-377)
        for (int s = 0; s < op.nbnd; ++s) {
          double wq, wr;
          int pq, pr;
          onesided(op, qside, i, B.mgx, B.pgx, s, wq, pq);
          onesided(op, rside, j, B.mgy, B.pgy, s, wr, pr);
          size_t kq = G2(D, pq, j), kr = G2(D, i, pr);
          for (int r = 0; r < c.nr; ++r) {
            const RateDef& rd = c.defs[r];
            double acc = 0; bool first = true;
            add_flux(c, rd, true, +1, g, kq, gmm, acc, first);
            D.DF[g + c.NN * r] = D.DF[g + c.NN * r] + bscale(c, B, g, rd.coef, acc, wq);
          }
          for (int r = 0; r < c.nr; ++r) {
            const RateDef& rd = c.defs[r];
            double acc = 0; bool first = true;
            add_flux(c, rd, false, +1, g, kr, gmm, acc, first);
            D.DF[g + c.NN * r] = D.DF[g + c.NN * r] + bscale(c, B, g, rd.coef, acc, wr);
          }
        }
        continue;
      }
      bool qone = qside >= 0;  // L/R strip: q one-sided, r central; B/T: r one-sided, q central
      for (int s = 0; s < op.nbnd; ++s) {
        double w; int pt;
        if (qone) onesided(op, qside, i, B.mgx, B.pgx, s, w, pt);
        else onesided(op, rside, j, B.mgy, B.pgy, s, w, pt);
        size_t k = qone ? G2(D, pt, j) : G2(D, i, pt);
        for (int r = 0; r < c.nr; ++r) {
          const RateDef& rd = c.defs[r];
          double acc = 0; bool first = true;
          add_flux(c, rd, qone, +1, g, k, gmm, acc, first);
          D.DF[g + c.NN * r] = D.DF[g + c.NN * r] + bscale(c, B, g, rd.coef, acc, w);
        }
      }
      for (int s = 1; s <= op.pI; ++s) {
        size_t kp = qone ? G2(D, i, j + s) : G2(D, i + s, j);
        size_t km = qone ? G2(D, i, j - s) : G2(D, i - s, j);
        for (int r = 0; r < c.nr; ++r) {
          const RateDef& rd = c.defs[r];
          double acc = 0; bool first = true;
          add_flux(c, rd, !qone, +1, g, kp, gmm, acc, first);
          add_flux(c, rd, !qone, -1, g, km, gmm, acc, first);
          D.DF[g + c.NN * r] = D.DF[g + c.NN * r] + bscale(c, B, g, rd.coef, acc, op.DI[s]);
        }
      }
    }
}


// ---------------------------------------------------------------------------
// Perfectly matched layer, mode II (rates_interior_mode2_pml and
// rates_boundary_mode2_pml, rates.f90:2024-2619).  These replace the
// curvilinear split-form rates of a block with pmlx or pmly: Cartesian
// differences scaled by hxi = Ji*yr and hyi = Ji*xq taken at the first node of
// each region, and the auxiliary fields Wx, Wy.
// ---------------------------------------------------------------------------
// damping at a node (rates.f90:2065-2068): sigma, or sigma*|distance past the layer start|^n
inline void pml_damping(const Blk& B, double x, double y, double& sx, double& sy) {
  sx = B.pml_sigma;
  sy = B.pml_sigma;
  if (B.pml_n > 0.0) {
    sx = B.pml_sigma * std::pow(std::fabs(std::max(0.0, std::max(B.pml_mx - x, x - B.pml_px))), B.pml_n);
    sy = B.pml_sigma * std::pow(std::fabs(std::max(0.0, std::max(B.pml_my - y, y - B.pml_py))), B.pml_n);
  }
}

// auxiliary-field terms of one node (rates.f90:2070-2088): -W couplings into DF
// and the decay -(sigma + kappa)*W of DW
inline void pml_node_terms(oracle_domain& D, const Blk& B, size_t g, double sx, double sy) {
  const size_t NN = (size_t)D.nx * D.ny;
  vec& DF = D.DF;
  const double rho = B.rho, G = B.G, M = B.M, gamma = B.gamma;
  if (B.pmlx) {
    const vec& W = D.Wx;
    DF[g] = DF[g] - W[g + 2 * NN] / rho;
    DF[g + NN] = DF[g + NN] - W[g + 3 * NN] / rho;
    DF[g + 2 * NN] = DF[g + 2 * NN] - W[g] * M;
    DF[g + 3 * NN] = DF[g + 3 * NN] - W[g + NN] * G;
    DF[g + 4 * NN] = DF[g + 4 * NN] - W[g] * gamma * M;
    for (int l = 0; l < D.nF; ++l) D.DWx[g + l * NN] = D.DWx[g + l * NN] - (sx + B.pml_kappa) * W[g + l * NN];
  }
  if (B.pmly) {
    const vec& W = D.Wy;
    DF[g] = DF[g] - W[g + 3 * NN] / rho;
    DF[g + NN] = DF[g + NN] - W[g + 4 * NN] / rho;
    DF[g + 2 * NN] = DF[g + 2 * NN] - W[g + NN] * gamma * M;
    DF[g + 3 * NN] = DF[g + 3 * NN] - W[g] * G;
    DF[g + 4 * NN] = DF[g + 4 * NN] - W[g + NN] * M;
    for (int l = 0; l < D.nF; ++l) D.DWy[g + l * NN] = D.DWy[g + l * NN] - (sy + B.pml_kappa) * W[g + l * NN];
  }
}

// interior (rates.f90:2024-2129).  The reference runs s = 1..3 with DI(s) = 0
// beyond pI; those terms add exact zeros and are left out.
void rates_interior_pml(oracle_domain& D, const Blk& B, int mx, int px, int my, int py) {
  const size_t NN = (size_t)D.nx * D.ny;
  const Ops& op = D.op;
  double a[4], b[4], c[4];
  for (int s = 1; s <= op.pI; ++s) { a[s] = op.DI[s] / B.rho; b[s] = op.DI[s] * B.G; c[s] = op.DI[s] * B.M; }
  const double gamma = B.gamma;
  const size_t g0 = G2(D, mx, my);
  const double hxi = D.Ji[g0] * D.yr[g0], hyi = D.Ji[g0] * D.xq[g0];
  vec& DF = D.DF;
  const vec& F = D.F;
#pragma omp parallel for schedule(static)
  for (int j = my; j <= py; ++j)
    for (int i = mx; i <= px; ++i) {
      const size_t g = G2(D, i, j);
      double sx, sy;
      pml_damping(B, D.x[g], D.y[g], sx, sy);
      pml_node_terms(D, B, g, sx, sy);
      for (int s = 1; s <= op.pI; ++s) {
        const size_t ip = G2(D, i + s, j), im = G2(D, i - s, j), jp = G2(D, i, j + s), jm = G2(D, i, j - s);
        if (B.pmlx)
          for (int l = 0; l < D.nF; ++l)
            D.DWx[g + l * NN] = D.DWx[g + l * NN] + sx * hxi * (F[ip + l * NN] - F[im + l * NN]) * op.DI[s];
        if (B.pmly)
          for (int l = 0; l < D.nF; ++l)
            D.DWy[g + l * NN] = D.DWy[g + l * NN] + sy * hyi * (F[jp + l * NN] - F[jm + l * NN]) * op.DI[s];
        auto dx = [&](int l) { return F[ip + l * NN] - F[im + l * NN]; };
        auto dy = [&](int l) { return F[jp + l * NN] - F[jm + l * NN]; };
        DF[g] = DF[g] + (hxi * dx(2) + hyi * dy(3)) * a[s];
        DF[g + NN] = DF[g + NN] + (hxi * dx(3) + hyi * dy(4)) * a[s];
        DF[g + 2 * NN] = DF[g + 2 * NN] + (hxi * dx(0) + hyi * dy(1) * gamma) * c[s];
        DF[g + 3 * NN] = DF[g + 3 * NN] + (hxi * dx(1) + hyi * dy(0)) * b[s];
        DF[g + 4 * NN] = DF[g + 4 * NN] + (hxi * dx(0) * gamma + hyi * dy(1)) * c[s];
      }
    }
}

// q-direction (x) contribution of one stencil point: field values at point k
// with weight w (one-sided) or the difference F(k) - F(km) (central)
inline void pml_q_term(oracle_domain& D, const Blk& B, size_t g, double sx, double hxi, const double* f, double w) {
  const size_t NN = (size_t)D.nx * D.ny;
  vec& DF = D.DF;
  if (B.pmlx)
    for (int l = 0; l < D.nF; ++l) D.DWx[g + l * NN] = D.DWx[g + l * NN] + sx * hxi * f[l] * w;
  DF[g] = DF[g] + hxi * f[2] * w / B.rho;
  DF[g + NN] = DF[g + NN] + hxi * f[3] * w / B.rho;
  DF[g + 2 * NN] = DF[g + 2 * NN] + hxi * f[0] * w * B.M;
  DF[g + 3 * NN] = DF[g + 3 * NN] + hxi * f[1] * w * B.G;
  DF[g + 4 * NN] = DF[g + 4 * NN] + hxi * f[0] * w * B.M * B.gamma;
}
inline void pml_r_term(oracle_domain& D, const Blk& B, size_t g, double sy, double hyi, const double* f, double w) {
  const size_t NN = (size_t)D.nx * D.ny;
  vec& DF = D.DF;
  if (B.pmly)
    for (int l = 0; l < D.nF; ++l) D.DWy[g + l * NN] = D.DWy[g + l * NN] + sy * hyi * f[l] * w;
  DF[g] = DF[g] + hyi * f[3] * w / B.rho;
  DF[g + NN] = DF[g + NN] + hyi * f[4] * w / B.rho;
  DF[g + 2 * NN] = DF[g + 2 * NN] + hyi * f[1] * w * B.M * B.gamma;
  DF[g + 3 * NN] = DF[g + 3 * NN] + hyi * f[0] * w * B.G;
  DF[g + 4 * NN] = DF[g + 4 * NN] + hyi * f[1] * w * B.M;
}

// boundary regions (rates.f90:2131-2619); qside/rside: -1 central, 0 minus end, 1 plus end
void rates_boundary_pml(oracle_domain& D, const Blk& B, int mx, int px, int my, int py, int qside, int rside) {
  const size_t NN = (size_t)D.nx * D.ny;
  const Ops& op = D.op;
  const size_t g0 = G2(D, mx, my);
  const double hxi = D.Ji[g0] * D.yr[g0], hyi = D.Ji[g0] * D.xq[g0];
  const vec& F = D.F;
  const int nF = D.nF;
#pragma omp parallel for schedule(static)
  for (int j = my; j <= py; ++j)
    for (int i = mx; i <= px; ++i) {
      const size_t g = G2(D, i, j);
      double sx, sy;
      pml_damping(B, D.x[g], D.y[g], sx, sy);
      pml_node_terms(D, B, g, sx, sy);
      double f[6];
      auto load = [&](size_t k) { for (int l = 0; l < nF; ++l) f[l] = F[k + l * NN]; };
      auto diff = [&](size_t kp, size_t km) { for (int l = 0; l < nF; ++l) f[l] = F[kp + l * NN] - F[km + l * NN]; };
      if (qside >= 0 && rside >= 0) {
        // corners: one-sided in both directions, q then r for each s
        for (int s = 0; s < op.nbnd; ++s) {
          double wq, wr;
          int pq, pr;
          onesided(op, qside, i, B.mgx, B.pgx, s, wq, pq);
          onesided(op, rside, j, B.mgy, B.pgy, s, wr, pr);
          load(G2(D, pq, j));
          pml_q_term(D, B, g, sx, hxi, f, wq);
          load(G2(D, i, pr));
          pml_r_term(D, B, g, sy, hyi, f, wr);
        }
      } else if (qside >= 0) {
        // L / R: one-sided in q, then central in r
        for (int s = 0; s < op.nbnd; ++s) {
          double w;
          int pt;
          onesided(op, qside, i, B.mgx, B.pgx, s, w, pt);
          load(G2(D, pt, j));
          pml_q_term(D, B, g, sx, hxi, f, w);
        }
        for (int s = 1; s <= op.pI; ++s) {
          diff(G2(D, i, j + s), G2(D, i, j - s));
          pml_r_term(D, B, g, sy, hyi, f, op.DI[s]);
        }
      } else {
        // B / T: central in q, then one-sided in r
        for (int s = 1; s <= op.pI; ++s) {
          diff(G2(D, i + s, j), G2(D, i - s, j));
          pml_q_term(D, B, g, sx, hxi, f, op.DI[s]);
        }
        for (int s = 0; s < op.nbnd; ++s) {
          double w;
          int pt;
          onesided(op, rside, j, B.mgy, B.pgy, s, w, pt);
          load(G2(D, i, pt));
          pml_r_term(D, B, g, sy, hyi, f, w);
        }
      }
    }
}

// ---------------------------------------------------------------------------
// Rates with artificial dissipation (set_rates_dissipation, time_step.f90:555-751;
// rates_dissipation_*_mode2/3, rates.f90:939-2021; in a heterogeneous medium
// rates_h_dissipation_*, rates_heterogeneous.f90:920-1997).
// ---------------------------------------------------------------------------
// interior (rates.f90:939-999 mode III, 1397-1482 mode II; heterogeneous
// rates_heterogeneous.f90:920-978, 1376-1458: the node's rho, G, M scale the
// rate bracket; mode III as (T*DI(s)/rho)*Ji, mode II as (DI(s)/rho*T + d(s)*S)*Ji)
void rates_dissipation_interior(Ctx& c, const Blk& B, int mx, int px, int my, int py) {
  oracle_domain& D = *c.D;
  const Ops& op = D.op;
  const double Cd = B.Cdiss;
  double dco[4] = {0.0, 0.0, 0.0, 0.0};  // c(s) / d(s): AI(s)*Cdiss; zero beyond pI
  for (int s = 1; s <= op.pI; ++s) dco[s] = op.AI[s] * Cd;
  dco[0] = 2.0 * op.AI[0] * Cd;  // used for both the q and the r derivative
  const int nf = c.nr;             // mode II: fields 1..5 (szz is set by rates_szz)
#pragma omp parallel for schedule(static)
  for (int j = my; j <= py; ++j)
    for (int i = mx; i <= px; ++i) {
      size_t g = G2(D, i, j);
      double gmm = gam(c, B, g);
      for (int l = 0; l < nf; ++l) D.DF[g + c.NN * l] = D.DF[g + c.NN * l] + dco[0] * D.F[g + c.NN * l];
      for (int s = 1; s <= op.pI; ++s) {
        size_t qp = G2(D, i + s, j), qm = G2(D, i - s, j), rp = G2(D, i, j + s), rm = G2(D, i, j - s);
        for (int r = 0; r < c.nr; ++r) {
          const RateDef& rd = c.defs[r];
          double T = 0;
          bool first = true;
          add_flux(c, rd, true, +1, g, qp, gmm, T, first);
          add_flux(c, rd, true, -1, g, qm, gmm, T, first);
          add_flux(c, rd, false, +1, g, rp, gmm, T, first);
          add_flux(c, rd, false, -1, g, rm, gmm, T, first);
          size_t off = c.NN * r;
          double S = D.J[qp] * D.F[qp + off] + D.J[qm] * D.F[qm + off] + D.J[rp] * D.F[rp + off] +
                     D.J[rm] * D.F[rm + off];
          double Ji = D.Ji[g];
          if (D.het) {
            const double m = mat(c, B, g, rd.coef);
            if (D.mode == 3) {
              const double Tm = rd.coef == 0 ? T * op.DI[s] / m : T * op.DI[s] * m;
              D.DF[g + off] = D.DF[g + off] + Tm * Ji + dco[s] * Ji * S;
            } else {
              const double a = rd.coef == 0 ? op.DI[s] / m : op.DI[s] * m;
              D.DF[g + off] = D.DF[g + off] + (a * T + dco[s] * S) * Ji;
            }
            continue;
          }
          double a = rd.coef == 0 ? op.DI[s] / B.rho : (rd.coef == 1 ? op.DI[s] * B.G : op.DI[s] * B.M);
          if (D.mode == 3) D.DF[g + off] = D.DF[g + off] + T * a * Ji + dco[s] * Ji * S;
          else D.DF[g + off] = D.DF[g + off] + (a * T + dco[s] * S) * Ji;
        }
      }
    }
}

// one-sided dissipation weight at node idx: AL(s, idx-m) at the minus end,
// AR(-s, idx-p) = AL(s, p-idx) at the plus end
inline double onesided_diss(const Ops& op, int side, int idx, int m, int p, int s) {
  return side == 0 ? op.AL[idx - m][s] : op.AL[p - idx][s];
}

// boundary strips and corners (rates.f90:1002-1394 mode III, 1485-2021 mode II)
void rates_dissipation_boundary(Ctx& c, const Blk& B, int mx, int px, int my, int py, int qside, int rside) {
  oracle_domain& D = *c.D;
  const Ops& op = D.op;
  const double Cd = B.Cdiss;
  const int nF = D.nF;  // DF(i,j,:) covers every field (szz is overwritten by rates_szz)
#pragma omp parallel for schedule(static)
  for (int j = my; j <= py; ++j)
    for (int i = mx; i <= px; ++i) {
      size_t g = G2(D, i, j);
      double gmm = gam(c, B, g);
      const double Ji = D.Ji[g];
      auto rates_at = [&](bool qdir, size_t k, double w) {
        for (int r = 0; r < c.nr; ++r) {
          const RateDef& rd = c.defs[r];
          double acc = 0; bool first = true;
          add_flux(c, rd, qdir, +1, g, k, gmm, acc, first);
          D.DF[g + c.NN * r] = D.DF[g + c.NN * r] + bscale(c, B, g, rd.coef, acc, w);
        }
      };
      auto diss_at = [&](size_t k, double wa) {
        for (int l = 0; l < nF; ++l)
          D.DF[g + c.NN * l] = D.DF[g + c.NN * l] + D.J[k] * D.F[k + c.NN * l] * wa * Ji * Cd;
      };
      if (qside >= 0 && rside >= 0) {
        // corners: per s, q rates + dissipation, then r rates + dissipation; no AI(0) term
        for (int s = 0; s < op.nbnd; ++s) {
          double wq, wr;
          int pq, pr;
          onesided(op, qside, i, B.mgx, B.pgx, s, wq, pq);
          onesided(op, rside, j, B.mgy, B.pgy, s, wr, pr);
          size_t kq = G2(D, pq, j), kr = G2(D, i, pr);
          rates_at(true, kq, wq);
          diss_at(kq, onesided_diss(op, qside, i, B.mgx, B.pgx, s));
          rates_at(false, kr, wr);
          diss_at(kr, onesided_diss(op, rside, j, B.mgy, B.pgy, s));
        }
        continue;
      }
      bool qone = qside >= 0;
      for (int s = 0; s < op.nbnd; ++s) {
        double w; int pt;
        double wa;
        if (qone) { onesided(op, qside, i, B.mgx, B.pgx, s, w, pt); wa = onesided_diss(op, qside, i, B.mgx, B.pgx, s); }
        else { onesided(op, rside, j, B.mgy, B.pgy, s, w, pt); wa = onesided_diss(op, rside, j, B.mgy, B.pgy, s); }
        size_t k = qone ? G2(D, pt, j) : G2(D, i, pt);
        rates_at(qone, k, w);
        diss_at(k, wa);
      }
      for (int l = 0; l < nF; ++l) D.DF[g + c.NN * l] = D.DF[g + c.NN * l] + D.F[g + c.NN * l] * op.AI[0] * Cd;
      for (int s = 1; s <= op.pI; ++s) {
        size_t kp = qone ? G2(D, i, j + s) : G2(D, i + s, j);
        size_t km = qone ? G2(D, i, j - s) : G2(D, i - s, j);
        for (int r = 0; r < c.nr; ++r) {
          const RateDef& rd = c.defs[r];
          double acc = 0; bool first = true;
          add_flux(c, rd, !qone, +1, g, kp, gmm, acc, first);
          add_flux(c, rd, !qone, -1, g, km, gmm, acc, first);
          D.DF[g + c.NN * r] = D.DF[g + c.NN * r] + bscale(c, B, g, rd.coef, acc, op.DI[s]);
        }
        for (int l = 0; l < nF; ++l)
          D.DF[g + c.NN * l] =
              D.DF[g + c.NN * l] + (D.J[kp] * D.F[kp + c.NN * l] + D.J[km] * D.F[km + c.NN * l]) * op.AI[s] * Ji * Cd;
      }
    }
}

// set_rates (time_step.f90:318-552) for one block
void set_rates(oracle_domain& D, const Blk& B) {
  Ctx c{&D, D.mode == 2 ? kMode2 : kMode3, D.mode == 2 ? 5 : 3, (size_t)D.nx * D.ny};
  int nbst = D.op.nbst;
  int mix = B.mgx + nbst, pix = B.pgx - nbst, miy = B.mgy + nbst, piy = B.pgy - nbst;
  if (B.Cdiss > 0.0) {
    // set_rates_dissipation: the same regions, dissipative rate routines
    rates_dissipation_interior(c, B, mix, pix, miy, piy);
    rates_dissipation_boundary(c, B, B.mgx, mix - 1, miy, piy, 0, -1);        // L
    rates_dissipation_boundary(c, B, pix + 1, B.pgx, miy, piy, 1, -1);        // R
    rates_dissipation_boundary(c, B, mix, pix, B.mgy, miy - 1, -1, 0);        // B
    rates_dissipation_boundary(c, B, mix, pix, piy + 1, B.pgy, -1, 1);        // T
    rates_dissipation_boundary(c, B, B.mgx, mix - 1, B.mgy, miy - 1, 0, 0);   // LB
    rates_dissipation_boundary(c, B, pix + 1, B.pgx, B.mgy, miy - 1, 1, 0);   // RB
    rates_dissipation_boundary(c, B, B.mgx, mix - 1, piy + 1, B.pgy, 0, 1);   // LT
    rates_dissipation_boundary(c, B, pix + 1, B.pgx, piy + 1, B.pgy, 1, 1);   // RT
  } else if (D.mode == 2 && (B.pmlx || B.pmly)) {
    // set_rates, PML branch (time_step.f90:354-420)
    rates_interior_pml(D, B, mix, pix, miy, piy);
    rates_boundary_pml(D, B, B.mgx, mix - 1, miy, piy, 0, -1);        // L
    rates_boundary_pml(D, B, pix + 1, B.pgx, miy, piy, 1, -1);        // R
    rates_boundary_pml(D, B, mix, pix, B.mgy, miy - 1, -1, 0);        // B
    rates_boundary_pml(D, B, mix, pix, piy + 1, B.pgy, -1, 1);        // T
    rates_boundary_pml(D, B, B.mgx, mix - 1, B.mgy, miy - 1, 0, 0);   // LB
    rates_boundary_pml(D, B, pix + 1, B.pgx, B.mgy, miy - 1, 1, 0);   // RB
    rates_boundary_pml(D, B, B.mgx, mix - 1, piy + 1, B.pgy, 0, 1);   // LT
    rates_boundary_pml(D, B, pix + 1, B.pgx, piy + 1, B.pgy, 1, 1);   // RT
  } else {
    rates_interior(c, B, mix, pix, miy, piy);
    rates_boundary(c, B, B.mgx, mix - 1, miy, piy, 0, -1);        // L
    rates_boundary(c, B, pix + 1, B.pgx, miy, piy, 1, -1);        // R
    rates_boundary(c, B, mix, pix, B.mgy, miy - 1, -1, 0);        // B
    rates_boundary(c, B, mix, pix, piy + 1, B.pgy, -1, 1);        // T
    rates_boundary(c, B, B.mgx, mix - 1, B.mgy, miy - 1, 0, 0);   // LB
    rates_boundary(c, B, pix + 1, B.pgx, B.mgy, miy - 1, 1, 0);   // RB
    rates_boundary(c, B, B.mgx, mix - 1, piy + 1, B.pgy, 0, 1);   // LT
    rates_boundary(c, B, pix + 1, B.pgx, piy + 1, B.pgy, 1, 1);   // RT
  }
  if (D.mode == 2) {
    // rates_szz / rates_h_szz (rates.f90:920-936, rates_heterogeneous.f90:901-917)
    size_t NN = c.NN;
    for (int j = B.mgy; j <= B.pgy; ++j)
      for (int i = B.mgx; i <= B.pgx; ++i) {
        size_t g = G2(D, i, j);
        double nu = D.het ? D.nu[g] : B.nu;
        D.DF[g + NN * 5] = nu * (D.DF[g + NN * 2] + D.DF[g + NN * 4]);
      }
  }
}

// singular_source (source.f90:327-406)
void singular_source(int i, int i0, double h, double a, double& d) {
  double beta = (1.0 - 2.0 * a) / 4.0 + 0.25;
  double gam_ = (2.0 * a - 1.0) / 16.0;
  double gap = (2.0 * a + 1.0) / 16.0;
  if (i == i0 - 2) d = (-gam_) / h;
  else if (i == i0 - 1) d = (beta + 3.0 * gam_ - gap) / h;
  else if (i == i0) d = (1.0 - a - 2.0 * beta - 3.0 * gam_ + 3.0 * gap) / h;
  else if (i == i0 + 1) d = (a + beta + gam_ - 3.0 * gap) / h;
  else if (i == i0 + 2) d = (gap) / h;
  else d = 0.0;
}

// set_source (source.f90:147-252) for one block; point source and gravity
void point_source(oracle_domain& D, const Blk& B, double t, double pi);

// diagonal SBP norm with unit spacing over a block's n nodes (Hnorm, fd.f90:14-39)
double hnorm(const Ops& op, int n, int k) {
  if (k < op.nbst) return op.HL[k];
  if (k > n - 1 - op.nbst) return op.HL[n - 1 - k];
  return 1.0;
}

// energy_block / energy_interior (energy.f90:9-96): the block's homogeneous
// material, the step-start fields, the Jacobian and the norm in both directions
void energy_interior(oracle_domain& D) {
  const size_t NN = (size_t)D.nx * D.ny;
  const vec& F = D.F;
  double Esum = 0.0;
  for (int b = 0; b < D.nblocks; ++b) {
    const Blk& B = D.blk[b];
    const int nxb = B.pgx - B.mgx + 1, nyb = B.pgy - B.mgy + 1;
    double E = 0.0;
    if (D.mode == 2) {
      const double lambda = B.M - 2.0 * B.G;
      const double v1 = 0.5 * B.rho, v2 = 0.5 * B.G, v3 = 0.25 * B.G;
      const double v4 = -0.25 * B.G * (lambda / (3.0 * lambda + 2.0 * B.G));
      for (int j = B.mgy; j <= B.pgy; ++j)
        for (int i = B.mgx; i <= B.pgx; ++i) {
          const size_t g = G2(D, i, j);
          const double f1 = F[g], f2 = F[g + NN], f3 = F[g + 2 * NN], f4 = F[g + 3 * NN], f5 = F[g + 4 * NN],
                       f6 = F[g + 5 * NN];
          E = E + hnorm(D.op, nxb, i - B.mgx) * hnorm(D.op, nyb, j - B.mgy) * D.J[g] *
                      (v1 * (f1 * f1 + f2 * f2) + v2 * (f4 * f4) + v3 * (f3 * f3 + f5 * f5 + f6 * f6) +
                       v4 * ((f3 + f5 + f6) * (f3 + f5 + f6)));
        }
    } else {
      for (int j = B.mgy; j <= B.pgy; ++j)
        for (int i = B.mgx; i <= B.pgx; ++i) {
          const size_t g = G2(D, i, j);
          const double f1 = F[g], f2 = F[g + NN], f3 = F[g + 2 * NN];
          E = E + 0.5 * D.J[g] * (B.rho * (f1 * f1) + (f2 * f2 + f3 * f3) / B.G) * hnorm(D.op, nxb, i - B.mgx) *
                      hnorm(D.op, nyb, j - B.mgy);
        }
    }
    D.Etot[b] = E;
    Esum = Esum + E;
  }
  D.Etot[D.nblocks] = Esum;
}

void set_source(oracle_domain& D, const Blk& B, double t) {
  const fdmap_source& S = D.src;
  size_t NN = (size_t)D.nx * D.ny;
  if (S.use_gravity) {
    for (int j = B.mgy; j <= B.pgy; ++j)
      for (int i = B.mgx; i <= B.pgx; ++i) {
        size_t g = G2(D, i, j);
        if (D.mode == 2) { D.DF[g] = D.DF[g] + S.gx; D.DF[g + NN] = D.DF[g + NN] + S.gy; }
        else D.DF[g] = D.DF[g] + S.gz;
      }
  }
  // a point source outside the block ends set_source for it, skipping the
  // forcing terms below as well (source.f90:200-206)
  if (S.use_singular && !B.src_ok) return;
  const double pi = 3.14159265358979323846264338327950288;
  if (S.use_singular) point_source(D, B, t, pi);
  // problem = 'Forcing': tsunami forcing, mode III only (source.f90:299-312)
  if (S.gauss_forcing && D.mode == 3) {
    for (int j = B.mgy; j <= B.pgy; ++j)
      for (int i = B.mgx; i <= B.pgx; ++i) {
        size_t g = G2(D, i, j);
        double x = D.x[g], y = D.y[g];
        double u = (t - 4.0 * S.gauss_sigmat) / S.gauss_sigmat;
        D.DF[g] = D.DF[g] + S.gauss_amp *
                                std::exp(-0.5 * ((x / S.gauss_sigma) * (x / S.gauss_sigma)) -
                                         0.5 * ((y / S.gauss_sigma) * (y / S.gauss_sigma))) *
                                std::exp(-0.5 * (u * u)) / (S.gauss_sigmat * std::sqrt(2.0 * pi));
      }
  }
  // forcing from file, interpolated linearly in time (source.f90:315-322)
  if (D.frc) {
    double w_old = (D.frc_t_new - t) / (D.frc_t_new - D.frc_t_old);
    double w_new = 1.0 - w_old;
    for (int l = 0; l < D.nF; ++l)
      for (int j = B.mgy; j <= B.pgy; ++j)
        for (int i = B.mgx; i <= B.pgx; ++i) {
          size_t g = G2(D, i, j) + NN * l;
          D.DF[g] = D.DF[g] + w_old * D.frc_old[g] + w_new * D.frc_new[g];
        }
  }
}

// reads the next (nx,ny,nF) forcing frame; values past the end of the file read as zero
void read_forcing_frame(oracle_domain& D, vec& frame) {
  frame.assign((size_t)D.nx * D.ny * D.nF, 0.0);
  size_t got = std::fread(frame.data(), sizeof(double), frame.size(), D.frc);
  (void)got;
}

// load_forcing (source.f90:467-502), at the start of every step
void load_forcing(oracle_domain& D, double t, double dt) {
  D.frc_t_old = t;
  D.frc_t_new = t + dt;
  D.frc_old = D.frc_new;
  read_forcing_frame(D, D.frc_new);
}

// singular point force / moment tensor (source.f90:185-252)
void point_source(oracle_domain& D, const Blk& B, double t, double pi) {
  const fdmap_source& S = D.src;
  size_t NN = (size_t)D.nx * D.ny;
  double A;
  double tc = t - S.t_center;
  switch (S.stf) {
    case FDMAP_STF_RAMP: A = std::max(std::min(tc / S.t_duration, 1.0), 0.0); break;
    case FDMAP_STF_SINUSOID: A = std::sin(2.0 * pi * tc / S.t_duration); break;
    case FDMAP_STF_GAUSSIAN: A = std::exp(-0.5 * (tc * tc) / (S.t_duration * S.t_duration)); break;
    default:
      A = (1.0 - 2.0 * (pi * pi) * (tc * tc) / (S.t_duration * S.t_duration)) *
          std::exp(-(pi * pi) * (tc * tc) / (S.t_duration * S.t_duration));
      break;
  }
  for (int j = std::max(B.mgy, B.src_j0 - 2); j <= std::min(B.pgy, B.src_j0 + 2); ++j)
    for (int i = std::max(B.mgx, B.src_i0 - 2); i <= std::min(B.pgx, B.src_i0 + 2); ++i) {
      double dx, dy;
      singular_source(i, B.src_i0, B.src_hx, B.src_ax, dx);
      singular_source(j, B.src_j0, B.src_hy, B.src_ay, dy);
      size_t g = G2(D, i, j);
      if (D.mode == 2) {
        D.DF[g] = D.DF[g] + A * S.Fx * dx * dy / B.rho;
        D.DF[g + NN] = D.DF[g + NN] + A * S.Fy * dx * dy / B.rho;
        D.DF[g + 2 * NN] = D.DF[g + 2 * NN] - A * S.Mxx * dx * dy;
        D.DF[g + 3 * NN] = D.DF[g + 3 * NN] - A * S.Mxy * dx * dy;
        D.DF[g + 4 * NN] = D.DF[g + 4 * NN] - A * S.Myy * dx * dy;
      } else {
        D.DF[g] = D.DF[g] + A * S.Fz * dx * dy / B.rho;
        D.DF[g + NN] = D.DF[g + NN] - A * S.Mzx * dx * dy;
        D.DF[g + 2 * NN] = D.DF[g + 2 * NN] - A * S.Mzy * dx * dy;
      }
    }
}

void set_rates_all(oracle_domain& D) {
  for (auto& B : D.blk) set_rates_SAT(D, B);
  for (auto& B : D.blk) set_rates(D, B);
  // set_rates_displacement (fields.f90:1245-1258): DU += F(:, :, 1:nU)
  if (!D.U.empty()) {
    for (size_t q = 0; q < D.DU.size(); ++q) D.DU[q] = D.DU[q] + D.F[q];  // U(:,:,l) pairs with F(:,:,l)
  }
  for (auto& B : D.blk) set_source(D, B, D.t);
  // set_rates_boundary (fields.f90:1261-1276): DU += Fhat(:, 1:nU) on every side
  const int nU = D.mode == 2 ? 2 : 1;
  for (auto& B : D.blk)
    for (auto& S : B.side)
      for (int c = 0; c < nU; ++c)
        for (int k = 0; k < S.n; ++k) {
          size_t q = (size_t)k + (size_t)S.n * c;
          S.DU[q] = S.DU[q] + S.Fhat[q];
        }
}

void scale_rates_all(oracle_domain& D, double A) {
  size_t n = D.DF.size();
#pragma omp parallel for schedule(static)
  for (long long q = 0; q < (long long)n; ++q) D.DF[q] = A * D.DF[q];
  // scale_rates_interior (fields.f90:1060-1078): the PML rates too
  for (vec* W : {&D.DWx, &D.DWy})
    for (double& v : *W) v = A * v;
  for (auto& I : D.ifc)
    if (I.coupling == FDMAP_COUPLING_FRICTION) scale_rates_friction(I.fr, A);
  for (double& v : D.DU) v = A * v;  // scale_rates_interior: body displacement rates
  // scale_rates_boundary (fields.f90:1083-1097): boundary displacement rates
  for (auto& B : D.blk)
    for (auto& S : B.side)
      for (double& v : S.DU) v = A * v;
}

void update_fields_all(oracle_domain& D, double Bdt) {
  size_t n = D.F.size();
#pragma omp parallel for schedule(static)
  for (long long q = 0; q < (long long)n; ++q) D.F[q] = D.F[q] + Bdt * D.DF[q];
  // update_fields_interior (fields.f90:1168-1186): the PML fields too
  for (size_t q = 0; q < D.Wx.size(); ++q) D.Wx[q] = D.Wx[q] + Bdt * D.DWx[q];
  for (size_t q = 0; q < D.Wy.size(); ++q) D.Wy[q] = D.Wy[q] + Bdt * D.DWy[q];
  for (auto& I : D.ifc)
    if (I.coupling == FDMAP_COUPLING_FRICTION) update_fields_friction(I.fr, Bdt);
  for (size_t q = 0; q < D.U.size(); ++q) D.U[q] = D.U[q] + Bdt * D.DU[q];  // update_fields_interior
  // update_fields_boundary (fields.f90:1189-1204)
  for (auto& B : D.blk)
    for (auto& S : B.side)
      for (size_t q = 0; q < S.U.size(); ++q) S.U[q] = S.U[q] + Bdt * S.DU[q];
}

// exchange_edge (mpi_routines2d.f90:168-208) for a partitioned run: the
// caller's callback replaces the edge values of every interface side that
// lives on another rank with that rank's values (oracle_set_iface_edge)
int exchange_edges(oracle_domain& D) {
  if (D.owned.empty()) return FDMAP_OK;
  if (!D.exchange) return FDMAP_ERR_INVALID_ARG;
  const int rc = D.exchange(D.exchange_user, D.xstage);
  D.xstage++;
  return rc ? FDMAP_ERR_IO : FDMAP_OK;
}

// side and side-local offset of interface I's minus (side 0) or plus (side 1) nodes
Side& iface_side(oracle_domain& D, const Ifc& I, int side, int& off) {
  Blk& B = D.blk[side == 0 ? I.im : I.ip];
  off = I.m - (I.direction == 0 ? B.mgy : B.mgx);
  return B.side[side == 0 ? (I.direction == 0 ? 1 : 3) : (I.direction == 0 ? 0 : 2)];
}

}  // namespace

extern "C" {

oracle_domain* oracle_create(const fdmap_desc* d) {
  if (!d || (d->mode != 2 && d->mode != 3)) return nullptr;
  oracle_domain* o = new (std::nothrow) oracle_domain();
  if (!o) return nullptr;
  o->mode = d->mode;
  o->nF = d->nF;
  o->nx = d->nx;
  o->ny = d->ny;
  o->nblocks = d->nblocks;
  o->nifaces = d->nifaces;
  o->het = d->heterogeneous;
  o->newton_fail = 0;
  o->newton_stop = 0;
  o->t = d->t0;
  if (!make_ops(d->fd_method, &o->op) || !make_rk(d->rk_order, &o->rk)) { delete o; return nullptr; }
  size_t NN = (size_t)d->nx * d->ny;
  o->F = copyv(d->F, NN * d->nF);
  o->DF = copyv(d->DF, NN * d->nF);
  o->x = copyv(d->x, NN); o->y = copyv(d->y, NN);
  o->xq = copyv(d->xq, NN); o->xr = copyv(d->xr, NN); o->yq = copyv(d->yq, NN); o->yr = copyv(d->yr, NN);
  o->Ji = copyv(d->Ji, NN);
  if (d->J) o->J = copyv(d->J, NN);
  if (o->het) {
    o->rho = copyv(d->rho, NN); o->G = copyv(d->G, NN); o->M = copyv(d->M, NN);
    o->gamma = copyv(d->gamma, NN); o->nu = copyv(d->nu, NN);
  }
  o->src = d->src;
  if (d->displacement) {
    const size_t nU = d->mode == 2 ? 2 : 1;
    o->U.assign(NN * nU, 0.0);
    o->DU.assign(NN * nU, 1e40);
  }
  if (d->peak) {
    o->pgv.assign(NN, 0.0);
    o->pga.assign(NN, 0.0);
  }
  o->energy = d->energy_balance != 0;
  o->Etot.assign((size_t)d->nblocks + 1, 1e40);  // BF%Etot = 1d40 until the first stage 1
  if (d->src.forcing_filename) {
    // init_forcing_from_file (source.f90:409-448): frame 0 into the new frame
    o->frc = std::fopen(d->src.forcing_filename, "rb");
    if (!o->frc) { delete o; return nullptr; }
    read_forcing_frame(*o, o->frc_new);
    o->frc_old.assign(o->frc_new.size(), 0.0);
  }
  o->blk.resize(d->nblocks);
  for (int b = 0; b < d->nblocks; ++b) {
    const fdmap_block& fb = d->blocks[b];
    Blk& B = o->blk[b];
    B.mgx = fb.mgx; B.pgx = fb.pgx; B.mgy = fb.mgy; B.pgy = fb.pgy;
    B.rho = fb.rho; B.G = fb.G; B.M = fb.M; B.gamma = fb.gamma; B.nu = fb.nu;
    for (int q = 0; q < 9; ++q) B.F0[q] = fb.F0[q];
    B.src_ok = fb.src_ok; B.src_i0 = fb.src_i0; B.src_j0 = fb.src_j0;
    B.src_hx = fb.src_hx; B.src_hy = fb.src_hy; B.src_ax = fb.src_ax; B.src_ay = fb.src_ay;
    B.Cdiss = fb.Cdiss;
    if (B.Cdiss > 0.0 && !d->J) { delete o; return nullptr; }
    B.pmlx = fb.pmlx != 0; B.pmly = fb.pmly != 0;
    B.pml_n = fb.pml_n; B.pml_sigma = fb.pml_sigma; B.pml_kappa = fb.pml_kappa;
    B.pml_mx = fb.pml_mx; B.pml_px = fb.pml_px; B.pml_my = fb.pml_my; B.pml_py = fb.pml_py;
    // Wx / Wy and their rates start at zero (fields.f90:203-210)
    if (B.pmlx && o->Wx.empty()) { o->Wx.assign(NN * d->nF, 0.0); o->DWx.assign(NN * d->nF, 0.0); }
    if (B.pmly && o->Wy.empty()) { o->Wy.assign(NN * d->nF, 0.0); o->DWy.assign(NN * d->nF, 0.0); }
    for (int s = 0; s < 4; ++s) {
      const fdmap_side& fs = fb.side[s];
      Side& S = B.side[s];
      S.bc = fs.bc; S.n = fs.n;
      if (d->mode == 3 && S.bc != FDMAP_BC_NONE && S.bc != FDMAP_BC_ABSORBING && S.bc != FDMAP_BC_FREE &&
          S.bc != FDMAP_BC_RIGID) { delete o; return nullptr; }
      S.M = copyv(fs.M, (size_t)fs.n * 5);
      S.F0 = copyv(fs.F0, (size_t)fs.n * d->nF);
      S.normal = copyv(fs.normal, (size_t)fs.n * 2);
      S.F.assign((size_t)fs.n * d->nF, 1e40);
      S.Fhat.assign((size_t)fs.n * d->nF, 1e40);
      // init_fields_side (fields.f90:854-856): U = 0, DU = 1e40
      const int nU = d->mode == 2 ? 2 : 1;
      S.U.assign((size_t)fs.n * nU, 0.0);
      S.DU.assign((size_t)fs.n * nU, 1e40);
    }
  }
  o->ifc.resize(d->nifaces);
  for (int k = 0; k < d->nifaces; ++k) {
    const fdmap_iface& fi = d->ifaces[k];
    Ifc& I = o->ifc[k];
    I.direction = fi.direction; I.im = fi.iblockm; I.ip = fi.iblockp; I.m = fi.m; I.p = fi.p;
    I.coupling = fi.coupling;
    size_t n = (size_t)(fi.p - fi.m + 1);
    I.nhat = copyv(fi.nhat, 2 * n); I.x = copyv(fi.x, n); I.y = copyv(fi.y, n);
    if (I.coupling != FDMAP_COUPLING_FRICTION) continue;
    const fdmap_friction& ff = fi.fr;
    Fric& FR = I.fr;
    FR.law = ff.law; FR.reg = ff.reg; FR.rup_field = ff.rup_field; FR.force = ff.force;
    FR.ld_shape = ff.ld_shape; FR.tp_use = ff.tp_use;
    FR.rup_threshold = ff.rup_threshold; FR.angle = ff.angle; FR.xlockm = ff.xlockm; FR.xlockp = ff.xlockp;
    FR.flock = ff.flock; FR.skempton = ff.skempton;
    FR.kn_c0 = ff.kn_c0; FR.kn_fd = ff.kn_fd; FR.kn_dfdx = ff.kn_dfdx; FR.kn_vL = ff.kn_vL; FR.kn_vR = ff.kn_vR;
    FR.kn_xL = ff.kn_xL; FR.kn_xR = ff.kn_xR; FR.kn_tmax = ff.kn_tmax;
    FR.ld_S = ff.ld_S; FR.ld_N = ff.ld_N; FR.ld_T = ff.ld_T; FR.ld_R = ff.ld_R; FR.ld_x0 = ff.ld_x0; FR.ld_y0 = ff.ld_y0;
    FR.tp_p0 = ff.tp_p0;
    FR.a = copyv(ff.a, n); FR.b = copyv(ff.b, n); FR.V0 = copyv(ff.V0, n); FR.f0 = copyv(ff.f0, n);
    FR.L = copyv(ff.L, n); FR.fw = copyv(ff.fw, n); FR.Vw = copyv(ff.Vw, n);
    FR.c0 = copyv(ff.c0, n); FR.fs = copyv(ff.fs, n); FR.fd = copyv(ff.fd, n); FR.Dc = copyv(ff.Dc, n);
    FR.bsS0 = copyv(ff.bsS0, n); FR.bsN0 = copyv(ff.bsN0, n);
    double* const st[FDMAP_FAULT_NFIELDS] = {ff.D, ff.Psi, ff.DPsi, ff.trup, ff.V, ff.O, ff.S, ff.N, ff.S0,
                                             ff.N0, ff.Ds, ff.Dn, ff.DDs, ff.DDn, ff.W, ff.DW, ff.Nreg, ff.DNreg};
    for (int f = 0; f < FDMAP_FAULT_NFIELDS; ++f) {
      if (!st[f]) { delete o; return nullptr; }
      FR.st[f] = copyv(st[f], n);
    }
    bool rs = FR.law >= FDMAP_FR_SL;
    if ((rs && (FR.a.empty() || FR.b.empty() || FR.V0.empty() || FR.f0.empty() || FR.L.empty() || FR.fw.empty() ||
                FR.Vw.empty())) ||
        (FR.law == FDMAP_FR_SW && (FR.c0.empty() || FR.fs.empty() || FR.fd.empty() || FR.Dc.empty()))) {
      delete o;
      return nullptr;
    }
  }
  return o;
}

void oracle_destroy(oracle_domain* o) { delete o; }

int oracle_init_edges(oracle_domain* o, double t) {
  if (!o) return FDMAP_ERR_INVALID_ARG;
  o->t = t;
  prepare_edges(*o);
  if (int rc = exchange_edges(*o)) return rc;
  enforce_edge_conditions(*o, 0.0);
  return FDMAP_OK;
}

int oracle_time_step(oracle_domain* o, double t0, double dt, int final_step) {
  if (!o) return FDMAP_ERR_INVALID_ARG;
  oracle_domain& D = *o;
  D.t = t0;
  if (D.frc) load_forcing(D, t0, dt);
  for (int stage = 1; stage <= D.rk.nstage; ++stage) {
    scale_rates_all(D, D.rk.A[stage - 1]);
    prepare_edges(D);
    if (int rc = exchange_edges(D)) return rc;
    enforce_edge_conditions(D, D.rk.B[stage - 1] * dt);
    set_rates_all(D);
    if (stage == 1 && D.tap)
      for (auto& I : D.ifc)
        if (I.coupling == FDMAP_COUPLING_FRICTION)
          for (int f = 0; f < FDMAP_FAULT_NFIELDS; ++f) I.fr.tap[f] = I.fr.st[f];
    if (stage == 1 && D.energy) energy_interior(D);
    if (stage == 1 && !D.pgv.empty()) {
      // update_fields_peak (fields.f90:1136-1164), stage 1 only
      const size_t NN = (size_t)D.nx * D.ny;
      for (size_t g = 0; g < NN; ++g) {
        if (D.mode == 2) {
          D.pgv[g] = std::max(D.pgv[g], std::sqrt(D.F[g] * D.F[g] + D.F[g + NN] * D.F[g + NN]));
          D.pga[g] = std::max(D.pga[g], std::sqrt(D.DF[g] * D.DF[g] + D.DF[g + NN] * D.DF[g + NN]));
        } else {
          D.pgv[g] = std::max(D.pgv[g], std::fabs(D.F[g]));
          D.pga[g] = std::max(D.pga[g], std::fabs(D.DF[g]));
        }
      }
    }
    if (final_step) return FDMAP_OK;
    D.t = t0 + D.rk.C[stage] * dt;
    update_fields_all(D, D.rk.B[stage - 1] * dt);
  }
  return FDMAP_OK;
}

int oracle_run(oracle_domain* o, double t_start, double dt, int n_first, int n_last, int nt) {
  if (!o) return FDMAP_ERR_INVALID_ARG;
  for (int n = n_first; n <= n_last; ++n) {
    int rc = oracle_time_step(o, t_start + (double)(n - 1) * dt, dt, n == nt);
    if (rc) return rc;
  }
  return FDMAP_OK;
}

int oracle_get_fields(const oracle_domain* o, double* F, double* DF) {
  if (!o) return FDMAP_ERR_INVALID_ARG;
  if (F) std::memcpy(F, o->F.data(), o->F.size() * sizeof(double));
  if (DF) std::memcpy(DF, o->DF.data(), o->DF.size() * sizeof(double));
  return FDMAP_OK;
}

int oracle_set_fields(oracle_domain* o, const double* F, const double* DF) {
  if (!o) return FDMAP_ERR_INVALID_ARG;
  if (F) std::memcpy(o->F.data(), F, o->F.size() * sizeof(double));
  if (DF) std::memcpy(o->DF.data(), DF, o->DF.size() * sizeof(double));
  return FDMAP_OK;
}

int oracle_get_fault(const oracle_domain* o, int iface, int field, double* out) {
  if (!o || iface < 0 || iface >= o->nifaces || field < 0 || field >= FDMAP_FAULT_NFIELDS || !out)
    return FDMAP_ERR_INVALID_ARG;
  const Ifc& I = o->ifc[iface];
  if (I.coupling != FDMAP_COUPLING_FRICTION) return FDMAP_ERR_INVALID_ARG;
  std::memcpy(out, I.fr.st[field].data(), I.fr.st[field].size() * sizeof(double));
  return FDMAP_OK;
}

int oracle_get_fhat(const oracle_domain* o, int b, int s, double* out) {
  if (!o || b < 0 || b >= o->nblocks || s < 0 || s > 3 || !out) return FDMAP_ERR_INVALID_ARG;
  const Side& S = o->blk[b].side[s];
  std::memcpy(out, S.Fhat.data(), S.Fhat.size() * sizeof(double));
  return FDMAP_OK;
}

long long oracle_newton_failures(const oracle_domain* o) { return o ? o->newton_fail : -1; }

long long oracle_newton_stops(const oracle_domain* o) { return o ? o->newton_stop : -1; }

int oracle_set_owned(oracle_domain* o, const int* owned) {
  if (!o || !owned) return FDMAP_ERR_INVALID_ARG;
  o->owned.assign(owned, owned + o->nblocks);
  // the other ranks' blocks hold NaN here: any read of them that is not an
  // exchanged edge value spreads NaN into the result
  const size_t NN = (size_t)o->nx * o->ny;
  const double nan = std::nan("");
  for (int b = 0; b < o->nblocks; ++b) {
    if (owned[b]) continue;
    const Blk& B = o->blk[b];
    for (int l = 0; l < o->nF; ++l)
      for (int j = B.mgy; j <= B.pgy; ++j)
        for (int i = B.mgx; i <= B.pgx; ++i) {
          o->F[G2(*o, i, j) + NN * l] = nan;
          o->DF[G2(*o, i, j) + NN * l] = nan;
        }
  }
  return FDMAP_OK;
}

int oracle_set_exchange(oracle_domain* o, int (*fn)(void*, long long), void* user) {
  if (!o) return FDMAP_ERR_INVALID_ARG;
  o->exchange = fn;
  o->exchange_user = user;
  return FDMAP_OK;
}

int oracle_get_iface_edge(oracle_domain* o, int iface, int side, double* out) {
  if (!o || iface < 0 || iface >= o->nifaces || side < 0 || side > 1 || !out) return FDMAP_ERR_INVALID_ARG;
  const Ifc& I = o->ifc[iface];
  int off = 0;
  const Side& S = iface_side(*o, I, side, off);
  const int n = I.p - I.m + 1;
  for (int l = 0; l < o->nF; ++l)
    for (int k = 0; k < n; ++k) out[(size_t)l * n + k] = S.F[off + k + (size_t)S.n * l];
  return FDMAP_OK;
}

int oracle_set_iface_edge(oracle_domain* o, int iface, int side, const double* in) {
  if (!o || iface < 0 || iface >= o->nifaces || side < 0 || side > 1 || !in) return FDMAP_ERR_INVALID_ARG;
  const Ifc& I = o->ifc[iface];
  int off = 0;
  Side& S = iface_side(*o, I, side, off);
  const int n = I.p - I.m + 1;
  for (int l = 0; l < o->nF; ++l)
    for (int k = 0; k < n; ++k) S.F[off + k + (size_t)S.n * l] = in[(size_t)l * n + k];
  return FDMAP_OK;
}

int oracle_set_tap(oracle_domain* o, int on) {
  if (!o) return FDMAP_ERR_INVALID_ARG;
  o->tap = on != 0;
  return FDMAP_OK;
}

int oracle_get_fault_tap(const oracle_domain* o, int iface, int field, double* out) {
  if (!o || iface < 0 || iface >= o->nifaces || field < 0 || field >= FDMAP_FAULT_NFIELDS || !out)
    return FDMAP_ERR_INVALID_ARG;
  const Ifc& I = o->ifc[iface];
  if (I.coupling != FDMAP_COUPLING_FRICTION || I.fr.tap[field].empty()) return FDMAP_ERR_INVALID_ARG;
  std::memcpy(out, I.fr.tap[field].data(), I.fr.tap[field].size() * sizeof(double));
  return FDMAP_OK;
}

int oracle_set_fault(oracle_domain* o, int iface, int field, const double* in) {
  if (!o || iface < 0 || iface >= o->nifaces || field < 0 || field >= FDMAP_FAULT_NFIELDS || !in)
    return FDMAP_ERR_INVALID_ARG;
  Ifc& I = o->ifc[iface];
  if (I.coupling != FDMAP_COUPLING_FRICTION) return FDMAP_ERR_INVALID_ARG;
  std::memcpy(I.fr.st[field].data(), in, I.fr.st[field].size() * sizeof(double));
  return FDMAP_OK;
}

// boundary displacement U and its rate DU of side s of block b, (n, nU) each (either may be NULL)
int oracle_set_side_u(oracle_domain* o, int b, int s, const double* U, const double* DU) {
  if (!o || b < 0 || b >= o->nblocks || s < 0 || s > 3) return -1;
  Side& S = o->blk[b].side[s];
  if (U) std::copy(U, U + S.U.size(), S.U.begin());
  if (DU) std::copy(DU, DU + S.DU.size(), S.DU.begin());
  return 0;
}

// body displacement U, DU (nx,ny,nU) and peak motion pgv, pga (nx,ny); any may be NULL, -1 when absent
int oracle_set_body_extras(oracle_domain* o, const double* U, const double* DU, const double* pgv, const double* pga) {
  if (!o) return -1;
  if ((U || DU) && o->U.empty()) return -1;
  if ((pgv || pga) && o->pgv.empty()) return -1;
  if (U) std::copy(U, U + o->U.size(), o->U.begin());
  if (DU) std::copy(DU, DU + o->DU.size(), o->DU.begin());
  if (pgv) std::copy(pgv, pgv + o->pgv.size(), o->pgv.begin());
  if (pga) std::copy(pga, pga + o->pga.size(), o->pga.begin());
  return 0;
}

// PML field Wx (which = 0) or Wy (1) from the global (nx,ny,nF) layout; -1 when the domain has none
int oracle_set_pml(oracle_domain* o, int which, const double* in) {
  if (!o || !in || which < 0 || which > 1) return -1;
  vec& W = which == 0 ? o->Wx : o->Wy;
  if (W.empty()) return -1;
  std::copy(in, in + W.size(), W.begin());
  return 0;
}

int oracle_set_newton_tolerance(oracle_domain* o, double scale) {
  if (!o || !(scale > 0.0)) return FDMAP_ERR_INVALID_ARG;
  o->newton_tol_scale = scale;
  return FDMAP_OK;
}

int oracle_set_newton_limit(oracle_domain* o, int imax) {
  if (!o || imax < 1) return FDMAP_ERR_INVALID_ARG;
  o->newton_imax = imax;
  return FDMAP_OK;
}

// body displacement U, DU (nx,ny,nU) and peak motion pgv, pga (nx,ny); any may be NULL, -1 when absent
int oracle_get_body_extras(const oracle_domain* o, double* U, double* DU, double* pgv, double* pga) {
  if (!o) return -1;
  if ((U || DU) && o->U.empty()) return -1;
  if ((pgv || pga) && o->pgv.empty()) return -1;
  if (U) std::copy(o->U.begin(), o->U.end(), U);
  if (DU) std::copy(o->DU.begin(), o->DU.end(), DU);
  if (pgv) std::copy(o->pgv.begin(), o->pgv.end(), pgv);
  if (pga) std::copy(o->pga.begin(), o->pga.end(), pga);
  return 0;
}

// boundary displacement U and its rate DU of side s of block b, (n, nU) each (either may be NULL)
int oracle_get_side_u(const oracle_domain* o, int b, int s, double* U, double* DU) {
  if (!o || b < 0 || b >= o->nblocks || s < 0 || s > 3) return -1;
  const Side& S = o->blk[b].side[s];
  if (U) std::copy(S.U.begin(), S.U.end(), U);
  if (DU) std::copy(S.DU.begin(), S.DU.end(), DU);
  return 0;
}

// mechanical energy of every block and their sum, as of the last stage 1 (energy_balance = T)
int oracle_get_energy(const oracle_domain* o, double* E) {
  if (!o || !E || !o->energy) return -1;
  std::copy(o->Etot.begin(), o->Etot.end(), E);
  return 0;
}

// PML field Wx (which = 0) or Wy (1) in the global (nx,ny,nF) layout; zeros when not allocated
int oracle_get_pml(const oracle_domain* o, int which, double* out) {
  if (!o || !out || which < 0 || which > 1) return -1;
  const vec& W = which == 0 ? o->Wx : o->Wy;
  size_t n = (size_t)o->nx * o->ny * o->nF;
  if (W.empty()) std::fill(out, out + n, 0.0);
  else std::copy(W.begin(), W.end(), out);
  return 0;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

}  // extern "C"
