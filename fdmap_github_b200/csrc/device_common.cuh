// Device-side data layout and the point-wise physics shared by the kernels:
// rotations (geometry.f90:285-336), characteristic boundary conditions
// (boundaries.f90:155-377), locked and frictional interface solves
// (interfaces.f90:676-1012) and friction laws (friction.f90:555-1506).
//
// HBM layout.  Each block is stored separately with a row pitch that is a
// multiple of 32 doubles (256 B), so every row starts on a 256-byte boundary
// and a warp reading 32 consecutive nodes touches exactly two 128-byte lines:
//   field l, block-local node (i, j):  base + l*plane + j*pitch + i,
//   plane = pitch*ny.
// Fields are ping-ponged (F[0], F[1]) between RK stages because the fused
// stencil reads neighbours of a node while other CTAs already write the
// updated state; rates DF are updated in place (only the node itself reads
// its own rate).
#pragma once

#include <cuda.h>

#include <cstdint>

#include "fdmap_desc.h"

namespace fdmap {

constexpr int MAX_BLOCKS = 16;
constexpr int MAX_IFACES = 32;

struct DevSide {
  int bc, n;
  int cov_lo, cov_hi;  // side-local nodes [cov_lo, cov_hi) whose hat variables come from an interface
  double* M;           // (n,5)
  double* F0;          // (n,nF)
  double* nrm;         // (n,2)
  double* Fhat;        // (n,nF)
  double* U;           // (n,nU) boundary displacement (bnd_fields, fields.f90:14-15)
  double* DU;          // (n,nU) its rate
  double* Utap;        // (n,nU) U at the start of stage 1 (the output point)
};

struct DevBlock {
  int nx, ny, pitch;
  long long plane;
  double* F[3];                        // F[0], F[1] ping-pong; F[2] the first stage's values near the
                                       // block edges in a two-stage pass (NULL when pairs are off)
  double* DF;
  double* DFalt;                       // second rate buffer of two-stage passes (NULL when pairs are off)
  double *xq, *xr, *yq, *yr, *Ji;      // (pitch, ny)
  double *rho, *G, *M, *gamma, *nu;    // heterogeneous only
  double rho_b, G_b, M_b, gamma_b, nu_b;
  double rinv_b;                       // 1/rho_b
  double coef[4][3];                   // homogeneous interior weights DI(s)/rho, DI(s)*G, DI(s)*M
                                       // (a, b, c of rates_interior_mode2, rates.f90:400-405)
  double F0v[9];
  DevSide side[4];
  int src_ok, src_i0, src_j0;          // block-local source indices
  double src_wx[5], src_wy[5];         // singular_source weights d for i0-2..i0+2
  double Cdiss;                        // scaled artificial dissipation (0: none)
  double* J;                           // Jacobian plane (dissipative blocks only)
  int pml;                             // perfectly matched layer: bit 0 Wx (pmlx), bit 1 Wy (pmly); 0 = none
  double pml_kappa;                    // frequency shift
  const double* pml_h;                 // [3][3][2] hxi, hyi of each region (q, r: 0 minus end, 1 plus end, 2 central)
  const double* pml_s;                 // 2 planes: damping sx, sy at every node
  double *Wx, *DWx, *Wy, *DWy;         // auxiliary fields and rates, nF planes each (NULL when off)
  const double* gforce;                // tsunami forcing: amp*exp(-(x/sigma)^2/2 - (y/sigma)^2/2) per node, or NULL
  const double* frc_old;               // forcing from file: frames at the step's start and end,
  const double* frc_new;               //   nF planes each (NULL when no forcing file)
  double *U, *DU, *Utap;               // body displacement, its rate, its stage-1 value: nU planes (displacement = T)
  double *pgv, *pga;                   // peak ground velocity / acceleration planes (peak = T)
  const double *Hx, *Hy;               // diagonal SBP norm along i and j (energy_balance = T)
  int tile_begin;                      // first stencil tile of this block
  int tiles_x;
  long long march_unit_begin;          // first row-group unit of this block (march kernel)
  long long pair_unit_begin;           // first row-group unit of this block (two-stage march)
};

// per-interface friction storage: st[f*n + k] for the 18 FDMAP_FAULT_* fields,
// par[p*n + k] for the per-node parameters below
enum { PAR_A = 0, PAR_B, PAR_V0, PAR_F0, PAR_L, PAR_FW, PAR_VW, PAR_C0, PAR_FS, PAR_FD, PAR_DC, PAR_BSS0, PAR_BSN0, PAR_N };

struct DevFriction {
  int law, reg, rup_field, force, ld_shape, tp_use, has_bsS0, has_bsN0;
  double rup_threshold, angle, xlockm, xlockp, flock, skempton;
  double cos_angle, sin_angle;  // cos/sin of the fault angle, evaluated once on the host
  double kn_c0, kn_fd, kn_dfdx, kn_vL, kn_vR, kn_xL, kn_xR, kn_tmax;
  double ld_S, ld_N, ld_T, ld_R, ld_x0, ld_y0, tp_p0;
  double* st;
  double* par;
  double* st_out;  // stage-1 snapshot of the 18 fields at the output point (outputs open), else null
};

// per-interface-node impedance terms, evaluated once on the host (each is a
// correctly rounded division, so the values equal the in-kernel ones):
// 1/Zs-, 1/Zs+, 1/Zp-, 1/Zp+, etas = 1/(1/Zs+ + 1/Zs-), etap = 1/(1/Zp+ + 1/Zp-)
enum { IC_ZSIM = 0, IC_ZSIP, IC_ZPIM, IC_ZPIP, IC_ETAS, IC_ETAP, IC_N };

struct DevIface {
  int direction, im, ip, m, p, n, coupling;
  int offm, offp;  // side-local index of global node m on the minus / plus side
  double* icoef;   // (n, IC_N)
  double* nhat;    // (n,2)
  double *x, *y;   // (n)
  DevFriction fr;
  // Block-aligned partition (a side's block lives on another GPU): the edge
  // values of that side arrive each stage in rem_m / rem_p ([l*n + k], the
  // nF fields of the interface nodes); the local side's edge values are
  // packed into `send` for the peer.  All NULL in an unpartitioned domain.
  const double* rem_m;
  const double* rem_p;
  double* send;
};

// Device layout of every field array: PADL doubles of front padding (so that
// halo boxes may start before column 0) and PADTAIL doubles of slack after
// the last row of each plane.
constexpr int PADL = 32;
constexpr int PADTAIL = 192;

// Register cap of the boundary kernels (interface solves, closure strips).
// They run on a side stream beside a resident interior kernel, and a warp
// takes its registers from one of the SM's four sub-partitions (16K
// registers each), not from the SM as a whole: beside a march CTA of 512
// threads at 96 registers (12K per sub-partition) only a warp of at most 128
// registers a thread fits.  Uncapped (166 and 196 registers) they waited for
// the interior kernel to finish.
constexpr int BOUNDARY_REGS = 128;

// Timeline of the stage kernels (fdmap_gpu_trace): one record of three words
// per CTA, (kind | SM << 8 | CTA << 16, start ns, end ns) on %globaltimer
enum { TRACE_MARCH = 1, TRACE_CLOSURE = 2, TRACE_EDGE = 3, TRACE_TILED = 4, TRACE_PAIR = 5, TRACE_BAND = 6 };
struct TraceBuf {
  unsigned long long* rec;  // NULL: tracing off
  unsigned int* n;
  unsigned int cap;
};

struct DevDomain {
  TraceBuf trace;
  int mode, nF, nblocks, nifaces, het;
  int nbst, nbnd, pI;
  double DI[4];     // DI[s], s = 1..pI (fd_coeff.f90)
  double DL[6][9];  // DL[r][s]: weight of point s for the derivative at boundary node r
  double AI[4];     // artificial dissipation AI(s), s = 0..pI (fd_coeff.f90)
  double AL[6][9];  // AL[r][s]: dissipation weight of point s at boundary node r (AR mirrors it)
  DevBlock blk[MAX_BLOCKS];
  DevIface ifc[MAX_IFACES];
  // closure strips of every block (bottom, top, left, right): thread offsets
  long long cstart[4 * MAX_BLOCKS + 1];
  // edge bands of width nbw = nbst + pI (second stage of a two-stage pass), same order
  long long bstart[4 * MAX_BLOCKS + 1];
  int nbw;
  // interface work segments (one thread per interface node)
  int nseg;
  int seg_kind[4 * MAX_BLOCKS + MAX_IFACES];   // 0 = BC side, 1 = interface
  int seg_a[4 * MAX_BLOCKS + MAX_IFACES];      // block (BC) or interface index
  int seg_b[4 * MAX_BLOCKS + MAX_IFACES];      // side (BC)
  int seg_start[4 * MAX_BLOCKS + MAX_IFACES + 1];
  fdmap_source src;
  unsigned long long* status;  // [0] Newton failures (first attempt), [1] flags (bit 1: a bounded wait gave up),
                               // [2] scratch of fdmap_gpu_check_finite, [3] Newton retries that failed too
  int newton_imax;             // Newton iteration limit (friction.f90:924 imax = 99; lowered only by tests)
  const double* energy;        // [nblocks + 1] stage-1 mechanical energy (energy_balance = T), or NULL
};

// TMA descriptors of every block, passed by value as a __grid_constant__ parameter
// (single domain) or read from device memory (batched instances)
struct TmapSet {
  CUtensorMap F[MAX_BLOCKS][2];    // rate fields, box {WH, MR, NR}
  CUtensorMap F6[MAX_BLOCKS][2];   // szz plane (mode II), box {MW, MR, 1}
  CUtensorMap DF[MAX_BLOCKS];      // rates, box {MW, MR, NR}
  CUtensorMap MH[MAX_BLOCKS];      // yr, xr, box {WH, MR, 2}
  CUtensorMap MC[MAX_BLOCKS];      // yq, xq, Ji, box {MW, MR, 3}
  CUtensorMap HT[MAX_BLOCKS];      // heterogeneous material, box {MW, MR, NH}
  CUtensorMap JH[MAX_BLOCKS];      // Jacobian of dissipative blocks, box {WH, MR, 1}
};

// Batched launches: CTAs [begin[k], begin[k+1]) serve instance k.  Returns
// the instance of CTA `cta` (binary search, uniform across the CTA).
__device__ __forceinline__ int batch_instance(const int* __restrict__ begin, int ninst, int cta) {
  int lo = 0, hi = ninst - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (begin[mid] <= cta) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Step clock kept on the device so that a captured CUDA graph can be replayed
// step after step: step n starts at t0 = t_start + (n-1)*dt (main.f90:176).
struct TimeState {
  double t_start, dt;
  long long n;
};

struct StageArgs {
  double A;      // RK coefficient A(stage): rates are scaled by it first
  double Bdt;    // B(stage)*dt: state update weight
  double t;      // stage time (when ts == nullptr)
  int in, out;   // F buffer read / written
  int scale;     // scale rates by A (0 for the initial edge solve)
  int update;    // update the state (0 on the final step and the initial solve)
  const TimeState* ts;  // device step clock (graph replays), or nullptr
  double C;      // RK C(stage-1): stage time = t0 + C*dt
  int tap;       // stage 1 with outputs open: interface kernels write their output snapshot
  double t0, dt; // step start and length (when ts == nullptr)
  int first;     // stage 1 (update_fields_peak)
  int dfr, dfw;  // rate buffer read (scaled by A) and written: 0 DF, 1 DFalt (two-stage passes)
};

// Stage time t0 + C*dt with t0 = t_start + (n-1)*dt, rounded exactly as the
// host (and the reference) evaluate it: no fused multiply-add.
__device__ __forceinline__ double stage_time(const StageArgs& a) {
  if (!a.ts) return a.t;
  const double t0 = __dadd_rn(a.ts->t_start, __dmul_rn((double)(a.ts->n - 1), a.ts->dt));
  return __dadd_rn(t0, __dmul_rn(a.C, a.ts->dt));
}

// The step's window [t0, t0 + dt] (load_forcing, source.f90:486-487)
__device__ __forceinline__ void step_window(const StageArgs& a, double& t_old, double& t_new) {
  if (!a.ts) {
    t_old = a.t0;
    t_new = __dadd_rn(a.t0, a.dt);
    return;
  }
  t_old = __dadd_rn(a.ts->t_start, __dmul_rn((double)(a.ts->n - 1), a.ts->dt));
  t_new = __dadd_rn(t_old, a.ts->dt);
}

// ---------------------------------------------------------------------------
// rotations (geometry.f90:285-336; fields.f90:1297-1356)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void xy2nt_vec(double wx, double wy, double& wt, double& wn, double n0, double n1) {
  wt = n1 * wx - n0 * wy;
  wn = n0 * wx + n1 * wy;
}
__device__ __forceinline__ void nt2xy_vec(double& wx, double& wy, double wt, double wn, double n0, double n1) {
  wx = n1 * wt + n0 * wn;
  wy = -n0 * wt + n1 * wn;
}
__device__ __forceinline__ void xy2nt_mat(double wxx, double wxy, double wyy, double& wtt, double& wnt, double& wnn,
                                          double n0, double n1) {
  wtt = -(2.0 * n0 * n1 * wxy) + (n1 * n1) * wxx + (n0 * n0) * wyy;
  wnt = n0 * n1 * (wxx - wyy) + ((n1 * n1) - (n0 * n0)) * wxy;
  wnn = 2.0 * n0 * n1 * wxy + (n0 * n0) * wxx + (n1 * n1) * wyy;
}
__device__ __forceinline__ void nt2xy_mat(double& wxx, double& wxy, double& wyy, double wtt, double wnt, double wnn,
                                          double n0, double n1) {
  wxx = 2.0 * n0 * n1 * wnt + (n1 * n1) * wtt + (n0 * n0) * wnn;
  wxy = -(n0 * n1 * (wtt - wnn)) + ((n1 * n1) - (n0 * n0)) * wnt;
  wyy = -(2.0 * n0 * n1 * wnt) + (n0 * n0) * wtt + (n1 * n1) * wnn;
}
__device__ __forceinline__ void rot2_xy2nt(const double* F, double n0, double n1, double* o) {
  xy2nt_vec(F[0], F[1], o[0], o[1], n0, n1);
  xy2nt_mat(F[2], F[3], F[4], o[2], o[3], o[4], n0, n1);
  o[5] = F[5];
}
__device__ __forceinline__ void rot2_nt2xy(double* F, double n0, double n1, double vt, double vn, double stt,
                                           double snt, double snn, double szz) {
  nt2xy_vec(F[0], F[1], vt, vn, n0, n1);
  nt2xy_mat(F[2], F[3], F[4], stt, snt, snn, n0, n1);
  F[5] = szz;
}
__device__ __forceinline__ void rot3_xy2nt(const double* F, double n0, double n1, double* o) {
  o[0] = F[0];
  xy2nt_vec(F[1], F[2], o[1], o[2], n0, n1);
}
__device__ __forceinline__ void rot3_nt2xy(double* F, double n0, double n1, double vz, double stz, double snz) {
  F[0] = vz;
  nt2xy_vec(F[1], F[2], stz, snz, n0, n1);
}

__device__ __forceinline__ double fsign(double a, double b) { return copysign(fabs(a), b); }

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// one timeline record for the calling CTA (call from one thread)
__device__ __forceinline__ void trace_record(const TraceBuf& T, int kind, unsigned long long t0) {
  if (!T.rec) return;
  unsigned sm;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
  const unsigned k = atomicAdd(T.n, 1u);
  if (k >= T.cap) return;
  unsigned long long* r = T.rec + 3 * (size_t)k;
  r[0] = (unsigned long long)kind | ((unsigned long long)sm << 8) | ((unsigned long long)blockIdx.x << 16);
  r[1] = t0;
  r[2] = globaltimer_ns();
}

}  // namespace fdmap
