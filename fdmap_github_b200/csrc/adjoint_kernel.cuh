// Discrete adjoint of one low-storage RK stage of the mode III heterogeneous
// SBP-SAT update (rates_h_interior_mode3 / rates_h_boundary_mode3,
// rates_heterogeneous.f90:8-372, with set_rates_SAT / set_bc_mode3,
// time_step.f90:754-851, boundaries.f90:155-235).
//
// Forward stage s (forward numbering, u = fields, q = rate register):
//   q_s = A_s q_{s-1} + R(u_{s-1}, t_s),   u_s = u_{s-1} + B_s dt q_s,
// with R(u) = L(rho, G) u + f(t) linear in u.  Its adjoint, run for
// s = nstage..1 with qbar' = A_{s+1} qbar_{s+1} carried between stages:
//   qs   = qbar' + B_s dt ubar            (adjoint of the update)
//   ubar = ubar + L^T qs                  (adjoint of the rates)
//   grad += (dR/dm)(u_{s-1})^T qs         (material gradient, rho and G)
//   qbar' = A_s qs
//
// L^T is applied as a gather: input node (i, j) collects, from every output
// node whose stencil holds it, that node's weight times its adjoint rate.  An
// output node's q-direction stencil depends only on its column (one-sided DL
// rows within nbst of the left/right side, DR = -reverse(DL) on the right,
// central DI elsewhere) and its r-direction stencil only on its row, so the
// candidate output nodes of an input node are enumerated per direction.
#pragma once

#include "march_kernel.cuh"
#include "stencil_kernel.cuh"

namespace fdmap {

struct AdjStage {
  double A, Bdt;                  // RK A(s), B(s)*dt of the forward stage
  int s, nstage;                  // forward stage index (0-based), stages per step
  const double* ub_in;            // ubar (3 planes, block layout)
  const double* qp_in;            // qbar' carried from the later stage
  double* ub_out;
  double* qp_out;
  const double* store;            // forward stage inputs u_{s-1}: store + (rel*nstage + s)*stride
  long long stride;
  const long long* rel;           // device: step index within the recomputed segment
  double* grho;                   // dJ/drho, dJ/dG (1 plane each), accumulated
  double* gG;
  int blk;                        // block whose nodes this stage covers
};

// SAT of one outer side at an edge node in mode III (set_bc_mode3 + SAT_term):
//   r0 = vz - vz0,  r2 = n0 (sxz - sxz0) + n1 (syz - syz0),
//   e = E(Zs) (r0, r2),   DF += Ks * (e0, n0 e2, n1 e2).
// E (absorbing) = -1/2 [[1, 1/Zs], [Zs, 1]], (free) [[0, -1/Zs], [0, -1]],
// (rigid) [[-1, 0], [-Zs, 0]].  Adds the transposed action on lam to ubar and
// the derivatives through Zs = rho*cs, Ks = cs*geo (cs = sqrt(G/rho)) to the gradient.
__device__ __forceinline__ void sat_adjoint(int bc, double Zs, double Ks, double n0, double n1, const double* lam,
                                            const double* ust, const double* F0, double rho, double G, double* ub,
                                            double* grho, double* gG) {
  const double a0 = Ks * lam[0], a2 = Ks * (n0 * lam[1] + n1 * lam[2]);
  const double r0 = ust[0] - F0[0], r2 = n0 * (ust[1] - F0[1]) + n1 * (ust[2] - F0[2]);
  double p0, p2, e0, e2, de0, de2;  // E^T a;  E r;  dE/dZs r
  if (bc == FDMAP_BC_ABSORBING) {
    p0 = -0.5 * a0 - 0.5 * Zs * a2;
    p2 = -0.5 * a0 / Zs - 0.5 * a2;
    e0 = -0.5 * r0 - 0.5 * r2 / Zs;
    e2 = -0.5 * Zs * r0 - 0.5 * r2;
    de0 = 0.5 * r2 / (Zs * Zs);
    de2 = -0.5 * r0;
  } else if (bc == FDMAP_BC_FREE) {
    p0 = 0.0;
    p2 = -a0 / Zs - a2;
    e0 = -r2 / Zs;
    e2 = -r2;
    de0 = r2 / (Zs * Zs);
    de2 = 0.0;
  } else {  // rigid
    p0 = -a0 - Zs * a2;
    p2 = 0.0;
    e0 = -r0;
    e2 = -Zs * r0;
    de0 = 0.0;
    de2 = -r0;
  }
  ub[0] += p0;
  ub[1] += n0 * p2;
  ub[2] += n1 * p2;
  const double lt = n0 * lam[1] + n1 * lam[2];
  const double gK = lam[0] * e0 + lt * e2;          // d/dKs of lam . SAT
  const double gZ = Ks * (lam[0] * de0 + lt * de2);  // d/dZs
  // Zs = sqrt(rho G), Ks = geo sqrt(G / rho)
  *grho += 0.5 * (gZ * Zs - gK * Ks) / rho;
  *gG += 0.5 * (gZ * Zs + gK * Ks) / G;
}

// One direction of one node of the adjoint stage through the cache hierarchy
// (closures, sides, corners): part 0 gathers the q direction, the q half of
// the node's own volume rates and the SAT of the L / R sides; part 1 the r
// direction, its half of the volume rates and the SAT of the B / T sides.
// The two partial sums are added by the caller.
template <int PI_>
__device__ __forceinline__ void adj_node_part(const DevDomain& D, const AdjStage& p, int i, int j, int part,
                                              double* acc, double* phi, double& grho, double& gG) {
  constexpr int nbnd = nbnd_of(PI_);
  const DevBlock& B = D.blk[p.blk];
  const int nx = B.nx, ny = B.ny, nbst = D.nbst;
  const long long pitch = B.pitch, plane = B.plane;
  const long long c = (long long)j * pitch + i;
  const double* __restrict__ ub = p.ub_in;
  const double* __restrict__ qp = p.qp_in;
  auto qs = [&](long long k, int f) { return qp[f * plane + k] + p.Bdt * ub[f * plane + k]; };
  acc[0] = acc[1] = acc[2] = 0.0;
  phi[0] = phi[1] = phi[2] = 0.0;
  grho = gG = 0.0;
  const double* __restrict__ ust = p.store + ((*p.rel) * p.nstage + p.s) * p.stride;
  if (part == 0) {
    const double yrc = B.yr[c], xrc = B.xr[c];
    // output node k (same row) whose q-stencil weights this node by W
    auto gather_q = [&](int ic, double W) {
      const long long k = (long long)j * pitch + ic;
      const double Y = 0.5 * (B.yr[k] + yrc), X = 0.5 * (B.xr[k] + xrc);
      const double wj = W * B.Ji[k], g = B.G[k];
      const double l0 = qs(k, 0) * (wj / B.rho[k]), l1 = qs(k, 1) * (wj * g), l2 = qs(k, 2) * (wj * g);
      acc[1] += Y * l0;
      acc[2] -= X * l0;
      acc[0] += Y * l1 - X * l2;
    };
    // this node's q-direction volume term from neighbour k with weight W
    auto phi_q = [&](long long k, double W) {
      const double Y = 0.5 * (B.yr[k] + yrc), X = 0.5 * (B.xr[k] + xrc);
      const double f0 = ust[k], f1 = ust[plane + k], f2 = ust[2 * plane + k];
      phi[0] += W * (Y * f1 - X * f2);
      phi[1] += W * (Y * f0);
      phi[2] += W * (-X * f0);
    };
#pragma unroll
    for (int s = 1; s <= PI_; ++s) {
      const int a = i - s, b = i + s;  // output columns with this node at +s / -s
      if (a >= nbst && a <= nx - 1 - nbst) gather_q(a, D.DI[s]);
      if (b >= nbst && b <= nx - 1 - nbst) gather_q(b, -D.DI[s]);
    }
    if (i < nbnd)
      for (int ic = 0; ic < nbst; ++ic) gather_q(ic, D.DL[ic][i]);
    if (nx - 1 - i < nbnd)
      for (int ic = nx - nbst; ic < nx; ++ic) gather_q(ic, -D.DL[nx - 1 - ic][nx - 1 - i]);
    if (i < nbst) {
#pragma unroll
      for (int s = 0; s < nbnd; ++s) phi_q((long long)j * pitch + s, D.DL[i][s]);
    } else if (i > nx - 1 - nbst) {
#pragma unroll
      for (int s = 0; s < nbnd; ++s) phi_q((long long)j * pitch + (nx - 1 - s), -D.DL[nx - 1 - i][s]);
    } else {
#pragma unroll
      for (int s = 1; s <= PI_; ++s) { phi_q(c + s, D.DI[s]); phi_q(c - s, -D.DI[s]); }
    }
  } else {
    const double yqc = B.yq[c], xqc = B.xq[c];
    auto gather_r = [&](int jc, double W) {
      const long long k = (long long)jc * pitch + i;
      const double Y = 0.5 * (B.yq[k] + yqc), X = 0.5 * (B.xq[k] + xqc);
      const double wj = W * B.Ji[k], g = B.G[k];
      const double l0 = qs(k, 0) * (wj / B.rho[k]), l1 = qs(k, 1) * (wj * g), l2 = qs(k, 2) * (wj * g);
      acc[1] -= Y * l0;
      acc[2] += X * l0;
      acc[0] += -Y * l1 + X * l2;
    };
    auto phi_r = [&](long long k, double W) {
      const double Y = 0.5 * (B.yq[k] + yqc), X = 0.5 * (B.xq[k] + xqc);
      const double f0 = ust[k], f1 = ust[plane + k], f2 = ust[2 * plane + k];
      phi[0] += W * (-Y * f1 + X * f2);
      phi[1] += W * (-Y * f0);
      phi[2] += W * (X * f0);
    };
#pragma unroll
    for (int s = 1; s <= PI_; ++s) {
      const int ar = j - s, br = j + s;
      if (ar >= nbst && ar <= ny - 1 - nbst) gather_r(ar, D.DI[s]);
      if (br >= nbst && br <= ny - 1 - nbst) gather_r(br, -D.DI[s]);
    }
    if (j < nbnd)
      for (int jc = 0; jc < nbst; ++jc) gather_r(jc, D.DL[jc][j]);
    if (ny - 1 - j < nbnd)
      for (int jc = ny - nbst; jc < ny; ++jc) gather_r(jc, -D.DL[ny - 1 - jc][ny - 1 - j]);
    if (j < nbst) {
#pragma unroll
      for (int s = 0; s < nbnd; ++s) phi_r((long long)s * pitch + i, D.DL[j][s]);
    } else if (j > ny - 1 - nbst) {
#pragma unroll
      for (int s = 0; s < nbnd; ++s) phi_r((long long)(ny - 1 - s) * pitch + i, -D.DL[ny - 1 - j][s]);
    } else {
#pragma unroll
      for (int s = 1; s <= PI_; ++s) { phi_r(c + s * pitch, D.DI[s]); phi_r(c - s * pitch, -D.DI[s]); }
    }
  }
  // SAT of the outer sides through this node (L, R on part 0; B, T on part 1)
  const double lam[3] = {qs(c, 0), qs(c, 1), qs(c, 2)};
  const double rho = B.rho[c], G = B.G[c];
  auto side = [&](int sd, int k) {
    const DevSide& S = B.side[sd];
    if (S.bc == FDMAP_BC_NONE) return;  // interface side: the fault adjoint's
    const double us[3] = {ust[c], ust[plane + c], ust[2 * plane + c]};
    const double F0[3] = {S.F0[k], S.F0[k + S.n], S.F0[k + 2 * S.n]};
    sat_adjoint(S.bc, S.M[k], S.M[k + 3 * S.n], S.nrm[k], S.nrm[k + S.n], lam, us, F0, rho, G, acc, &grho, &gG);
  };
  if (part == 0) {
    if (i == 0) side(0, j);
    if (i == nx - 1) side(1, j);
  } else {
    if (j == 0) side(2, i);
    if (j == ny - 1) side(3, i);
  }
}

constexpr int ATX = 32, ATY = 8;

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(w),
      "r"(smem_u32(bar))
      : "memory");
}


// nodes within nbnd of a side use closure rows somewhere in their gather or
// their own rates: the band handled by adj_band_kernel
__device__ __forceinline__ bool adj_node_interior(int i, int j, int nx, int ny, int nbnd) {
  return i >= nbnd && i <= nx - 1 - nbnd && j >= nbnd && j <= ny - 1 - nbnd;
}

// band node q -> (i, j): nbnd full rows at the bottom, nbnd at the top, then
// nbnd columns on the left and right of the rows between
__device__ __forceinline__ void band_node(long long q, int nx, int ny, int nbnd, int& i, int& j) {
  const long long rows = (long long)nbnd * nx;
  if (q < rows) { j = (int)(q / nx); i = (int)(q % nx); return; }
  q -= rows;
  if (q < rows) { j = ny - nbnd + (int)(q / nx); i = (int)(q % nx); return; }
  q -= rows;
  const int k = (int)(q % (2 * nbnd));
  j = nbnd + (int)(q / (2 * nbnd));
  i = k < nbnd ? k : nx - 2 * nbnd + k;
}

// the band (closures, sides, corners): 128 nodes per 256-thread CTA; threads
// 0..127 take the q direction of their node, threads 128..255 the r direction
// of the same node (whole warps per direction, so the branches do not
// diverge), and the partial sums meet in shared memory
constexpr int BAND_NODES = 128;

template <int PI_>
__global__ void __launch_bounds__(2 * BAND_NODES) adj_band_kernel(const __grid_constant__ DevDomain D, AdjStage p,
                                                                   long long nband) {
  __shared__ double part1[8][BAND_NODES];  // acc 3, phi 3, grho, gG of the r direction
  const int part = threadIdx.x / BAND_NODES, slot = threadIdx.x % BAND_NODES;
  const long long q = (long long)blockIdx.x * BAND_NODES + slot;
  const bool valid = q < nband;
  const DevBlock& B = D.blk[p.blk];
  int i = 0, j = 0;
  double acc[3], phi[3], grho = 0.0, gG = 0.0;
  if (valid) {
    band_node(q, B.nx, B.ny, nbnd_of(PI_), i, j);
    adj_node_part<PI_>(D, p, i, j, part, acc, phi, grho, gG);
    if (part == 1) {
#pragma unroll
      for (int f = 0; f < 3; ++f) { part1[f][slot] = acc[f]; part1[3 + f][slot] = phi[f]; }
      part1[6][slot] = grho;
      part1[7][slot] = gG;
    }
  }
  __syncthreads();
  if (!valid || part != 0) return;
#pragma unroll
  for (int f = 0; f < 3; ++f) { acc[f] += part1[f][slot]; phi[f] += part1[3 + f][slot]; }
  grho += part1[6][slot];
  gG += part1[7][slot];
  const long long pitch = B.pitch, plane = B.plane;
  const long long c = (long long)j * pitch + i;
  double lam[3], ubc[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    ubc[f] = p.ub_in[f * plane + c];
    lam[f] = p.qp_in[f * plane + c] + p.Bdt * ubc[f];
  }
  const double Ji = B.Ji[c], rinv = 1.0 / B.rho[c];
  grho -= lam[0] * (phi[0] * Ji) * (rinv * rinv);
  gG += lam[1] * (phi[1] * Ji) + lam[2] * (phi[2] * Ji);
  p.grho[c] += grho;
  p.gG[c] += gG;
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    p.ub_out[f * plane + c] = ubc[f] + acc[f];
    p.qp_out[f * plane + c] = p.A * lam[f];
  }
}

// Edge impedance and penalty of a heterogeneous mode III side from the node's
// (rho, G): Zs = rho*cs, Ks = cs*geo with cs = sqrt(G/rho) (init_edges,
// domain.f90:1349-1459, with the material given as rho and G)
__global__ void adj_edge_material(DevSide S, const double* __restrict__ rho, const double* __restrict__ G,
                                  const double* __restrict__ geo, int side, int nx, int ny, long long pitch) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= S.n) return;
  int i, j;
  side_node_local(side, k, nx, ny, i, j);
  const long long c = (long long)j * pitch + i;
  const double cs = sqrt(G[c] / rho[c]);
  S.M[k] = rho[c] * cs;
  S.M[k + 3 * S.n] = cs * geo[k];
}

// edge geometry factor H00i*|grad|/J of side `side` from the device metric
// planes, with J formed as the device-built body forms it (side_impedance_kernel)
__global__ void adj_edge_geometry(DevBlock B, int side, int n, double H00i, double* geo) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int i, j;
  side_node_local(side, k, B.nx, B.ny, i, j);
  const long long o = (long long)j * B.pitch + i;
  const double xq = B.xq[o], xr = B.xr[o], yq = B.yq[o], yr = B.yr[o];
  const double J = xq * yr - xr * yq;
  const double mag = side < 2 ? sqrt(xr * xr + yr * yr) : sqrt(xq * xq + yq * yq);
  geo[k] = H00i * mag / J;
}

// vz at the receivers of state u for sample n = ts->n (1-based)
__global__ void adj_sample(const double* __restrict__ u, const long long* __restrict__ rec, int nrec,
                           const TimeState* ts, double* traces, int nsamples) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = ts->n;
  if (r >= nrec || n < 1 || n > nsamples) return;
  traces[(n - 1) * nrec + r] = u[rec[r]];
}

// stage input u_{s-1} -> stage store slot (rel*nstage + s)
__global__ void adj_stash(const double* __restrict__ u, double* store, long long stride, const long long* rel, int s,
                          int nstage, long long count) {
  double* dst = store + ((*rel) * nstage + s) * stride;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (long long)gridDim.x * blockDim.x)
    dst[k] = u[k];
}

struct AdjClock {
  long long rel;   // step within the current segment
  long long n;     // global step whose adjoint runs next (backward) / sample index
};

// end of a recomputed step: advance the forward clock and the segment index
__global__ void adj_forward_advance(TimeState* ts, AdjClock* ck) {
  ts->n += 1;
  ck->rel += 1;
}

// ---------------------------------------------------------------------------
// Interior adjoint stage, 32 x 8 nodes per CTA, for nodes at least nbnd from
// every side (every output node they gather from, and their own volume
// rates, use the central stencil); the band is adj_band_kernel's.  The tile
// is delivered by TMA: five 3-D boxes
// (qbar' 3 planes, ubar 3, stage input 3, metrics yr xr yq xq Ji 5, rho G 2)
// land in shared memory on one mbarrier; the box starts HX = PI_ rounded up
// to even columns left of the tile so every box starts on a 16-byte boundary.
// ---------------------------------------------------------------------------
struct AdjMaps {
  CUtensorMap ub[2];  // ubar buffers, box {WX, WY, 3}
  CUtensorMap qp[2];  // qbar' buffers, box {WX, WY, 3}
  CUtensorMap st;     // stage-input store: 4-D (x, y, plane, slot), box {WX, WY, 3, 1}
  CUtensorMap met;    // yr, xr, yq, xq, Ji, box {WX, WY, 5}
  CUtensorMap het;    // rho, G, box {WX, WY, 2}
};

template <int PI_>
struct AdjTile {
  static constexpr int HX = (PI_ + 1) & ~1;
  static constexpr int HY = PI_;
  static constexpr int WX = ATX + 2 * HX;
  static constexpr int WY = ATY + 2 * HY;
  static constexpr int PL = WX * WY;                 // doubles per plane of the tile
  static constexpr int NPL = 16;                     // qp 3, ub 3, st 3, met 5, het 2
  static constexpr unsigned BYTES = (unsigned)NPL * PL * 8;  // bytes the five boxes deliver
  // each box lands on a 128-byte aligned group (offsets in doubles)
  static constexpr int grp(int planes) { return (planes * PL * 8 + 127) / 128 * 16; }
  static constexpr int QP = 0, UB = QP + grp(3), ST = UB + grp(3), MET = ST + grp(3), HET = MET + grp(5);
  static constexpr unsigned SMEM = (unsigned)(HET + grp(2)) * 8;
};

template <int PI_>
__global__ void __launch_bounds__(ATX* ATY) adj_stage_tma(const __grid_constant__ DevDomain D, AdjStage p,
                                                           const __grid_constant__ AdjMaps maps, int q) {
  using T = AdjTile<PI_>;
  constexpr int nbnd = nbnd_of(PI_);
  extern __shared__ unsigned char adj_smem_raw[];
  double* sm = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(adj_smem_raw) + 127) & ~uintptr_t(127));
  __shared__ unsigned long long bar;
  const DevBlock& B = D.blk[p.blk];
  const int nx = B.nx, ny = B.ny;
  const int i0 = blockIdx.x * ATX, j0 = blockIdx.y * ATY;
  const int tx = threadIdx.x % ATX, ty = threadIdx.x / ATX;
  if (i0 + ATX - 1 < nbnd || i0 > nx - 1 - nbnd || j0 + ATY - 1 < nbnd || j0 > ny - 1 - nbnd) return;
  // P(group, plane, yy, xx): plane `plane` of a box group, tile row yy, column xx
  auto P = [&](int grp, int plane, int yy, int xx) -> double& { return sm[grp + (plane * T::WY + yy) * T::WX + xx]; };
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async();
    const int x = i0 - T::HX, y = j0 - T::HY;
    const int slot = (int)((*p.rel) * p.nstage + p.s);
    mbar_arrive_tx(&bar, T::BYTES);
    tma_load_3d(&P(T::QP, 0, 0, 0), &maps.qp[q], x, y, 0, &bar);
    tma_load_3d(&P(T::UB, 0, 0, 0), &maps.ub[q], x, y, 0, &bar);
    tma_load_4d(&P(T::ST, 0, 0, 0), &maps.st, x, y, 0, slot, &bar);
    tma_load_3d(&P(T::MET, 0, 0, 0), &maps.met, x, y, 0, &bar);
    tma_load_3d(&P(T::HET, 0, 0, 0), &maps.het, x, y, 0, &bar);
  }
  __syncthreads();
  if (__syncthreads_or(!mbar_wait_bounded(&bar, 0, D.status))) {
    // the tile never arrived: no compute; wait once more for the copies before leaving
    if (threadIdx.x == 0) mbar_wait_bounded(&bar, 0, D.status);
    __syncthreads();
    return;
  }
  const int X0 = tx + T::HX, Y0 = ty + T::HY;
  const bool mine = adj_node_interior(i0 + tx, j0 + ty, nx, ny, nbnd);
  double lam[3], ubc[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    ubc[f] = P(T::UB, f, Y0, X0);
    lam[f] = P(T::QP, f, Y0, X0) + p.Bdt * ubc[f];
  }
  const double Jc = P(T::MET, 4, Y0, X0), rho_c = P(T::HET, 0, Y0, X0);
  __syncthreads();
  // weighted adjoint rates l_r = qs_r * Ji * (1/rho | G), in place of qbar'
  for (int k = threadIdx.x; k < T::PL; k += ATX * ATY) {
    const int yy = k / T::WX, xx = k % T::WX;
    const double Jk = P(T::MET, 4, yy, xx), wv = Jk / P(T::HET, 0, yy, xx), ws = Jk * P(T::HET, 1, yy, xx);
    P(T::QP, 0, yy, xx) = (P(T::QP, 0, yy, xx) + p.Bdt * P(T::UB, 0, yy, xx)) * wv;
    P(T::QP, 1, yy, xx) = (P(T::QP, 1, yy, xx) + p.Bdt * P(T::UB, 1, yy, xx)) * ws;
    P(T::QP, 2, yy, xx) = (P(T::QP, 2, yy, xx) + p.Bdt * P(T::UB, 2, yy, xx)) * ws;
  }
  __syncthreads();
  if (!mine) return;  // band node (adj_band_kernel)
  const double yrc = P(T::MET, 0, Y0, X0), xrc = P(T::MET, 1, Y0, X0), yqc = P(T::MET, 2, Y0, X0),
               xqc = P(T::MET, 3, Y0, X0);
  double acc[3] = {0.0, 0.0, 0.0};
  double phi[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int s = 1; s <= PI_; ++s) {
    const double w = D.DI[s];
#pragma unroll
    for (int side = -1; side <= 1; side += 2) {
      const int xa = X0 + side * s;
      const double W = -side * w;  // left output (side -1): +DI, right output: -DI
      const double Y = 0.5 * (P(T::MET, 0, Y0, xa) + yrc), X = 0.5 * (P(T::MET, 1, Y0, xa) + xrc);
      const double l0 = P(T::QP, 0, Y0, xa), l1 = P(T::QP, 1, Y0, xa), l2 = P(T::QP, 2, Y0, xa);
      acc[1] += W * (Y * l0);
      acc[2] -= W * (X * l0);
      acc[0] += W * (Y * l1 - X * l2);
      const double u0 = P(T::ST, 0, Y0, xa), u1 = P(T::ST, 1, Y0, xa), u2 = P(T::ST, 2, Y0, xa);
      const double Wf = side * w;
      phi[0] += Wf * (Y * u1 - X * u2);
      phi[1] += Wf * (Y * u0);
      phi[2] += Wf * (-X * u0);
      const int ya = Y0 + side * s;
      const double Yr = 0.5 * (P(T::MET, 2, ya, X0) + yqc), Xr = 0.5 * (P(T::MET, 3, ya, X0) + xqc);
      const double m0 = P(T::QP, 0, ya, X0), m1 = P(T::QP, 1, ya, X0), m2 = P(T::QP, 2, ya, X0);
      acc[1] -= W * (Yr * m0);
      acc[2] += W * (Xr * m0);
      acc[0] += W * (-Yr * m1 + Xr * m2);
      const double v0 = P(T::ST, 0, ya, X0), v1 = P(T::ST, 1, ya, X0), v2 = P(T::ST, 2, ya, X0);
      phi[0] += Wf * (-Yr * v1 + Xr * v2);
      phi[1] += Wf * (-Yr * v0);
      phi[2] += Wf * (Xr * v0);
    }
  }
  const long long pitch = B.pitch, plane = B.plane;
  const long long c = (long long)(j0 + ty) * pitch + (i0 + tx);
  const double rinv = 1.0 / rho_c;
  p.grho[c] += -lam[0] * (phi[0] * Jc) * (rinv * rinv);
  p.gG[c] += lam[1] * (phi[1] * Jc) + lam[2] * (phi[2] * Jc);
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    p.ub_out[f * plane + c] = ubc[f] + acc[f];
    p.qp_out[f * plane + c] = p.A * lam[f];
  }
}

// end of an adjoint step n: ubar += dJ/dU^n at the receivers, then step back.
// One thread per distinct receiver node; receivers sharing a node (rlist
// entries rstart[t]..rstart[t+1]) are summed in a fixed order.
__global__ void adj_inject(double* ub, const long long* __restrict__ node, const int* __restrict__ rstart,
                           const int* __restrict__ rlist, int nnode, int nrec, const double* __restrict__ resid,
                           AdjClock* ck, int back) {
  const long long n = ck->n;
  for (int t = threadIdx.x; t < nnode; t += blockDim.x) {
    double sum = 0.0;
    for (int q = rstart[t]; q < rstart[t + 1]; ++q) sum += resid[(n - 1) * nrec + rlist[q]];
    ub[node[t]] += sum;
  }
  __syncthreads();
  if (back && threadIdx.x == 0) {
    ck->n -= 1;
    ck->rel -= 1;
  }
}

// end of a forward step: vz at the receivers of the new state (sample n+1),
// then n += 1 and, given the store clock, its step index += 1
__global__ void adj_sample_advance(const double* __restrict__ u, const long long* __restrict__ rec, int nrec,
                                   TimeState* ts, double* traces, int nsamples, AdjClock* ck) {
  const long long n = ts->n + 1;
  for (int r = threadIdx.x; r < nrec; r += blockDim.x)
    if (n >= 1 && n <= nsamples) traces[(n - 1) * nrec + r] = u[rec[r]];
  __syncthreads();
  if (threadIdx.x == 0) {
    ts->n = n;
    if (ck) ck->rel += 1;
  }
}

}  // namespace fdmap
