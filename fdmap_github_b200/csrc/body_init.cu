// On-device initialisation of a domain's body: the transfinite grid
// (transfinite_interp, geometry.f90:153-200), its SBP metric terms and
// Jacobian (init_grid_partials, grid.f90:465-618), the initial body fields
// (init_fields + perturb_fields, fields.f90:774-934), the edge impedances of
// every side (init_edges, domain.f90:1349-1459) and the grid spacings set_dt
// reduces (domain.f90:1481-1495), built in place in the engine's padded block
// planes.  The host keeps only the O(nx + ny) part of init_domain.
//
// This file is compiled with -fmad=false: every node evaluates the formulas of
// body_formulas.h with the same roundings as the host restatement, so the
// device-built grid, metrics, Jacobian and impedances are bit-identical to the
// host's (the initial fields too, except for last-bit differences of exp() in
// 'smooth' and 'gaussian' perturbations).
#include <cmath>
#include <cstring>
#include <vector>

#include "body_formulas.h"
#include "pml_formula.h"
#include "engine.h"

namespace fdmap {
namespace {

struct BodyOp {
  int nbst, nbnd, pI;
  double H00i;
  double DI[SBP_MAX_PI + 1];
  double DL[SBP_MAX_NBST][SBP_MAX_NBND];
};

struct BodyBlock {
  int nx, ny, pitch, mgx, mgy, nF;
  long long plane;
  const double* cx[4];  // edge curves L, R (length ny), B, T (length nx)
  const double* cy[4];
  double LB[2], LT[2], RB[2], RT[2];
  double* x;  // scratch planes of the grid
  double* y;
  double *yr, *xr, *yq, *xq, *Ji, *J;  // J may be NULL
  double* F;
  double* DF;
  double F0[6];
  int pshape[5];
  double px0[5], py0[5], pLx[5], pLy[5];
  double pv[5][6];
};

struct BodySide {
  int n, side;
  double* M;            // (n,5)
  const double* mat;    // (n,3) rho, cs, cp or NULL
  double rho, cs, cp;   // block material when mat is NULL
};

// grid node and initial fields of one node (the perturbation amplitudes need
// only the node's own coordinates)
__global__ void grid_fields_kernel(BodyBlock B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= B.nx || j >= B.ny) return;
  const double qmin = B.mgx, qmax = B.mgx + B.nx - 1, rmin = B.mgy, rmax = B.mgy + B.ny - 1;
  double Wq = qmax - qmin, Wr = rmax - rmin;
  if (Wq == 0.0) Wq = 1.0;
  if (Wr == 0.0) Wr = 1.0;
  const double q = B.mgx + i, r = B.mgy + j;
  const double xv = transfinite(q, r, qmin, qmax, rmin, rmax, Wq, Wr, B.cx[0][j], B.cx[1][j], B.cx[2][i], B.cx[3][i],
                                B.LB[0], B.LT[0], B.RB[0], B.RT[0]);
  const double yv = transfinite(q, r, qmin, qmax, rmin, rmax, Wq, Wr, B.cy[0][j], B.cy[1][j], B.cy[2][i], B.cy[3][i],
                                B.LB[1], B.LT[1], B.RB[1], B.RT[1]);
  const long long o = (long long)j * B.pitch + i;
  B.x[o] = xv;
  B.y[o] = yv;
  double A[5];
  for (int k = 0; k < 5; ++k) A[k] = perturb_amp(B.pshape[k], xv, yv, B.px0[k], B.py0[k], B.pLx[k], B.pLy[k]);
  for (int l = 0; l < B.nF; ++l) {
    B.F[l * B.plane + o] =
        B.F0[l] + A[0] * B.pv[0][l] + A[1] * B.pv[1][l] + A[2] * B.pv[2][l] + A[3] * B.pv[3][l] + A[4] * B.pv[4][l];
    B.DF[l * B.plane + o] = 1e40;  // fields.f90:850 sentinel
  }
}

// metric terms, Jacobian and the node's grid spacings; hmin / hmax reduced
// through their IEEE bit patterns (non-negative doubles order as integers)
__global__ void metrics_kernel(BodyBlock B, BodyOp op, unsigned long long* hminmax) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  double lo = HUGE_VAL, hi = 0.0;
  if (i < B.nx && j < B.ny) {
    const double* x = B.x;
    const double* y = B.y;
    const long long row = (long long)j * B.pitch;
    const double xq = sbp_diff_at(op.nbst, op.nbnd, op.pI, op.DI, op.DL, B.nx, i, [&](int k) { return x[row + k]; });
    const double yq = sbp_diff_at(op.nbst, op.nbnd, op.pI, op.DI, op.DL, B.nx, i, [&](int k) { return y[row + k]; });
    const double xr = sbp_diff_at(op.nbst, op.nbnd, op.pI, op.DI, op.DL, B.ny, j,
                                  [&](int k) { return x[(long long)k * B.pitch + i]; });
    const double yr = sbp_diff_at(op.nbst, op.nbnd, op.pI, op.DI, op.DL, B.ny, j,
                                  [&](int k) { return y[(long long)k * B.pitch + i]; });
    const double J = xq * yr - xr * yq;
    const long long o = row + i;
    B.yr[o] = yr;
    B.xr[o] = xr;
    B.yq[o] = yq;
    B.xq[o] = xq;
    B.Ji[o] = 1.0 / J;
    if (B.J) B.J[o] = J;
    const double dq = spacing_q(J, xr, yr), dr = spacing_r(J, xq, yq);
    if (dq == dq) { lo = fmin(lo, dq); hi = fmax(hi, dq); }
    if (dr == dr) { lo = fmin(lo, dr); hi = fmax(hi, dr); }
  }
  for (int off = 16; off > 0; off >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, off));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&hminmax[0], (unsigned long long)__double_as_longlong(lo));
    atomicMax(&hminmax[1], (unsigned long long)__double_as_longlong(hi));
  }
}

// PML damping planes sx, sy from the grid (pml_damping, rates.f90:2065-2068)
__global__ void pml_damping_kernel(BodyBlock B, double* damp, double sigma, double n, double mx, double px, double my,
                                   double py) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= B.nx || j >= B.ny) return;
  const long long o = (long long)j * B.pitch + i;
  damp[o] = pml_damping(sigma, n, mx, px, B.x[o]);
  damp[B.plane + o] = pml_damping(sigma, n, my, py, B.y[o]);
}

// hxi = Ji*yr, hyi = Ji*xq at the first node of each PML region (q, r: 0 minus
// end, 1 plus end, 2 interior), one thread per region
__global__ void pml_regions_kernel(BodyBlock B, double* hh, int nbst) {
  const int k = threadIdx.x;
  if (k >= 9) return;
  const int q = k / 3, r = k % 3;
  const int qi = q == 0 ? 0 : (q == 1 ? B.nx - nbst : nbst);
  const int rj = r == 0 ? 0 : (r == 1 ? B.ny - nbst : nbst);
  const long long o = (long long)rj * B.pitch + qi;
  hh[2 * k] = B.Ji[o] * B.yr[o];
  hh[2 * k + 1] = B.Ji[o] * B.xq[o];
}

// edge impedances (Zs, Zp, gamma, Ks, Kp) of the nodes of one side
__global__ void side_impedance_kernel(BodyBlock B, BodySide S, double H00i) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= S.n) return;
  int i, j;
  if (S.side == 0) { i = 0; j = k; }
  else if (S.side == 1) { i = B.nx - 1; j = k; }
  else if (S.side == 2) { i = k; j = 0; }
  else { i = k; j = B.ny - 1; }
  const long long o = (long long)j * B.pitch + i;
  const double xq = B.xq[o], xr = B.xr[o], yq = B.yq[o], yr = B.yr[o];
  const double J = xq * yr - xr * yq;
  const double mag = S.side < 2 ? sqrt(xr * xr + yr * yr) : sqrt(xq * xq + yq * yq);
  double rho = S.rho, cs = S.cs, cp = S.cp;
  if (S.mat) { rho = S.mat[k]; cs = S.mat[k + S.n]; cp = S.mat[k + 2 * (long long)S.n]; }
  edge_impedances(rho, cs, cp, mag, J, H00i, &S.M[k], S.n);
}

// device scratch released when the build returns
struct Scratch {
  std::vector<void*> p;
  ~Scratch() {
    for (void* q : p) cudaFree(q);
  }
  template <class T>
  cudaError_t get(T** out, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 16);
    if (e == cudaSuccess) p.push_back(q);
    *out = (T*)q;
    return e;
  }
};

}  // namespace

int build_body(fdmap_gpu* h, const fdmap_desc* d, const SbpOperator& sop) {
  const fdmap_body* body = d->body;
  BodyOp op{};
  op.nbst = sop.nbst; op.nbnd = sop.nbnd; op.pI = sop.pI; op.H00i = sop.H00i;
  std::memcpy(op.DI, sop.DI, sizeof(op.DI));
  std::memcpy(op.DL, sop.DL, sizeof(op.DL));
  Scratch sc;
  unsigned long long* hmm = nullptr;
  CUDA_TRY(sc.get(&hmm, 2));
  unsigned long long init[2] = {0ull, 0ull};
  const double big = HUGE_VAL;
  std::memcpy(&init[0], &big, sizeof(double));
  CUDA_TRY(cudaMemcpyAsync(hmm, init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
  std::vector<BodyBlock> blocks(d->nblocks);
  for (int b = 0; b < d->nblocks; ++b) {
    const fdmap_block& fb = d->blocks[b];
    const fdmap_block_body& bb = body->blocks[b];
    const BlockGeom& g = h->geom[b];
    DevBlock& D = h->hdom.blk[b];
    BodyBlock& B = blocks[b];
    B.nx = g.nx; B.ny = g.ny; B.pitch = g.pitch; B.mgx = g.mgx; B.mgy = g.mgy; B.nF = d->nF; B.plane = g.plane;
    for (int s = 0; s < 4; ++s) {
      const fdmap_side& fs = fb.side[s];
      double* c = nullptr;
      CUDA_TRY(sc.get(&c, 2 * (size_t)fs.n));
      CUDA_TRY(cudaMemcpyAsync(c, fs.x, fs.n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
      CUDA_TRY(cudaMemcpyAsync(c + fs.n, fs.y, fs.n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
      B.cx[s] = c;
      B.cy[s] = c + fs.n;
    }
    for (int c = 0; c < 2; ++c) {
      B.LB[c] = bb.LB[c]; B.LT[c] = bb.LT[c]; B.RB[c] = bb.RB[c]; B.RT[c] = bb.RT[c];
    }
    CUDA_TRY(sc.get(&B.x, (size_t)g.plane));
    CUDA_TRY(sc.get(&B.y, (size_t)g.plane));
    B.yr = D.yr; B.xr = D.xr; B.yq = D.yq; B.xq = D.xq; B.Ji = D.Ji; B.J = D.J;
    B.F = D.F[h->cur];
    B.DF = D.DF;
    for (int l = 0; l < 6; ++l) B.F0[l] = bb.F0[l];
    for (int k = 0; k < 5; ++k) {
      B.pshape[k] = bb.p[k].shape;
      B.px0[k] = bb.p[k].x0; B.py0[k] = bb.p[k].y0; B.pLx[k] = bb.p[k].Lx; B.pLy[k] = bb.p[k].Ly;
      for (int l = 0; l < 6; ++l) B.pv[k][l] = bb.p[k].v[l];
    }
    dim3 grid((g.nx + 127) / 128, g.ny);
    grid_fields_kernel<<<grid, 128, 0, h->stream>>>(B);
    CUDA_TRY(cudaGetLastError());
    metrics_kernel<<<grid, 128, 0, h->stream>>>(B, op, hmm);
    CUDA_TRY(cudaGetLastError());
    if (D.pml) {
      pml_damping_kernel<<<grid, 128, 0, h->stream>>>(B, const_cast<double*>(D.pml_s), fb.pml_sigma, fb.pml_n,
                                                      fb.pml_mx, fb.pml_px, fb.pml_my, fb.pml_py);
      CUDA_TRY(cudaGetLastError());
      pml_regions_kernel<<<1, 32, 0, h->stream>>>(B, const_cast<double*>(D.pml_h), op.nbst);
      CUDA_TRY(cudaGetLastError());
    }
    for (int s = 0; s < 4; ++s) {
      const fdmap_side& fs = fb.side[s];
      BodySide S{};
      S.n = fs.n; S.side = s; S.M = D.side[s].M;
      S.rho = fb.rho; S.cs = fb.cs; S.cp = fb.cp;
      if (bb.side_mat[s]) {
        double* m = nullptr;
        CUDA_TRY(sc.get(&m, 3 * (size_t)fs.n));
        CUDA_TRY(cudaMemcpyAsync(m, bb.side_mat[s], 3 * fs.n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        S.mat = m;
      }
      side_impedance_kernel<<<(fs.n + 127) / 128, 128, 0, h->stream>>>(B, S, op.H00i);
      CUDA_TRY(cudaGetLastError());
    }
  }
  unsigned long long out[2];
  CUDA_TRY(cudaMemcpyAsync(out, hmm, sizeof(out), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  double hmin, hmax;
  std::memcpy(&hmin, &out[0], sizeof(double));
  std::memcpy(&hmax, &out[1], sizeof(double));
  if (!(hmin > 0.0)) return set_err(FDMAP_ERR_INVALID_ARG, "Minimum grid spacing must be positive");
  double dt, CFL;
  int nt;
  finish_time_step(body->dt_in, body->CFL_in, body->refine, body->tend, body->nt_in, body->c, hmin, &dt, &CFL, &nt);
  h->tp[0] = d->t0; h->tp[1] = dt; h->tp[2] = CFL; h->tp[3] = hmin; h->tp[4] = hmax;
  h->tp_nt = nt;
  for (int b = 0; b < d->nblocks; ++b) h->hdom.blk[b].Cdiss = body->blocks[b].Cdiss * CFL / dt;
  return FDMAP_OK;
}

}  // namespace fdmap
