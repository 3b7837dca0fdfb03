// Mechanical energy of every block in stage 1 (energy_block / energy_interior,
// energy.f90:9-96): sum over the block's nodes of Hx(i) Hy(j) J(i,j) times the
// energy density of the step-start fields with the block's homogeneous
// material.  Two passes with a fixed launch shape, so the sums are
// deterministic: per CTA a partial over a strided set of nodes, then one CTA
// adds the partials of each block in order.
#include "engine.h"

namespace fdmap {
namespace {

constexpr int ETHREADS = 256;
constexpr int ECTAS = 148;  // partial sums per block

template <int MODE>
__global__ void __launch_bounds__(ETHREADS) energy_partial_kernel(const DevDomain* __restrict__ Dp, int b, int cur,
                                                                  double* __restrict__ part) {
  const DevDomain& D = *Dp;
  const DevBlock& B = D.blk[b];
  const long long n = (long long)B.nx * B.ny;
  const double* __restrict__ F = B.F[cur];
  double e = 0.0;
  double v1 = 0, v2 = 0, v3 = 0, v4 = 0;
  if (MODE == 2) {
    const double lambda = B.M_b - 2.0 * B.G_b;
    v1 = 0.5 * B.rho_b; v2 = 0.5 * B.G_b; v3 = 0.25 * B.G_b;
    v4 = -0.25 * B.G_b * (lambda / (3.0 * lambda + 2.0 * B.G_b));
  }
  for (long long q = (long long)blockIdx.x * ETHREADS + threadIdx.x; q < n; q += (long long)ECTAS * ETHREADS) {
    const int j = (int)(q / B.nx), i = (int)(q % B.nx);
    const long long c = (long long)j * B.pitch + i;
    const double w = B.Hx[i] * B.Hy[j] * B.J[c];
    if (MODE == 2) {
      const double f1 = F[c], f2 = F[B.plane + c], f3 = F[2 * B.plane + c], f4 = F[3 * B.plane + c],
                   f5 = F[4 * B.plane + c], f6 = F[5 * B.plane + c];
      e += w * (v1 * (f1 * f1 + f2 * f2) + v2 * (f4 * f4) + v3 * (f3 * f3 + f5 * f5 + f6 * f6) +
                v4 * ((f3 + f5 + f6) * (f3 + f5 + f6)));
    } else {
      const double f1 = F[c], f2 = F[B.plane + c], f3 = F[2 * B.plane + c];
      e += 0.5 * w * (B.rho_b * (f1 * f1) + (f2 * f2 + f3 * f3) / B.G_b);
    }
  }
  __shared__ double red[ETHREADS / 32];
  for (int off = 16; off > 0; off >>= 1) e += __shfl_down_sync(0xffffffffu, e, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < ETHREADS / 32; ++k) s += red[k];
    part[(long long)b * ECTAS + blockIdx.x] = s;
  }
}

// one thread: per block the partials in order, then the sum over blocks
__global__ void energy_final_kernel(const double* __restrict__ part, int nblocks, double* __restrict__ energy) {
  double total = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    double s = 0.0;
    for (int k = 0; k < ECTAS; ++k) s += part[(long long)b * ECTAS + k];
    energy[b] = s;
    total += s;
  }
  energy[nblocks] = total;
}

}  // namespace

int energy_scratch_size(int nblocks) { return nblocks * ECTAS; }

int launch_energy(fdmap_gpu* h, int cur) {
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (h->mode == 2) energy_partial_kernel<2><<<ECTAS, ETHREADS, 0, h->stream>>>(h->ddom, b, cur, h->d_epart);
    else energy_partial_kernel<3><<<ECTAS, ETHREADS, 0, h->stream>>>(h->ddom, b, cur, h->d_epart);
    CUDA_TRY(cudaGetLastError());
    h->launches++;
  }
  energy_final_kernel<<<1, 1, 0, h->stream>>>(h->d_epart, h->hdom.nblocks, h->d_energy);
  CUDA_TRY(cudaGetLastError());
  h->launches++;
  return FDMAP_OK;
}

}  // namespace fdmap
