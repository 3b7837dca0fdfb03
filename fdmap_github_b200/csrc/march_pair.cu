// Host side of the two-stage march (march_pair.cuh): eligibility, the scratch
// buffers, the band table, the tensor maps and the launches.
#include <cuda.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>

#include "engine.h"
#include "march_host.cuh"
#include "march_pair.cuh"

namespace fdmap {

void pair_free(fdmap_gpu* h) {
  delete h->tmaps_pair;
  h->tmaps_pair = nullptr;
}

namespace {

template <int MODE, int PI_>
int pair_maps(fdmap_gpu* h) {
  using L = PairLayout<MODE, PI_>;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult qr;
  CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr));
  if (!fn || qr != cudaDriverEntryPointSuccess) return set_err(FDMAP_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  auto enc = (march_detail::EncodeTiledFn)fn;
  if (!h->tmaps_pair) h->tmaps_pair = new (std::nothrow) TmapPair();
  if (!h->tmaps_pair) return set_err(FDMAP_ERR_NOMEM, "out of host memory");
  std::memset(h->tmaps_pair, 0, sizeof(TmapPair));
  TmapPair& T = *h->tmaps_pair;
  int rc;
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    const BlockGeom& g = h->geom[b];
    const DevBlock& B = h->hdom.blk[b];
    for (int q = 0; q < 2; ++q) {
      if ((rc = march_detail::encode_map(enc, &T.F[b][q], B.F[q], g, h->nF, L::WB, L::MR, L::NR))) return rc;
      if ((rc = march_detail::encode_map(enc, &T.F6[b][q], B.F[q], g, h->nF, L::WB, L::MR, 1))) return rc;
    }
    if ((rc = march_detail::encode_map(enc, &T.DF[b][0], B.DF, g, h->nF, L::WB, L::MR, L::NR))) return rc;
    if ((rc = march_detail::encode_map(enc, &T.DF[b][1], B.DFalt, g, h->nF, L::WB, L::MR, L::NR))) return rc;
    if ((rc = march_detail::encode_map(enc, &T.MT[b], h->met_base[b], g, 5, L::WB, L::MR, 5))) return rc;
  }
  return FDMAP_OK;
}

template <int MODE, int PI_>
int pair_setup(fdmap_gpu* h) {
  using L = PairLayout<MODE, PI_>;
  int optin = 0, sms = 0, per_sm = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
  if (L::BYTES > (size_t)optin) return FDMAP_ERR_UNSUPPORTED;
  DevDomain& D = h->hdom;
  // scratch buffers: the first stage's fields near the edges, the second rate buffer
  for (int b = 0; b < D.nblocks; ++b) {
    DevBlock& B = D.blk[b];
    const BlockGeom& g = h->geom[b];
    int rc;
    if (!B.F[2] && (rc = h->alloc_planes(&B.F[2], h->nF, g.plane))) return rc;
    if (!B.DFalt && (rc = h->alloc_planes(&B.DFalt, h->nF, g.plane))) return rc;
  }
  // units: strips of MWC core columns x row groups of MR rows, block after block
  long long units = 0;
  for (int b = 0; b < D.nblocks; ++b) {
    DevBlock& B = D.blk[b];
    B.pair_unit_begin = units;
    units += (long long)((B.nx + L::MWC - 1) / L::MWC) * ((B.ny + L::MR - 1) / L::MR);
  }
  h->pair_units = units;
  // bands of width nbst + PI along the four sides of every block
  const int w = D.nbst + PI_;
  D.nbw = w;
  long long bs = 0;
  for (int b = 0; b < D.nblocks; ++b) {
    const BlockGeom& g = h->geom[b];
    const long long strip[4] = {(long long)w * g.nx, (long long)w * g.nx, (long long)(g.ny - 2 * w) * w,
                                (long long)(g.ny - 2 * w) * w};
    for (int q = 0; q < 4; ++q) { D.bstart[4 * b + q] = bs; bs += strip[q]; }
  }
  D.bstart[4 * D.nblocks] = bs;
  h->band_threads = bs;
  int rc = pair_maps<MODE, PI_>(h);
  if (rc) return rc;
  auto k = march_pair_kernel<MODE, PI_>;
  CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES));
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, L::THREADS, L::BYTES));
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
  if (per_sm < 1) return FDMAP_ERR_UNSUPPORTED;
  h->pair_grid = (int)std::max<long long>(1, std::min<long long>((long long)sms * per_sm, units));
  // the band kernel runs beside nothing, but the closure and interface kernels
  // of the pair run beside the pass: they already take the largest carveout
  CUDA_TRY(cudaFuncSetAttribute((const void*)band_kernel<MODE, PI_>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  return FDMAP_OK;
}

template <typename Fn>
int pair_dispatch(const fdmap_gpu* h, Fn&& fn) {
  if (h->mode == 2) {
    if (h->pI == 1) return fn(std::integral_constant<int, 2>{}, std::integral_constant<int, 1>{});
    if (h->pI == 2) return fn(std::integral_constant<int, 2>{}, std::integral_constant<int, 2>{});
  } else {
    if (h->pI == 1) return fn(std::integral_constant<int, 3>{}, std::integral_constant<int, 1>{});
    if (h->pI == 2) return fn(std::integral_constant<int, 3>{}, std::integral_constant<int, 2>{});
  }
  return FDMAP_ERR_UNSUPPORTED;
}

}  // namespace

int pair_configure(fdmap_gpu* h) {
  h->pair_ok = false;
  h->use_pairs = false;
  // the pass does the plain split form on homogeneous blocks; the rest stays per stage
  if (!h->use_march || h->het || h->dissipation || h->pml || h->forcing || h->extras || h->d_energy ||
      h->partitioned() || h->pI > 2)
    return FDMAP_OK;
  const DevDomain& D = h->hdom;
  for (int b = 0; b < D.nblocks; ++b)
    if (h->geom[b].nx < 2 * (D.nbst + h->pI) + 1 || h->geom[b].ny < 2 * (D.nbst + h->pI) + 1) return FDMAP_OK;
  const int rc = pair_dispatch(h, [&](auto m, auto p) { return pair_setup<decltype(m)::value, decltype(p)::value>(h); });
  if (rc == FDMAP_ERR_UNSUPPORTED) return FDMAP_OK;
  if (rc) return rc;
  h->pair_ok = true;
  h->use_pairs = true;
  return FDMAP_OK;
}

int pair_launch(fdmap_gpu* h, const StageArgs& a0, const StageArgs& a1, int dfr, int dfw) {
  return pair_dispatch(h, [&](auto m, auto p) -> int {
    constexpr int MODE = decltype(m)::value, PI_ = decltype(p)::value;
    using L = PairLayout<MODE, PI_>;
    PairPlan plan{h->pair_units, nullptr, nullptr, 1, dfr, dfw};
    march_pair_kernel<MODE, PI_><<<h->pair_grid, L::THREADS, L::BYTES, h->stream>>>(h->ddom, a0, a1, plan,
                                                                                   *h->tmaps_pair);
    CUDA_TRY(cudaGetLastError());
    return FDMAP_OK;
  });
}

int band_launch(fdmap_gpu* h, const StageArgs& a) {
  if (h->band_threads == 0) return FDMAP_OK;
  const int nb = (int)((h->band_threads + 127) / 128);
  return pair_dispatch(h, [&](auto m, auto p) -> int {
    band_kernel<decltype(m)::value, decltype(p)::value><<<nb, 128, 0, h->stream>>>(h->hdom, a);
    CUDA_TRY(cudaGetLastError());
    return FDMAP_OK;
  });
}

int pair_batch(const fdmap_gpu* proto, const StageArgs& a0, const StageArgs& a1, int dfr, int dfw,
               const PairBatch& p, cudaStream_t s) {
  return pair_dispatch(proto, [&](auto m, auto pi) -> int {
    constexpr int MODE = decltype(m)::value, PI_ = decltype(pi)::value;
    using L = PairLayout<MODE, PI_>;
    PairPlan plan{p.units, p.tmaps, p.unit_begin, p.ninst, dfr, dfw};
    march_pair_kernel<MODE, PI_><<<p.grid, L::THREADS, L::BYTES, s>>>(p.doms, a0, a1, plan, *proto->tmaps_pair);
    CUDA_TRY(cudaGetLastError());
    return FDMAP_OK;
  });
}

int band_batch(const fdmap_gpu* proto, const StageArgs& a, const PairBatch& p, cudaStream_t s) {
  if (p.band_ctas == 0) return FDMAP_OK;
  return pair_dispatch(proto, [&](auto m, auto pi) -> int {
    band_kernel_batch<decltype(m)::value, decltype(pi)::value><<<p.band_ctas, 128, 0, s>>>(p.doms, p.band_cta_begin,
                                                                                           p.ninst, a);
    CUDA_TRY(cudaGetLastError());
    return FDMAP_OK;
  });
}

}  // namespace fdmap
