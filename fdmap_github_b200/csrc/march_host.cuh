// Host side of the march kernel for one tile shape SH: the row-group unit
// decomposition of the handle's blocks, the TMA tensor maps whose boxes
// follow the shape, the launch configuration, and the launches (single
// domain and batched instances).  Each march_s<SH>.cu instantiates it for
// one shape, so the variants of the four shapes compile in parallel.
#pragma once

#include <cuda.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>

#include "engine.h"
#include "march_kernel.cuh"

namespace fdmap {
namespace march_detail {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// 3-D FP64 tensor map over `nplanes` consecutive planes of a block array,
// nx columns wide (the pitch padding reads as zeros without touching memory),
// box {box_x, rows, box_z}.  No L2 promotion: boxes with halo columns start
// 16 bytes before a 256-byte line, and promotion would pull a whole line at
// each end of every row for those 16 bytes; fetched by sector, the halos cost
// what they hold.
inline int encode_map(EncodeTiledFn enc, CUtensorMap* map, const double* base, const BlockGeom& g, int nplanes,
                      int box_x, int rows, int box_z) {
  cuuint64_t dims[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)nplanes};
  cuuint64_t strides[2] = {(cuuint64_t)g.pitch * 8, (cuuint64_t)g.plane * 8};
  cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)rows, (cuuint32_t)box_z};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_err(FDMAP_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return FDMAP_OK;
}

template <int MODE, int PI_, bool HET, int EXT, int SH>
int maps(fdmap_gpu* h) {
  using L = MarchLayout<MODE, PI_, HET, EXT, SH>;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult qr;
  CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr));
  if (!fn || qr != cudaDriverEntryPointSuccess) return set_err(FDMAP_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  EncodeTiledFn enc = (EncodeTiledFn)fn;
  if (!h->tmaps) h->tmaps = new (std::nothrow) TmapSet();
  if (!h->tmaps) return set_err(FDMAP_ERR_NOMEM, "out of host memory");
  std::memset(h->tmaps, 0, sizeof(TmapSet));
  int rc;
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    const BlockGeom& g = h->geom[b];
    const DevBlock& B = h->hdom.blk[b];
    for (int q = 0; q < 2; ++q) {
      if ((rc = encode_map(enc, &h->tmaps->F[b][q], B.F[q], g, h->nF, L::WH, L::MR, L::NR))) return rc;
      if ((rc = encode_map(enc, &h->tmaps->F6[b][q], B.F[q], g, h->nF, L::MW, L::MR, 1))) return rc;
    }
    if ((rc = encode_map(enc, &h->tmaps->DF[b], B.DF, g, h->nF, L::MW, L::MR, L::NR))) return rc;
    if ((rc = encode_map(enc, &h->tmaps->MH[b], h->met_base[b], g, 5, L::WH, L::MR, 2))) return rc;
    if ((rc = encode_map(enc, &h->tmaps->MC[b], h->met_base[b], g, 5, L::MW, L::MR, 3))) return rc;
    if (HET && (rc = encode_map(enc, &h->tmaps->HT[b], h->het_base[b], g, 5, L::MW, L::MR, L::NH))) return rc;
    if (EXT == MARCH_DISS && B.J && B.Cdiss > 0.0 &&
        (rc = encode_map(enc, &h->tmaps->JH[b], B.J, g, 1, L::WH, L::MR, 1)))
      return rc;
  }
  return FDMAP_OK;
}

// FDMAP_ERR_UNSUPPORTED when the shape cannot serve the variant (its rings do
// not fit in shared memory, or a row group is thinner than the stencil's
// half-width, so rows j +- PI would lie outside the three resident groups)
template <int MODE, int PI_, bool HET, int EXT, int SH>
int configure(fdmap_gpu* h) {
  using L = MarchLayout<MODE, PI_, HET, EXT, SH>;
  if (PI_ > L::MR) return set_err(FDMAP_ERR_UNSUPPORTED, "row groups thinner than the stencil");
  int optin = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
  if (L::BYTES > (size_t)optin) return set_err(FDMAP_ERR_UNSUPPORTED, "march rings do not fit in shared memory");
  // units: strips of MW columns x row groups of MR rows, block after block
  long long units = 0;
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    DevBlock& B = h->hdom.blk[b];
    B.march_unit_begin = units;
    if (h->owns(b)) units += (long long)((B.nx + L::MW - 1) / L::MW) * ((B.ny + L::MR - 1) / L::MR);
  }
  h->march_units = units;
  int rc = maps<MODE, PI_, HET, EXT, SH>(h);
  if (rc) return rc;
  auto k = march_kernel<MODE, PI_, HET, EXT, SH>;
  CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES));
  int per_sm = 0, sms = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, L::THREADS, L::BYTES));
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
  if (per_sm < 1) return set_err(FDMAP_ERR_UNSUPPORTED, "march kernel does not fit on an SM");
  h->march_grid = (int)std::max<long long>(1, std::min<long long>((long long)sms * per_sm, units));
  h->march_shape = SH;
  return FDMAP_OK;
}

template <int MODE, int PI_, bool HET, int EXT, int SH>
int launch(fdmap_gpu* h, const StageArgs& a) {
  using L = MarchLayout<MODE, PI_, HET, EXT, SH>;
  MarchPlan plan{h->march_grid, h->march_units, nullptr, nullptr, 1};
  march_kernel<MODE, PI_, HET, EXT, SH><<<h->march_grid, L::THREADS, L::BYTES, h->stream>>>(h->ddom, a, plan, *h->tmaps);
  CUDA_TRY(cudaGetLastError());
  return FDMAP_OK;
}

template <int MODE, int PI_, bool HET, int EXT, int SH>
int launch_batch(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s) {
  using L = MarchLayout<MODE, PI_, HET, EXT, SH>;
  MarchPlan plan{p.march_grid, p.units, p.tmaps, p.unit_begin, p.ninst};
  march_kernel<MODE, PI_, HET, EXT, SH><<<p.march_grid, L::THREADS, L::BYTES, s>>>(p.doms, a, plan, *proto->tmaps);
  CUDA_TRY(cudaGetLastError());
  return FDMAP_OK;
}

// calls fn(mode, pI, het, ext) as compile-time constants for the handle's variant
template <int SH, typename Fn>
int dispatch(const fdmap_gpu* h, Fn&& fn) {
  auto with_pi = [&](auto mode_c, auto het_c, auto ext_c) -> int {
    constexpr int MODE = decltype(mode_c)::value;
    if (h->pI == 1) return fn(mode_c, std::integral_constant<int, 1>{}, het_c, ext_c);
    if (h->pI == 2) return fn(mode_c, std::integral_constant<int, 2>{}, het_c, ext_c);
    if constexpr (shape_mr(SH) >= 3) return fn(mode_c, std::integral_constant<int, 3>{}, het_c, ext_c);
    (void)MODE;
    return set_err(FDMAP_ERR_UNSUPPORTED, "row groups thinner than the stencil");
  };
  auto with_ext = [&](auto mode_c, auto het_c) -> int {
    if (h->march_ext == MARCH_DISS) return with_pi(mode_c, het_c, std::integral_constant<int, MARCH_DISS>{});
    if (h->march_ext == MARCH_PML) return with_pi(mode_c, het_c, std::integral_constant<int, MARCH_PML>{});
    return with_pi(mode_c, het_c, std::integral_constant<int, MARCH_PLAIN>{});
  };
  auto with_het = [&](auto mode_c) -> int {
    return h->het ? with_ext(mode_c, std::true_type{}) : with_ext(mode_c, std::false_type{});
  };
  return h->mode == 2 ? with_het(std::integral_constant<int, 2>{}) : with_het(std::integral_constant<int, 3>{});
}

}  // namespace march_detail

// One tile shape's entry points (defined in march_s<SH>.cu)
template <int SH>
int march_configure_shape(fdmap_gpu* h) {
  return march_detail::dispatch<SH>(h, [&](auto m, auto p, auto het, auto ext) {
    return march_detail::configure<decltype(m)::value, decltype(p)::value, decltype(het)::value,
                                   decltype(ext)::value, SH>(h);
  });
}

template <int SH>
int march_launch_shape(fdmap_gpu* h, const StageArgs& a) {
  return march_detail::dispatch<SH>(h, [&](auto m, auto p, auto het, auto ext) {
    return march_detail::launch<decltype(m)::value, decltype(p)::value, decltype(het)::value, decltype(ext)::value,
                                SH>(h, a);
  });
}

template <int SH>
int march_batch_shape(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& bp, cudaStream_t s) {
  return march_detail::dispatch<SH>(proto, [&](auto m, auto p, auto het, auto ext) {
    return march_detail::launch_batch<decltype(m)::value, decltype(p)::value, decltype(het)::value,
                                      decltype(ext)::value, SH>(proto, a, bp, s);
  });
}

}  // namespace fdmap
