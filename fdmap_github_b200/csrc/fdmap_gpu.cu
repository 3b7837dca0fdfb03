// Host side of the B200 engine: device allocation and layout conversion,
// the RK stage loop (time_step_LS, time_step.f90:71-167) and the C ABI
// declared in include/fdmap_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <cstdlib>
#include <type_traits>
#include <string>
#include <vector>

#include "edge_kernel.cuh"
#include "engine.h"
#include "pml_formula.h"
#include "march_kernel.cuh"
#include "sbp_tables.h"
#include "stencil_kernel.cuh"

using namespace fdmap;

namespace fdmap {
thread_local std::string g_err;

int set_err(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace fdmap

namespace {

// singular_source weights (source.f90:327-406) for the 5 nodes i0-2..i0+2
void source_weights(double h, double a, double* w) {
  double beta = (1.0 - 2.0 * a) / 4.0 + 0.25;
  double gam = (2.0 * a - 1.0) / 16.0;
  double gap = (2.0 * a + 1.0) / 16.0;
  w[0] = (-gam) / h;
  w[1] = (beta + 3.0 * gam - gap) / h;
  w[2] = (1.0 - a - 2.0 * beta - 3.0 * gam + 3.0 * gap) / h;
  w[3] = (a + beta + gam - 3.0 * gap) / h;
  w[4] = (gap) / h;
}

}  // namespace

namespace fdmap {
// global (i fastest, j, field) array <-> padded block planes of one block
__global__ void scatter_block(const double* __restrict__ g, double* __restrict__ dst, int nxg, long long NN, int mgx,
                              int mgy, int nx, int ny, int pitch, long long plane, int nF) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= pitch || j >= ny) return;
  for (int l = 0; l < nF; ++l)
    dst[l * plane + (long long)j * pitch + i] =
        i < nx ? g[l * NN + (long long)(mgy - 1 + j) * nxg + (mgx - 1 + i)] : 0.0;
}
__global__ void gather_block(const double* __restrict__ src, double* __restrict__ g, int nxg, long long NN, int mgx,
                             int mgy, int nx, int ny, int pitch, long long plane, int nF) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= nx || j >= ny) return;
  for (int l = 0; l < nF; ++l)
    g[l * NN + (long long)(mgy - 1 + j) * nxg + (mgx - 1 + i)] = src[l * plane + (long long)j * pitch + i];
}
// end of a replayed step: advance the device step clock
__global__ void advance_step(TimeState* ts) { ts->n += 1; }

// non-finite values among nF planes of nx x ny nodes (row pitch, plane
// stride), added to *count once per warp
__global__ void count_nonfinite_block(const double* __restrict__ F, int nx, int ny, long long pitch, long long plane,
                                      int nF, unsigned long long* count) {
  const long long n = (long long)nF * ny * nx;
  unsigned c = 0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx);
    const long long r = t / nx;
    const int j = (int)(r % ny), l = (int)(r / ny);
    if (!isfinite(F[l * plane + (long long)j * pitch + i])) ++c;
  }
  for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}
// Test kernel for the bounded wait: one CTA waits on a fresh mbarrier that no
// copy or arrival will ever complete, with a short limit, so the wait gives
// up and reports FDMAP_ERR_TIMEOUT through the status word.
__global__ void wait_timeout_probe(unsigned long long* status, unsigned long long limit_ns) {
  __shared__ unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool ok = mbar_wait_bounded(&bar, 0, status, limit_ns);
  __syncthreads();
  if (threadIdx.x == 0 && ok) atomicOr(&status[1], 4ull);  // would mean a phase completed with no arrival
}

// start of a replayed sequence: set the step clock (by value, no host buffer to keep alive)
__global__ void set_step_clock(TimeState* ts, double t_start, double dt, long long n) {
  ts->t_start = t_start;
  ts->dt = dt;
  ts->n = n;
}
}  // namespace fdmap


namespace {

struct ProfScope {
  fdmap_gpu* h;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(fdmap_gpu* h_, int kind_) : h(h_), kind(kind_) {
    if (h->profiling) { a = h->take_event(); b = h->take_event(); cudaEventRecord(a, h->stream); }
  }
  ~ProfScope() {
    if (a) { cudaEventRecord(b, h->stream); h->ev_pending.push_back({kind, {a, b}}); }
  }
};

int launch_edges(fdmap_gpu* h, const StageArgs& a) {
  if (h->edge_threads == 0) return FDMAP_OK;
  int tpb = 64;
  int nb = (h->edge_threads + tpb - 1) / tpb;
  ProfScope ps(h, 2);
  if (h->mode == 2) edge_kernel<2><<<nb, tpb, 0, h->stream>>>(h->hdom, a);
  else edge_kernel<3><<<nb, tpb, 0, h->stream>>>(h->hdom, a);
  h->launches++;
  CUDA_TRY(cudaGetLastError());
  return FDMAP_OK;
}

template <int MODE>
void launch_stencil_mode(fdmap_gpu* h, const StageArgs& a) {
  dim3 grid(h->total_tiles), block(TX * TY);
  if (h->het) {
    if (h->pI == 1) stencil_kernel<MODE, 1, true><<<grid, block, 0, h->stream>>>(h->ddom, a);
    else if (h->pI == 2) stencil_kernel<MODE, 2, true><<<grid, block, 0, h->stream>>>(h->ddom, a);
    else stencil_kernel<MODE, 3, true><<<grid, block, 0, h->stream>>>(h->ddom, a);
  } else {
    if (h->pI == 1) stencil_kernel<MODE, 1, false><<<grid, block, 0, h->stream>>>(h->ddom, a);
    else if (h->pI == 2) stencil_kernel<MODE, 2, false><<<grid, block, 0, h->stream>>>(h->ddom, a);
    else stencil_kernel<MODE, 3, false><<<grid, block, 0, h->stream>>>(h->ddom, a);
  }
}

template <int MODE, bool HET, typename Fn>
int dispatch_pi(int pI, Fn&& fn) {
  if (pI == 1) return fn(std::integral_constant<int, 1>{});
  if (pI == 2) return fn(std::integral_constant<int, 2>{});
  return fn(std::integral_constant<int, 3>{});
}

int march_dispatch(fdmap_gpu* h, const StageArgs& a) {
  switch (h->march_shape) {
    case 0: return march_launch_s0(h, a);
    case 1: return march_launch_s1(h, a);
    case 2: return march_launch_s2(h, a);
    default: return march_launch_s3(h, a);
  }
}

int march_configure(fdmap_gpu* h, int shape) {
  switch (shape) {
    case 0: return march_configure_s0(h);
    case 1: return march_configure_s1(h);
    case 2: return march_configure_s2(h);
    case 3: return march_configure_s3(h);
  }
  return set_err(FDMAP_ERR_INVALID_ARG, "march tile shape must be 0..3");
}

int launch_stage(fdmap_gpu* h, const StageArgs& a);

// (mode, SBP half-width, heterogeneity) of a handle as compile-time constants
template <typename Fn>
int dispatch_variant(const fdmap_gpu* h, Fn&& fn) {
  auto go = [&](auto mode_c, auto het_c) {
    return dispatch_pi<decltype(mode_c)::value, decltype(het_c)::value>(
        h->pI, [&](auto pi_c) { return fn(mode_c, pi_c, het_c); });
  };
  if (h->mode == 2) return h->het ? go(std::integral_constant<int, 2>{}, std::true_type{}) : go(std::integral_constant<int, 2>{}, std::false_type{});
  return h->het ? go(std::integral_constant<int, 3>{}, std::true_type{}) : go(std::integral_constant<int, 3>{}, std::false_type{});
}

}  // namespace

namespace fdmap {

int engine_stage(fdmap_gpu* h, const StageArgs& a) { return launch_stage(h, a); }

int batch_march(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s) {
  switch (proto->march_shape) {
    case 0: return march_batch_s0(proto, a, p, s);
    case 1: return march_batch_s1(proto, a, p, s);
    case 2: return march_batch_s2(proto, a, p, s);
    default: return march_batch_s3(proto, a, p, s);
  }
}

int state_snapshot(fdmap_gpu* h, std::vector<void*>& out, cudaStream_t s) {
  out.clear();
  for (size_t q = 0; q < h->allocs.size(); ++q) {
    void* d = nullptr;
    if (cudaMalloc(&d, h->alloc_sizes[q]) != cudaSuccess) {
      for (void* p : out) cudaFree(p);
      out.clear();
      return set_err(FDMAP_ERR_NOMEM, "no device memory for the tuning snapshot");
    }
    out.push_back(d);
    CUDA_TRY(cudaMemcpyAsync(d, h->allocs[q], h->alloc_sizes[q], cudaMemcpyDeviceToDevice, s));
  }
  return FDMAP_OK;
}

int state_restore(fdmap_gpu* h, std::vector<void*>& saved, cudaStream_t s) {
  int rc = FDMAP_OK;
  for (size_t q = 0; q < saved.size() && q < h->allocs.size(); ++q)
    if (cudaMemcpyAsync(h->allocs[q], saved[q], h->alloc_sizes[q], cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      rc = set_err(FDMAP_ERR_CUDA, "restoring the tuning snapshot failed");
  if (cudaStreamSynchronize(s) != cudaSuccess && !rc) rc = set_err(FDMAP_ERR_CUDA, "restoring the tuning snapshot failed");
  for (void* p : saved) cudaFree(p);
  saved.clear();
  return rc;
}

int march_set_shape(fdmap_gpu* h, int shape) {
  if (!h->use_march) return set_err(FDMAP_ERR_UNSUPPORTED, "the domain does not use the march kernel");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  const int keep = h->march_shape;
  int rc = march_configure(h, shape);
  if (rc) {
    std::string msg = g_err;
    march_configure(h, keep);  // back to the shape in use
    g_err = msg;
    return rc;
  }
  CUDA_TRY(cudaMemcpy(h->ddom, &h->hdom, sizeof(DevDomain), cudaMemcpyHostToDevice));
  for (auto& ge : h->step_graph)
    if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  h->graph_dt = 0.0;
  return FDMAP_OK;
}

int batch_closure(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s) {
  if (p.closure_ctas == 0) return FDMAP_OK;
  return dispatch_variant(proto, [&](auto mode_c, auto pi_c, auto het_c) {
    constexpr int MODE = decltype(mode_c)::value;
    constexpr int PI_ = decltype(pi_c)::value;
    constexpr bool HET = decltype(het_c)::value;
    if (proto->march_ext == 0 && !proto->dissipation && !proto->pml && !proto->forcing && !proto->extras)
      closure_kernel_batch<MODE, PI_, HET, true><<<p.closure_ctas, p.closure_tpb, 0, s>>>(p.doms, p.closure_cta_begin,
                                                                                        p.ninst, a);
    else
      closure_kernel_batch<MODE, PI_, HET><<<p.closure_ctas, p.closure_tpb, 0, s>>>(p.doms, p.closure_cta_begin,
                                                                                  p.ninst, a);
    CUDA_TRY(cudaGetLastError());
    return (int)FDMAP_OK;
  });
}

int batch_edges(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s) {
  if (p.edge_ctas == 0) return FDMAP_OK;
  if (proto->mode == 2) edge_kernel_batch<2><<<p.edge_ctas, p.edge_tpb, 0, s>>>(p.doms, p.edge_cta_begin, p.ninst, a);
  else edge_kernel_batch<3><<<p.edge_ctas, p.edge_tpb, 0, s>>>(p.doms, p.edge_cta_begin, p.ninst, a);
  CUDA_TRY(cudaGetLastError());
  return FDMAP_OK;
}

}  // namespace fdmap

namespace {

// 64-thread closure CTAs (two warps, capped at BOUNDARY_REGS registers a
// thread) fit beside a resident march CTA
constexpr int CLOSURE_TPB = 64;

// a domain without PML, dissipation, forcing and body extras: the closure
// kernel without those branches
bool plain_domain(const fdmap_gpu* h) { return !h->dissipation && !h->pml && !h->forcing && !h->extras; }

template <int MODE>
void launch_closure_mode(fdmap_gpu* h, const StageArgs& a) {
  const int t = CLOSURE_TPB;
  int nb = (int)((h->closure_threads + t - 1) / t);
  if (plain_domain(h)) {
    if (h->het) {
      if (h->pI == 1) closure_kernel<MODE, 1, true, true><<<nb, t, 0, h->stream>>>(h->hdom, a);
      else if (h->pI == 2) closure_kernel<MODE, 2, true, true><<<nb, t, 0, h->stream>>>(h->hdom, a);
      else closure_kernel<MODE, 3, true, true><<<nb, t, 0, h->stream>>>(h->hdom, a);
    } else {
      if (h->pI == 1) closure_kernel<MODE, 1, false, true><<<nb, t, 0, h->stream>>>(h->hdom, a);
      else if (h->pI == 2) closure_kernel<MODE, 2, false, true><<<nb, t, 0, h->stream>>>(h->hdom, a);
      else closure_kernel<MODE, 3, false, true><<<nb, t, 0, h->stream>>>(h->hdom, a);
    }
    return;
  }
  if (h->het) {
    if (h->pI == 1) closure_kernel<MODE, 1, true><<<nb, t, 0, h->stream>>>(h->hdom, a);
    else if (h->pI == 2) closure_kernel<MODE, 2, true><<<nb, t, 0, h->stream>>>(h->hdom, a);
    else closure_kernel<MODE, 3, true><<<nb, t, 0, h->stream>>>(h->hdom, a);
  } else {
    if (h->pI == 1) closure_kernel<MODE, 1, false><<<nb, t, 0, h->stream>>>(h->hdom, a);
    else if (h->pI == 2) closure_kernel<MODE, 2, false><<<nb, t, 0, h->stream>>>(h->hdom, a);
    else closure_kernel<MODE, 3, false><<<nb, t, 0, h->stream>>>(h->hdom, a);
  }
}

// The boundary kernels run beside the persistent march CTAs, which configure
// their SMs for the largest shared-memory carveout; a kernel launched with
// another carveout preference is not placed on an SM configured otherwise, so
// without this the boundary CTAs would wait for the march CTAs to retire.
template <int MODE>
int boundary_carveout_mode() {
  const void* ks[] = {
      (const void*)edge_kernel<MODE>, (const void*)edge_kernel_batch<MODE>, (const void*)pack_edges<MODE>,
      (const void*)closure_kernel<MODE, 1, false>, (const void*)closure_kernel<MODE, 2, false>,
      (const void*)closure_kernel<MODE, 3, false>, (const void*)closure_kernel<MODE, 1, true>,
      (const void*)closure_kernel<MODE, 2, true>, (const void*)closure_kernel<MODE, 3, true>,
      (const void*)closure_kernel_batch<MODE, 1, false>, (const void*)closure_kernel_batch<MODE, 2, false>,
      (const void*)closure_kernel_batch<MODE, 3, false>, (const void*)closure_kernel_batch<MODE, 1, true>,
      (const void*)closure_kernel_batch<MODE, 2, true>, (const void*)closure_kernel_batch<MODE, 3, true>,
      (const void*)closure_kernel<MODE, 1, false, true>, (const void*)closure_kernel<MODE, 2, false, true>,
      (const void*)closure_kernel<MODE, 3, false, true>, (const void*)closure_kernel<MODE, 1, true, true>,
      (const void*)closure_kernel<MODE, 2, true, true>, (const void*)closure_kernel<MODE, 3, true, true>,
      (const void*)closure_kernel_batch<MODE, 1, false, true>, (const void*)closure_kernel_batch<MODE, 2, false, true>,
      (const void*)closure_kernel_batch<MODE, 3, false, true>, (const void*)closure_kernel_batch<MODE, 1, true, true>,
      (const void*)closure_kernel_batch<MODE, 2, true, true>, (const void*)closure_kernel_batch<MODE, 3, true, true>,
  };
  for (const void* k : ks)
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
  return FDMAP_OK;
}

template <int MODE>
void launch_boundary_mode(fdmap_gpu* h, const StageArgs& a) {
  long long items = h->edge_threads + h->closure_threads;
  int nb = (int)((items + 127) / 128);
  if (h->het) {
    if (h->pI == 1) boundary_kernel<MODE, 1, true><<<nb, 128, 0, h->stream>>>(h->hdom, a);
    else if (h->pI == 2) boundary_kernel<MODE, 2, true><<<nb, 128, 0, h->stream>>>(h->hdom, a);
    else boundary_kernel<MODE, 3, true><<<nb, 128, 0, h->stream>>>(h->hdom, a);
  } else {
    if (h->pI == 1) boundary_kernel<MODE, 1, false><<<nb, 128, 0, h->stream>>>(h->hdom, a);
    else if (h->pI == 2) boundary_kernel<MODE, 2, false><<<nb, 128, 0, h->stream>>>(h->hdom, a);
    else boundary_kernel<MODE, 3, false><<<nb, 128, 0, h->stream>>>(h->hdom, a);
  }
}

// one stage.  Boundary work first -- with no multi-interface junction nodes a
// single boundary kernel (interface solves and closure strips are
// independent items); otherwise interface solves, then closure strips (which
// read the interface hat variables) -- then the interior.  All of them read
// F[in] and write disjoint nodes.
int launch_interior(fdmap_gpu* h, const StageArgs& a) {
  ProfScope ps(h, 0);
  if (h->use_march) {
    int rc = march_dispatch(h, a);
    if (rc) return rc;
  } else if (h->mode == 2) launch_stencil_mode<2>(h, a);
  else launch_stencil_mode<3>(h, a);
  h->launches++;
  CUDA_TRY(cudaGetLastError());
  return FDMAP_OK;
}

int launch_boundary(fdmap_gpu* h, const StageArgs& a) {
  int rc = launch_edges(h, a);
  if (rc) return rc;
  ProfScope pc(h, 1);
  if (h->mode == 2) launch_closure_mode<2>(h, a);
  else launch_closure_mode<3>(h, a);
  h->launches++;
  CUDA_TRY(cudaGetLastError());
  return FDMAP_OK;
}

bool stage_overlaps(const fdmap_gpu* h) { return h->overlap && !h->profiling && !h->fused; }

// stream of the stage's boundary work (interface solves, closure strips)
cudaStream_t boundary_stream(const fdmap_gpu* h) { return stage_overlaps(h) ? h->side_stream : h->stream; }

// Partitioned domain: the edge values of this stage's input buffer for every
// interface with one side on a peer GPU, into the stage's send slot.
int pack_partition_edges(fdmap_gpu* h, const StageArgs& a, cudaStream_t s) {
  for (int k : h->part_ifaces) {
    DevDomain& D = h->hdom;
    DevIface& I = D.ifc[k];
    double* slot0 = I.send;
    I.send = slot0 + (size_t)(h->xstage & 1) * h->nF * I.n;
    const int nb = (I.n + 127) / 128;
    if (h->mode == 2) pack_edges<2><<<nb, 128, 0, s>>>(D, a.in, k);
    else pack_edges<3><<<nb, 128, 0, s>>>(D, a.in, k);
    I.send = slot0;
    h->launches++;
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaEventRecord(h->ev_packed, s));
  return FDMAP_OK;
}

// First half of a stage: with overlap, fork and issue the interior march on
// the (high-priority) main stream, so its persistent CTAs take the SMs; then
// the partition's edge values are packed on the boundary stream.
int stage_begin(fdmap_gpu* h, const StageArgs& a) {
  if (stage_overlaps(h)) {
    CUDA_TRY(cudaEventRecord(h->ev_fork, h->stream));
    CUDA_TRY(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
    int rc = launch_interior(h, a);
    if (rc) return rc;
  }
  if (!h->part_ifaces.empty()) return pack_partition_edges(h, a, boundary_stream(h));
  return FDMAP_OK;
}

// Second half, after the peers' edge values have been queued on the boundary
// stream: edge + closure on the side stream (filling the registers the march
// leaves free) and join; or, serialised, boundary work then the interior.
int stage_end(fdmap_gpu* h, const StageArgs& a) {
  if (stage_overlaps(h)) {
    cudaStream_t main_stream = h->stream;
    h->stream = h->side_stream;
    int rc = launch_boundary(h, a);
    h->stream = main_stream;
    if (rc) return rc;
    CUDA_TRY(cudaEventRecord(h->ev_join, h->side_stream));
    CUDA_TRY(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    return FDMAP_OK;
  }
  if (h->fused) {
    ProfScope pc(h, 1);
    if (h->mode == 2) launch_boundary_mode<2>(h, a);
    else launch_boundary_mode<3>(h, a);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
  } else {
    int rc = launch_boundary(h, a);
    if (rc) return rc;
  }
  return launch_interior(h, a);
}

// One stage of a single handle: with a partition, the caller's exchange
// callback queues the transfer of the peers' edge values between the halves.
int launch_stage(fdmap_gpu* h, const StageArgs& a) {
  int rc = stage_begin(h, a);
  if (rc) return rc;
  if (!h->part_ifaces.empty()) {
    if (!h->exchange) return set_err(FDMAP_ERR_INVALID_ARG, "partitioned domain without an exchange callback");
    rc = h->exchange(h->exchange_user, h->xstage, (void*)boundary_stream(h));
    if (rc) return set_err(FDMAP_ERR_CUDA, "edge exchange callback failed (" + std::to_string(rc) + ")");
  }
  h->xstage++;
  return stage_end(h, a);
}

// reads the next forcing frame into the blocks' new-frame planes (values past
// the end of the file read as zero)
int forcing_read_frame(fdmap_gpu* h) {
  const int nF = h->nF;
  const long long NN = (long long)h->nx_g * h->ny_g;
  h->frc_host.assign((size_t)NN * nF, 0.0);
  size_t got = std::fread(h->frc_host.data(), sizeof(double), h->frc_host.size(), h->frc_file);
  (void)got;
  CUDA_TRY(cudaMemcpyAsync(h->d_global, h->frc_host.data(), h->frc_host.size() * sizeof(double),
                           cudaMemcpyHostToDevice, h->stream));
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    const BlockGeom& g = h->geom[b];
    dim3 grid((g.pitch + 255) / 256, g.ny);
    scatter_block<<<grid, 256, 0, h->stream>>>(h->d_global, const_cast<double*>(h->hdom.blk[b].frc_new), h->nx_g, NN,
                                               g.mgx, g.mgy, g.nx, g.ny, g.pitch, g.plane, nF);
    CUDA_TRY(cudaGetLastError());
    h->launches++;
  }
  return FDMAP_OK;
}

// load_forcing (source.f90:467-502), at the start of every step: the new frame
// becomes the old one and the next frame is read
int forcing_load(fdmap_gpu* h) {
  if (!h->frc_file) return FDMAP_OK;
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    const DevBlock& B = h->hdom.blk[b];
    CUDA_TRY(cudaMemcpyAsync(const_cast<double*>(B.frc_old), B.frc_new, (size_t)h->nF * B.plane * sizeof(double),
                             cudaMemcpyDeviceToDevice, h->stream));
  }
  return forcing_read_frame(h);
}

int validate(const fdmap_desc* d) {
  if (!d) return set_err(FDMAP_ERR_INVALID_ARG, "null descriptor");
  if (d->mode != 2 && d->mode != 3) return set_err(FDMAP_ERR_INVALID_ARG, "mode must be 2 or 3");
  if (d->nF != (d->mode == 2 ? 6 : 3)) return set_err(FDMAP_ERR_INVALID_ARG, "nF does not match mode");
  if (d->nblocks < 1 || d->nblocks > MAX_BLOCKS) return set_err(FDMAP_ERR_UNSUPPORTED, "1..16 blocks supported");
  if (d->nifaces < 0 || d->nifaces > MAX_IFACES) return set_err(FDMAP_ERR_UNSUPPORTED, "at most 32 interfaces supported");
  const bool dev_body = d->body != nullptr;
  if (!dev_body && (!d->F || !d->DF || !d->xq || !d->xr || !d->yq || !d->yr || !d->Ji))
    return set_err(FDMAP_ERR_INVALID_ARG, "missing body arrays");
  if (dev_body && !d->body->blocks) return set_err(FDMAP_ERR_INVALID_ARG, "missing block body recipes");
  if (d->src.gauss_forcing && d->mode == 3 && (!d->x || !d->y))
    return set_err(dev_body ? FDMAP_ERR_UNSUPPORTED : FDMAP_ERR_INVALID_ARG,
                   "the tsunami forcing needs the grid coordinates on the host");
  if (d->heterogeneous && (!d->rho || !d->G || (d->mode == 2 && (!d->M || !d->gamma || !d->nu))))
    return set_err(FDMAP_ERR_INVALID_ARG, "missing heterogeneous material arrays");
  fdmap::SbpOperator op;
  if (!fdmap::sbp_operator(d->fd_method, &op)) return set_err(FDMAP_ERR_UNSUPPORTED, "unknown FD method");
  for (int b = 0; b < d->nblocks; ++b) {
    const fdmap_block& B = d->blocks[b];
    int nx = B.pgx - B.mgx + 1, ny = B.pgy - B.mgy + 1;
    if (B.mgx < 1 || B.mgy < 1 || B.pgx > d->nx || B.pgy > d->ny)
      return set_err(FDMAP_ERR_INVALID_ARG, "block index limits outside the domain");
    // in a heterogeneous medium the dissipative rates scale by the node's
    // material (rates_h_dissipation_*) and the PML rates keep the block's
    // homogeneous material (time_step.f90:354-420): both kernels cover that
    if (!dev_body && B.Cdiss > 0.0 && !d->J)
      return set_err(FDMAP_ERR_INVALID_ARG, "artificial dissipation needs the Jacobian array J");
    if (d->mode == 2 && (B.pmlx || B.pmly) && B.Cdiss == 0.0 && !(dev_body && d->body->blocks[b].Cdiss > 0.0)) {
      if (!dev_body && B.pml_n > 0.0 && (!d->x || !d->y))
        return set_err(FDMAP_ERR_INVALID_ARG, "the PML profile needs x and y");
    }
    if (nx < 2 * op.nbst || ny < 2 * op.nbst || nx < op.nbnd || ny < op.nbnd)
      return set_err(FDMAP_ERR_UNSUPPORTED, "block too small for the SBP boundary closures");
    for (int s = 0; s < 4; ++s) {
      const fdmap_side& S = B.side[s];
      if (S.n != (s < 2 ? ny : nx)) return set_err(FDMAP_ERR_INVALID_ARG, "side length mismatch");
      if ((!S.M && !dev_body) || !S.F0 || !S.normal) return set_err(FDMAP_ERR_INVALID_ARG, "missing side arrays");
      if (dev_body && (!S.x || !S.y)) return set_err(FDMAP_ERR_INVALID_ARG, "missing side coordinates");
      if (d->mode == 3 && S.bc != FDMAP_BC_NONE && S.bc != FDMAP_BC_ABSORBING && S.bc != FDMAP_BC_FREE &&
          S.bc != FDMAP_BC_RIGID)
        return set_err(FDMAP_ERR_UNSUPPORTED, "boundary condition not available in mode III");
    }
  }
  for (int k = 0; k < d->nifaces; ++k) {
    const fdmap_iface& I = d->ifaces[k];
    if (I.iblockm < 0 || I.iblockm >= d->nblocks || I.iblockp < 0 || I.iblockp >= d->nblocks || I.p < I.m)
      return set_err(FDMAP_ERR_INVALID_ARG, "bad interface description");
    if (I.coupling == FDMAP_COUPLING_FRICTION) {
      const fdmap_friction& fr = I.fr;
      if (!fr.V || !fr.O || !fr.S || !fr.N || !fr.S0 || !fr.N0 || !fr.Ds || !fr.Dn || !fr.DDs || !fr.DDn ||
          !fr.Psi || !fr.DPsi || !fr.D || !fr.trup || !fr.W || !fr.DW || !fr.Nreg || !fr.DNreg)
        return set_err(FDMAP_ERR_INVALID_ARG, "missing friction state arrays");
      if (fr.law >= FDMAP_FR_SL && (!fr.a || !fr.b || !fr.V0 || !fr.f0 || !fr.L || !fr.fw || !fr.Vw))
        return set_err(FDMAP_ERR_INVALID_ARG, "missing rate-and-state parameters");
      if (fr.law == FDMAP_FR_SW && (!fr.c0 || !fr.fs || !fr.fd || !fr.Dc))
        return set_err(FDMAP_ERR_INVALID_ARG, "missing slip-weakening parameters");
    }
  }
  return FDMAP_OK;
}

int build(fdmap_gpu* h, const fdmap_desc* d) {
  DevDomain& D = h->hdom;
  std::memset(&D, 0, sizeof(D));
  fdmap::SbpOperator op;
  fdmap::sbp_operator(d->fd_method, &op);
  fdmap::rk_table(d->rk_order, &h->rk);
  if (h->rk.nstage == 0) return set_err(FDMAP_ERR_INVALID_ARG, "Invalid Runge-Kutta order");
  h->mode = d->mode; h->nF = d->nF; h->pI = op.pI; h->het = d->heterogeneous;
  h->nx_g = d->nx; h->ny_g = d->ny;
  D.mode = d->mode; D.nF = d->nF; D.nblocks = d->nblocks; D.nifaces = d->nifaces; D.het = d->heterogeneous;
  D.nbst = op.nbst; D.nbnd = op.nbnd; D.pI = op.pI;
  for (int s = 0; s <= op.pI; ++s) D.DI[s] = op.DI[s];
  for (int r = 0; r < op.nbst; ++r)
    for (int s = 0; s < op.nbnd; ++s) D.DL[r][s] = op.DL[r][s];
  for (int s = 0; s <= op.pI; ++s) D.AI[s] = op.AI[s];
  for (int r = 0; r < op.nbst; ++r)
    for (int s = 0; s < op.nbnd; ++s) D.AL[r][s] = op.AL[r][s];
  D.src = d->src;
  const int nF = d->nF;
  int tiles = 0;
  h->geom.resize(d->nblocks);
  for (int b = 0; b < d->nblocks; ++b) {
    const fdmap_block& fb = d->blocks[b];
    DevBlock& B = D.blk[b];
    BlockGeom& g = h->geom[b];
    g.mgx = fb.mgx; g.mgy = fb.mgy;
    g.nx = fb.pgx - fb.mgx + 1; g.ny = fb.pgy - fb.mgy + 1;
    g.pitch = (g.nx + 31) / 32 * 32;
    g.plane = ((long long)g.pitch * g.ny + PADTAIL + 31) / 32 * 32;
    B.nx = g.nx; B.ny = g.ny; B.pitch = g.pitch; B.plane = g.plane;
    int rc;
    // a block another GPU owns (block-aligned partition): no body arrays
    // here, only its side arrays, which the interface solve writes
    const bool own = h->owns(b);
    if (own) {
      for (int q = 0; q < 2; ++q)
        if ((rc = h->alloc_planes(&B.F[q], nF, g.plane))) return rc;
      if ((rc = h->alloc_planes(&B.DF, nF, g.plane))) return rc;
      // metric terms as 5 consecutive planes yr, xr, yq, xq, Ji (one TMA tensor)
      double* met_base = nullptr;
      if ((rc = h->alloc_planes(&met_base, 5, g.plane))) return rc;
      double** met[5] = {&B.yr, &B.xr, &B.yq, &B.xq, &B.Ji};
      const double* msrc[5] = {d->yr, d->xr, d->yq, d->xq, d->Ji};
      for (int q = 0; q < 5; ++q) {
        *met[q] = met_base + (size_t)q * g.plane;
        if (!d->body && (rc = h->upload_plane(*met[q], msrc[q], g))) return rc;
      }
      h->met_base[b] = met_base;
      if (d->heterogeneous) {
        double* het_base = nullptr;
        if ((rc = h->alloc_planes(&het_base, 5, g.plane))) return rc;
        double** hm[5] = {&B.rho, &B.G, &B.M, &B.gamma, &B.nu};
        const double* hs[5] = {d->rho, d->G, d->M, d->gamma, d->nu};
        for (int q = 0; q < 5; ++q) {
          *hm[q] = het_base + (size_t)q * g.plane;
          if (hs[q] && (rc = h->upload_plane(*hm[q], hs[q], g))) return rc;
        }
        h->het_base[b] = het_base;
      }
      B.rho_b = fb.rho; B.G_b = fb.G; B.M_b = fb.M; B.gamma_b = fb.gamma; B.nu_b = fb.nu;
      B.Cdiss = fb.Cdiss;  // on-device body: scaled by build_body once dt is known
      B.J = nullptr;
      const double cdiss_in = d->body ? d->body->blocks[b].Cdiss : fb.Cdiss;
      if (cdiss_in > 0.0 || d->energy_balance) {  // dissipation and the energy weight nodes by J itself
        if ((rc = h->alloc_planes(&B.J, 1, g.plane))) return rc;
        if (!d->body && (rc = h->upload_plane(B.J, d->J, g))) return rc;
        if (cdiss_in > 0.0) h->dissipation = true;
      }
      B.Hx = B.Hy = nullptr;
      if (d->energy_balance) {
        // diagonal norm with unit spacing (Hnorm, fd.f90:14-39)
        std::vector<double> hx(g.nx, 1.0), hy(g.ny, 1.0);
        for (int k = 0; k < op.nbst; ++k) {
          hx[k] = op.HL[k]; hx[g.nx - 1 - k] = op.HL[k];
          hy[k] = op.HL[k]; hy[g.ny - 1 - k] = op.HL[k];
        }
        double *dx = nullptr, *dy = nullptr;
        if ((rc = h->upload(&dx, hx.data(), hx.size())) || (rc = h->upload(&dy, hy.data(), hy.size()))) return rc;
        B.Hx = dx; B.Hy = dy;
      }
      B.pml = 0; B.pml_kappa = 0.0; B.pml_h = nullptr; B.pml_s = nullptr;
      B.Wx = B.DWx = B.Wy = B.DWy = nullptr;
      if (d->mode == 2 && (fb.pmlx || fb.pmly) && cdiss_in == 0.0) {
        // perfectly matched layer (set_rates PML branch, time_step.f90:354-420)
        B.pml = (fb.pmlx ? 1 : 0) | (fb.pmly ? 2 : 0);
        B.pml_kappa = fb.pml_kappa;
        if (fb.pmlx && ((rc = h->alloc_planes(&B.Wx, nF, g.plane)) || (rc = h->alloc_planes(&B.DWx, nF, g.plane))))
          return rc;
        if (fb.pmly && ((rc = h->alloc_planes(&B.Wy, nF, g.plane)) || (rc = h->alloc_planes(&B.DWy, nF, g.plane))))
          return rc;
        // damping at every node (rates.f90:2065-2068), evaluated once: here from
        // the host grid, or by build_body from the device grid
        double* ds = nullptr;
        if ((rc = h->alloc_planes(&ds, 2, g.plane))) return rc;
        double* dh = nullptr;
        if ((rc = h->alloc(&dh, 18))) return rc;
        if (!d->body) {
          std::vector<double> damp(2 * (size_t)g.plane, 0.0);
          for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
              const size_t q = (size_t)(g.mgx - 1 + i) + (size_t)d->nx * (size_t)(g.mgy - 1 + j);
              const bool prof = fb.pml_n > 0.0;
              damp[(size_t)j * g.pitch + i] = pml_damping(fb.pml_sigma, fb.pml_n, fb.pml_mx, fb.pml_px, prof ? d->x[q] : 0.0);
              damp[(size_t)g.plane + (size_t)j * g.pitch + i] =
                  pml_damping(fb.pml_sigma, fb.pml_n, fb.pml_my, fb.pml_py, prof ? d->y[q] : 0.0);
            }
          CUDA_TRY(cudaMemcpy(ds, damp.data(), damp.size() * sizeof(double), cudaMemcpyHostToDevice));
          // hxi = Ji*yr, hyi = Ji*xq at the first node of each region: q and r
          // index 0 = minus-end strip, 1 = plus-end strip, 2 = interior
          double hh[18];
          const int qi[3] = {0, g.nx - op.nbst, op.nbst}, rj[3] = {0, g.ny - op.nbst, op.nbst};
          for (int q = 0; q < 3; ++q)
            for (int r = 0; r < 3; ++r) {
              const size_t k = (size_t)(g.mgx - 1 + qi[q]) + (size_t)d->nx * (size_t)(g.mgy - 1 + rj[r]);
              hh[(q * 3 + r) * 2] = d->Ji[k] * d->yr[k];
              hh[(q * 3 + r) * 2 + 1] = d->Ji[k] * d->xq[k];
            }
          CUDA_TRY(cudaMemcpy(dh, hh, sizeof(hh), cudaMemcpyHostToDevice));
        }
        B.pml_s = ds;
        B.pml_h = dh;
        h->pml = true;
      }
      B.gforce = nullptr; B.frc_old = nullptr; B.frc_new = nullptr;
      if (d->src.gauss_forcing && d->mode == 3) {
        // spatial factor amp*exp(-(x/sigma)^2/2 - (y/sigma)^2/2) of the tsunami forcing (source.f90:308)
        const fdmap_source& S = d->src;
        std::vector<double> gf((size_t)g.plane, 0.0);
        for (int j = 0; j < g.ny; ++j)
          for (int i = 0; i < g.nx; ++i) {
            const size_t q = (size_t)(g.mgx - 1 + i) + (size_t)d->nx * (size_t)(g.mgy - 1 + j);
            const double x = d->x[q], y = d->y[q];
            gf[(size_t)j * g.pitch + i] =
                S.gauss_amp * std::exp(-0.5 * ((x / S.gauss_sigma) * (x / S.gauss_sigma)) -
                                       0.5 * ((y / S.gauss_sigma) * (y / S.gauss_sigma)));
          }
        double* dg = nullptr;
        if ((rc = h->alloc_planes(&dg, 1, g.plane))) return rc;
        CUDA_TRY(cudaMemcpy(dg, gf.data(), gf.size() * sizeof(double), cudaMemcpyHostToDevice));
        B.gforce = dg;
        h->forcing = true;
      }
      if (d->src.forcing_filename) {
        double* fo = nullptr;
        double* fn = nullptr;
        if ((rc = h->alloc_planes(&fo, nF, g.plane)) || (rc = h->alloc_planes(&fn, nF, g.plane))) return rc;
        B.frc_old = fo;
        B.frc_new = fn;
        h->forcing = true;
      }
      B.U = B.DU = B.Utap = B.pgv = B.pga = nullptr;
      if (d->displacement) {
        // U = 0, DU = 1e40 (fields.f90:183-186)
        const int nU = d->mode == 2 ? 2 : 1;
        if ((rc = h->alloc_planes(&B.U, nU, g.plane)) || (rc = h->alloc_planes(&B.DU, nU, g.plane)) ||
            (rc = h->alloc_planes(&B.Utap, nU, g.plane)))
          return rc;
        std::vector<double> big((size_t)nU * g.plane, 1e40);
        CUDA_TRY(cudaMemcpy(B.DU, big.data(), big.size() * sizeof(double), cudaMemcpyHostToDevice));
        h->extras = true;
      }
      if (d->peak) {
        if ((rc = h->alloc_planes(&B.pgv, 1, g.plane)) || (rc = h->alloc_planes(&B.pga, 1, g.plane))) return rc;
        h->extras = true;
      }
    }
    B.rinv_b = 1.0 / fb.rho;
    for (int s = 1; s <= op.pI; ++s) {
      B.coef[s][0] = op.DI[s] / fb.rho;
      B.coef[s][1] = op.DI[s] * fb.G;
      B.coef[s][2] = op.DI[s] * fb.M;
    }
    for (int q = 0; q < 9; ++q) B.F0v[q] = fb.F0[q];
    for (int s = 0; s < 4; ++s) {
      const fdmap_side& fs = fb.side[s];
      DevSide& S = B.side[s];
      S.bc = fs.bc; S.n = fs.n; S.cov_lo = 0; S.cov_hi = 0;
      if (d->body) {
        if ((rc = h->alloc(&S.M, (size_t)fs.n * 5))) return rc;
      } else if ((rc = h->upload(&S.M, fs.M, (size_t)fs.n * 5))) {
        return rc;
      }
      if ((rc = h->upload(&S.F0, fs.F0, (size_t)fs.n * nF))) return rc;
      if ((rc = h->upload(&S.nrm, fs.normal, (size_t)fs.n * 2))) return rc;
      if ((rc = h->alloc(&S.Fhat, (size_t)fs.n * nF))) return rc;
      std::vector<double> big((size_t)fs.n * nF, 1e40);  // fields.f90:850 sentinel
      CUDA_TRY(cudaMemcpy(S.Fhat, big.data(), big.size() * sizeof(double), cudaMemcpyHostToDevice));
      h->dev_fhat[b][s] = S.Fhat;
      h->side_n[b][s] = fs.n;
      // boundary displacement U = 0 and its rate DU = 1e40 (init_fields_side, fields.f90:854-856)
      const size_t nu = (size_t)fs.n * (d->mode == 2 ? 2 : 1);
      if ((rc = h->alloc(&S.U, nu)) || (rc = h->alloc(&S.DU, nu)) || (rc = h->alloc(&S.Utap, nu))) return rc;
      CUDA_TRY(cudaMemset(S.U, 0, nu * sizeof(double)));
      CUDA_TRY(cudaMemset(S.Utap, 0, nu * sizeof(double)));
      CUDA_TRY(cudaMemcpy(S.DU, big.data(), nu * sizeof(double), cudaMemcpyHostToDevice));
    }
    B.src_ok = 0;
    if (d->src.use_singular && fb.src_ok) {
      B.src_ok = 1;
      B.src_i0 = fb.src_i0 - fb.mgx;
      B.src_j0 = fb.src_j0 - fb.mgy;
      source_weights(fb.src_hx, fb.src_ax, B.src_wx);
      source_weights(fb.src_hy, fb.src_ay, B.src_wy);
    }
    B.tiles_x = own ? (g.nx + TX - 1) / TX : 0;
    int tiles_y = own ? (g.ny + TY - 1) / TY : 0;
    B.tile_begin = tiles;
    tiles += B.tiles_x * tiles_y;
  }
  h->total_tiles = tiles;
  h->body_on_device = d->body != nullptr;
  if (h->body_on_device) {
    h->cur = 0;
    int rcb = build_body(h, d, op);
    if (rcb) return rcb;
  } else {
    h->tp[0] = d->t0; h->tp[1] = d->dt; h->tp[2] = d->CFL; h->tp[3] = d->hmin; h->tp[4] = d->hmax;
    h->tp_nt = d->nt;
  }

  // interfaces
  h->iface_n.resize(d->nifaces);
  h->iface_fric.resize(d->nifaces);
  for (int k = 0; k < d->nifaces; ++k) {
    const fdmap_iface& fi = d->ifaces[k];
    DevIface& I = D.ifc[k];
    I.direction = fi.direction; I.im = fi.iblockm; I.ip = fi.iblockp; I.m = fi.m; I.p = fi.p;
    I.n = fi.p - fi.m + 1; I.coupling = fi.coupling;
    h->iface_n[k] = I.n;
    h->iface_fric[k] = fi.coupling == FDMAP_COUPLING_FRICTION;
    const fdmap_block& Bm = d->blocks[fi.iblockm];
    const fdmap_block& Bp = d->blocks[fi.iblockp];
    I.offm = fi.m - (fi.direction == 0 ? Bm.mgy : Bm.mgx);
    I.offp = fi.m - (fi.direction == 0 ? Bp.mgy : Bp.mgx);
    // sides whose hat variables come from this interface
    DevSide& Sm = D.blk[fi.iblockm].side[fi.direction == 0 ? 1 : 3];
    DevSide& Sp = D.blk[fi.iblockp].side[fi.direction == 0 ? 0 : 2];
    Sm.cov_lo = I.offm; Sm.cov_hi = I.offm + I.n;
    Sp.cov_lo = I.offp; Sp.cov_hi = I.offp + I.n;
    int rc;
    {
      // impedance terms of both sides (interfaces.f90:696-699, 735-760, 851-855, 956-965)
      const int sm = fi.direction == 0 ? 1 : 3, sp = fi.direction == 0 ? 0 : 2;
      const fdmap_side& fsm = Bm.side[sm];
      const fdmap_side& fsp = Bp.side[sp];
      // Zs = rho*cs and Zp = rho*cp (side impedance columns 0 and 1); with the
      // body built on the device they are formed here from the same material
      auto Z = [&](const fdmap_block& fb, const fdmap_side& fs, int blk, int side, int k, int c) {
        if (!d->body) return fs.M[k + (size_t)c * fs.n];
        const double* mat = d->body->blocks[blk].side_mat[side];
        if (!mat) return fb.rho * (c == 0 ? fb.cs : fb.cp);
        return mat[k] * mat[k + (size_t)(c == 0 ? 1 : 2) * fs.n];
      };
      std::vector<double> ic((size_t)IC_N * I.n);
      for (int q = 0; q < I.n; ++q) {
        double Zsm = Z(Bm, fsm, fi.iblockm, sm, I.offm + q, 0), Zsp = Z(Bp, fsp, fi.iblockp, sp, I.offp + q, 0);
        double Zpm = Z(Bm, fsm, fi.iblockm, sm, I.offm + q, 1), Zpp = Z(Bp, fsp, fi.iblockp, sp, I.offp + q, 1);
        double Zsim = 1.0 / Zsm, Zsip = 1.0 / Zsp, Zpim = 1.0 / Zpm, Zpip = 1.0 / Zpp;
        ic[(size_t)IC_ZSIM * I.n + q] = Zsim;
        ic[(size_t)IC_ZSIP * I.n + q] = Zsip;
        ic[(size_t)IC_ZPIM * I.n + q] = Zpim;
        ic[(size_t)IC_ZPIP * I.n + q] = Zpip;
        ic[(size_t)IC_ETAS * I.n + q] = 1.0 / (Zsip + Zsim);
        ic[(size_t)IC_ETAP * I.n + q] = 1.0 / (Zpip + Zpim);
      }
      if ((rc = h->upload(&I.icoef, ic.data(), ic.size()))) return rc;
    }
    I.rem_m = I.rem_p = nullptr;
    I.send = nullptr;
    if (h->owns(fi.iblockm) != h->owns(fi.iblockp)) {
      // one side on this GPU, the other on a peer: receive buffer for the
      // peer's edge values, two send slots (alternating stages) for ours
      double *rem = nullptr, *snd = nullptr;
      if ((rc = h->alloc(&rem, (size_t)nF * I.n)) || (rc = h->alloc(&snd, 2 * (size_t)nF * I.n))) return rc;
      CUDA_TRY(cudaMemset(rem, 0, (size_t)nF * I.n * sizeof(double)));
      (h->owns(fi.iblockm) ? I.rem_p : I.rem_m) = rem;
      I.send = snd;
      h->part_ifaces.push_back(k);
    }
    if ((rc = h->upload(&I.nhat, fi.nhat, 2 * (size_t)I.n))) return rc;
    if ((rc = h->upload(&I.x, fi.x, (size_t)I.n))) return rc;
    if ((rc = h->upload(&I.y, fi.y, (size_t)I.n))) return rc;
    if (fi.coupling != FDMAP_COUPLING_FRICTION) continue;
    const fdmap_friction& ff = fi.fr;
    DevFriction& FR = I.fr;
    FR.law = ff.law; FR.reg = ff.reg; FR.rup_field = ff.rup_field; FR.force = ff.force;
    FR.ld_shape = ff.ld_shape; FR.tp_use = ff.tp_use;
    FR.has_bsS0 = ff.bsS0 != nullptr; FR.has_bsN0 = ff.bsN0 != nullptr;
    FR.rup_threshold = ff.rup_threshold; FR.angle = ff.angle; FR.xlockm = ff.xlockm; FR.xlockp = ff.xlockp;
    FR.cos_angle = std::cos(ff.angle); FR.sin_angle = std::sin(ff.angle);
    FR.flock = ff.flock; FR.skempton = ff.skempton;
    FR.kn_c0 = ff.kn_c0; FR.kn_fd = ff.kn_fd; FR.kn_dfdx = ff.kn_dfdx; FR.kn_vL = ff.kn_vL; FR.kn_vR = ff.kn_vR;
    FR.kn_xL = ff.kn_xL; FR.kn_xR = ff.kn_xR; FR.kn_tmax = ff.kn_tmax;
    FR.ld_S = ff.ld_S; FR.ld_N = ff.ld_N; FR.ld_T = ff.ld_T; FR.ld_R = ff.ld_R; FR.ld_x0 = ff.ld_x0;
    FR.ld_y0 = ff.ld_y0; FR.tp_p0 = ff.tp_p0;
    const int n = I.n;
    std::vector<double> st((size_t)FDMAP_FAULT_NFIELDS * n), par((size_t)PAR_N * n, 0.0);
    const double* sp[FDMAP_FAULT_NFIELDS] = {ff.D, ff.Psi, ff.DPsi, ff.trup, ff.V, ff.O, ff.S, ff.N, ff.S0,
                                             ff.N0, ff.Ds, ff.Dn, ff.DDs, ff.DDn, ff.W, ff.DW, ff.Nreg, ff.DNreg};
    for (int f = 0; f < FDMAP_FAULT_NFIELDS; ++f) std::memcpy(&st[(size_t)f * n], sp[f], n * sizeof(double));
    const double* pp[PAR_N] = {ff.a, ff.b, ff.V0, ff.f0, ff.L, ff.fw, ff.Vw, ff.c0, ff.fs, ff.fd, ff.Dc, ff.bsS0, ff.bsN0};
    for (int q = 0; q < PAR_N; ++q)
      if (pp[q]) std::memcpy(&par[(size_t)q * n], pp[q], n * sizeof(double));
    if ((rc = h->upload(&FR.st, st.data(), st.size()))) return rc;
    if ((rc = h->upload(&FR.par, par.data(), par.size()))) return rc;
  }

  // interface work segments; closure strips per block
  int nseg = 0, start = 0;
  for (int k = 0; k < d->nifaces; ++k) {
    // an interface between two blocks of other GPUs is solved there
    if (!h->owns(D.ifc[k].im) && !h->owns(D.ifc[k].ip)) continue;
    D.seg_kind[nseg] = 1; D.seg_a[nseg] = k; D.seg_b[nseg] = 0; D.seg_start[nseg] = start;
    start += D.ifc[k].n;
    ++nseg;
  }
  {
    long long cs = 0;
    for (int b = 0; b < d->nblocks; ++b) {
      const BlockGeom& g = h->geom[b];
      const long long w = h->owns(b) ? 1 : 0;
      long long strip[4] = {w * op.nbst * g.nx, w * op.nbst * g.nx, w * (g.ny - 2 * op.nbst) * op.nbst,
                            w * (g.ny - 2 * op.nbst) * op.nbst};
      for (int q = 0; q < 4; ++q) { D.cstart[4 * b + q] = cs; cs += strip[q]; }
    }
    D.cstart[4 * d->nblocks] = cs;
    h->closure_threads = cs;
  }
  D.seg_start[nseg] = start;
  D.nseg = nseg;
  h->edge_threads = start;

  int rc;
  {
    const char* ek = getenv("FDMAP_STENCIL");
    // the march serves every variant: dissipation (J halo rows in the ring),
    // PML, forcing and body extras through its extras variant; the first
    // tile shape whose rings fit is taken (the autotuner may change it)
    // (a domain with both dissipative and PML blocks keeps the tiled kernel)
    h->march_ext = h->pml ? 2 : ((h->dissipation || h->forcing || h->extras) ? 1 : 0);
    h->use_march = !(ek && std::string(ek) == "tile") && !(h->pml && h->dissipation);
    if (h->use_march) {
      rc = FDMAP_ERR_UNSUPPORTED;
      for (int sh = 0; sh < MARCH_SHAPES && rc == FDMAP_ERR_UNSUPPORTED; ++sh) rc = march_configure(h, sh);
      if (rc == FDMAP_ERR_UNSUPPORTED) h->use_march = 0;  // no shape fits: the tiled interior kernel
      else if (rc) return rc;
    }
    // boundary kernels on the march's carveout (FDMAP_CARVEOUT=default leaves the driver's choice)
    const char* ec = getenv("FDMAP_CARVEOUT");
    if (h->use_march && !(ec && std::string(ec) == "default")) {
      rc = h->mode == 2 ? boundary_carveout_mode<2>() : boundary_carveout_mode<3>();
      if (rc) return rc;
    }
    // fused stage launches need every interface-side node to sit on one interface only
    bool junction = false;
    for (int b = 0; b < d->nblocks; ++b) {
      const DevBlock& B = D.blk[b];
      bool cov[4];
      for (int q = 0; q < 4; ++q) cov[q] = B.side[q].cov_hi > B.side[q].cov_lo;
      // a corner node shared by two interface sides
      if ((cov[0] || cov[1]) && (cov[2] || cov[3])) junction = true;
    }
    // one merged boundary launch is opt-in: the two separate launches measure faster
    const char* ef = getenv("FDMAP_FUSED");
    h->fused = !junction && (ef && std::string(ef) == "1");
    // concurrent boundary work needs the interior march (it leaves registers
    // free); FDMAP_OVERLAP=0 serialises the stage
    const char* eo = getenv("FDMAP_OVERLAP");
    h->overlap = h->use_march && !h->fused && !(eo && std::string(eo) == "0");
  }
  if ((rc = h->alloc(&h->d_status, 4))) return rc;
  if ((rc = h->alloc(&h->d_time, 1))) return rc;
  {
    const char* eg = getenv("FDMAP_GRAPHS");
    h->use_graphs = !(eg && std::string(eg) == "0");
  }
  CUDA_TRY(cudaMemset(h->d_status, 0, 4 * sizeof(unsigned long long)));
  D.status = h->d_status;
  D.newton_imax = 99;  // friction.f90:924
  D.energy = nullptr;
  if (d->energy_balance) {
    if ((rc = h->alloc(&h->d_energy, (size_t)d->nblocks + 1)) ||
        (rc = h->alloc(&h->d_epart, (size_t)energy_scratch_size(d->nblocks))))
      return rc;
    std::vector<double> big((size_t)d->nblocks + 1, 1e40);  // BF%Etot = 1d40 until the first stage 1
    CUDA_TRY(cudaMemcpy(h->d_energy, big.data(), big.size() * sizeof(double), cudaMemcpyHostToDevice));
    D.energy = h->d_energy;
  }
  // two-stage passes where the domain allows them (FDMAP_PAIRS=0 keeps stage by stage)
  if (h->rk.A[0] == 0.0) {
    const char* ep = getenv("FDMAP_PAIRS");
    if (!(ep && std::string(ep) == "0") && (rc = pair_configure(h))) return rc;
  }
  if ((rc = h->alloc(&h->ddom, 1))) return rc;
  CUDA_TRY(cudaMemcpy(h->ddom, &D, sizeof(DevDomain), cudaMemcpyHostToDevice));

  // global-layout staging buffer and initial fields
  if ((rc = h->alloc(&h->d_global, (size_t)d->nx * d->ny * nF))) return rc;
  if (d->src.forcing_filename) {
    // init_forcing_from_file (source.f90:409-448): frame 0 becomes the new frame
    h->frc_file = std::fopen(d->src.forcing_filename, "rb");
    if (!h->frc_file)
      return set_err(FDMAP_ERR_IO, std::string("cannot open forcing file ") + d->src.forcing_filename);
    if ((rc = forcing_read_frame(h))) return rc;
  }
  if (h->body_on_device) return FDMAP_OK;  // fields already built in F[0], DF
  h->cur = 0;
  return fdmap_gpu_set_fields(h, d->F, d->DF);
}

// Two consecutive stages a0, a1 (F[a0.in] -> F[a1.out]) as one interior pass
// (march_pair.cuh).  Beside the pass, on the side stream: the interface solve
// and closure strips of the first stage (writing the scratch buffer F[2]),
// then the interface solve of the second stage from F[2]; after both, the
// band kernel does the second stage near the block edges.  Rates go from
// buffer dfr to buffer dfw.  `gather`: a0 is stage 1 with outputs open; the
// output gather runs between the first stage's closure strips and the second
// stage's interface solve, while the hat variables are still stage 1's (the
// body fields it samples, F[a0.in], are not written by the pair).
int launch_pair(fdmap_gpu* h, const StageArgs& a0, const StageArgs& a1, int dfr, int dfw, bool gather,
                long long n) {
  StageArgs c0 = a0;  // first stage at the closure strips: into the scratch buffer
  c0.out = 2;
  c0.dfr = dfr;
  c0.dfw = dfw;
  StageArgs e1 = a1;  // second stage's interface solve and band: from the scratch buffer
  e1.in = 2;
  e1.dfr = dfw;
  e1.dfw = dfw;
  const bool ov = h->overlap && !h->profiling;
  if (ov) {
    CUDA_TRY(cudaEventRecord(h->ev_fork, h->stream));
    CUDA_TRY(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
  }
  {
    ProfScope ps(h, 3);
    int rc = pair_launch(h, a0, a1, dfr, dfw);
    if (rc) return rc;
    h->launches++;
  }
  cudaStream_t main_stream = h->stream;
  if (ov) h->stream = h->side_stream;
  int rc = launch_boundary(h, c0);
  if (rc == FDMAP_OK && gather) rc = output_gather(h, a0.ts, n, a0.in);
  if (rc == FDMAP_OK) rc = launch_edges(h, e1);
  h->stream = main_stream;
  if (rc) return rc;
  if (ov) {
    CUDA_TRY(cudaEventRecord(h->ev_join, h->side_stream));
    CUDA_TRY(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
  }
  ProfScope pb(h, 4);
  if ((rc = band_launch(h, e1))) return rc;
  h->launches++;
  return FDMAP_OK;
}

// F buffer swaps of one (non-final) step: one per stage, or one per pass
// when stages run in two-stage passes
int step_swaps(const fdmap_gpu* h) {
  return h->use_pairs ? h->rk.nstage / 2 + (h->rk.nstage & 1) : h->rk.nstage;
}

// all stages of one step starting from buffer `cur`; final = stage 1 only.
// With outputs open, stage 1 taps the interface state and the output gather
// follows it (step index from the device clock `ts`, else `n`).  With
// two-stage passes, stages (1,2), (3,4), ... run as pairs and an odd last
// stage alone; the pairs' rate buffers alternate so that the last pair
// writes DF and the step ends with its rates in DF, as stage by stage.
int issue_step(fdmap_gpu* h, int cur, double t0, double dt, bool final_step, const TimeState* ts, long long n = 0) {
  const bool outputs = output_is_open(h);
  const int cur0 = cur;
  const int npairs = (h->use_pairs && !final_step) ? h->rk.nstage / 2 : 0;
  auto args = [&](int s, int in) {
    StageArgs a{};
    a.tap = (s == 0 && outputs) ? 1 : 0;
    a.A = h->rk.A[s];
    a.Bdt = h->rk.B[s] * dt;
    a.t = t0 + h->rk.C[s] * dt;
    a.C = h->rk.C[s];
    a.t0 = t0;
    a.dt = dt;
    a.first = s == 0 ? 1 : 0;
    a.ts = ts;
    a.in = in;
    a.out = 1 - in;
    a.scale = 1;
    a.update = final_step ? 0 : 1;
    return a;
  };
  for (int s = 0; s < h->rk.nstage; ++s) {
    int rc;
    const StageArgs a = args(s, cur);
    if (s < 2 * npairs) {
      const int p = s / 2;
      const int dfw = ((npairs - 1 - p) & 1) ? 1 : 0;
      const int dfr = p == 0 ? 0 : 1 - dfw;  // the first pair reads no rates (A(1) = 0)
      StageArgs a1 = args(s + 1, cur);
      a1.out = 1 - cur;
      if ((rc = launch_pair(h, a, a1, dfr, dfw, a.first && outputs, n))) return rc;
      ++s;
    } else {
      if ((rc = launch_stage(h, a))) return rc;
      if (a.first && h->d_energy && (rc = launch_energy(h, cur0))) return rc;
      if (a.first && outputs && (rc = output_gather(h, ts, n, cur0))) return rc;
    }
    if (final_step) return FDMAP_OK;
    cur = 1 - cur;
  }
  return FDMAP_OK;
}

// capture one step per starting buffer; kernels read the step clock from d_time
int build_step_graphs(fdmap_gpu* h, double dt) {
  for (auto& ge : h->step_graph)
    if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  bool prof = h->profiling;
  h->profiling = false;
  cudaStream_t keep = h->stream;
  h->stream = h->own_stream;
  long long before = h->launches;
  int rc = FDMAP_OK;
  for (int c = 0; c < 2 && rc == FDMAP_OK; ++c) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { rc = set_err(FDMAP_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e)); break; }
    long long l0 = h->launches;
    rc = issue_step(h, c, 0.0, dt, false, h->d_time);
    if (rc == FDMAP_OK) advance_step<<<1, 1, 0, h->stream>>>(h->d_time);
    h->graph_launches = h->launches - l0 + 1;
    e = cudaStreamEndCapture(h->stream, &g);
    if (rc == FDMAP_OK && e != cudaSuccess) rc = set_err(FDMAP_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(e));
    if (rc == FDMAP_OK) {
      e = cudaGraphInstantiate(&h->step_graph[c], g, cudaGraphInstantiateFlagUseNodePriority);
      if (e != cudaSuccess) rc = set_err(FDMAP_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    }
    if (g) cudaGraphDestroy(g);
  }
  h->launches = before;
  h->stream = keep;
  h->profiling = prof;
  if (rc == FDMAP_OK) h->graph_dt = dt;
  return rc;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

int create_impl(const fdmap_desc* d, int device, int init_edges, const int* owned, fdmap_gpu** out) {
  if (!out) return set_err(FDMAP_ERR_INVALID_ARG, "null handle pointer");
  *out = nullptr;
  int rc = validate(d);
  if (rc) return rc;
  if (owned) {
    int nown = 0;
    for (int b = 0; b < d->nblocks; ++b) nown += owned[b] != 0;
    if (nown == 0) return set_err(FDMAP_ERR_INVALID_ARG, "a partition must own at least one block");
    if (d->body) return set_err(FDMAP_ERR_UNSUPPORTED, "a partitioned domain needs the body built on the host");
    if (d->energy_balance || d->src.forcing_filename)
      return set_err(FDMAP_ERR_UNSUPPORTED, "energy balance and forcing files are not available on a partition");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_err(FDMAP_ERR_CUDA, "no CUDA device available");
  if (device < 0 || device >= ndev) return set_err(FDMAP_ERR_INVALID_ARG, "bad device index");
  fdmap_gpu* h = new (std::nothrow) fdmap_gpu();
  if (!h) return set_err(FDMAP_ERR_NOMEM, "out of host memory");
  h->device = device;
  int prio_low = 0, prio_high = 0;
  if (cudaSetDevice(device) != cudaSuccess || cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess ||
      cudaStreamCreateWithPriority(&h->own_stream, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
      cudaStreamCreateWithPriority(&h->side_stream, cudaStreamNonBlocking, prio_low) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    delete h;
    return set_err(FDMAP_ERR_CUDA, "cannot initialise device");
  }
  h->stream = h->own_stream;
  if (owned) {
    h->owned.assign(owned, owned + d->nblocks);
    for (auto& o : h->owned) o = o != 0;
    if (cudaEventCreateWithFlags(&h->ev_packed, cudaEventDisableTiming) != cudaSuccess) {
      delete h;
      return set_err(FDMAP_ERR_CUDA, "cannot create events");
    }
  }
  rc = build(h, d);
  if (rc == FDMAP_OK && h->partitioned()) {
    // the edge exchange is a host callback (or a group step): no step graphs,
    // and interface solves stay apart from the closure strips
    h->use_graphs = false;
    h->fused = 0;
  }
  if (rc == FDMAP_OK && init_edges) rc = fdmap_gpu_init_edges(h, d->t0);
  if (rc == FDMAP_OK) rc = fdmap_gpu_synchronize(h);
  if (rc) {
    std::string keep = g_err;
    delete h;
    g_err = keep;
    return rc;
  }
  *out = h;
  return FDMAP_OK;
}

StageArgs init_edge_args(const fdmap_gpu* h, double t) {
  StageArgs a{};
  a.A = 0.0; a.Bdt = 0.0; a.t = t; a.in = h->cur; a.out = 1 - h->cur; a.scale = 0; a.update = 0;
  return a;
}

// the stage arguments of every stage of one step from buffer `cur`
std::vector<StageArgs> step_args(const fdmap_gpu* h, int cur, double t0, double dt, bool final_step) {
  std::vector<StageArgs> v;
  for (int s = 0; s < h->rk.nstage; ++s) {
    StageArgs a{};
    a.A = h->rk.A[s];
    a.Bdt = h->rk.B[s] * dt;
    a.t = t0 + h->rk.C[s] * dt;
    a.C = h->rk.C[s];
    a.t0 = t0;
    a.dt = dt;
    a.first = s == 0 ? 1 : 0;
    a.in = cur;
    a.out = 1 - cur;
    a.scale = 1;
    a.update = final_step ? 0 : 1;
    v.push_back(a);
    if (final_step) break;
    cur = 1 - cur;
  }
  return v;
}

// Group of partitions driven from one host thread (one handle per GPU, or
// several on one GPU): after every handle has packed its edge values for the
// stage, each handle's boundary stream waits for its peers' pack and copies
// their values into its receive buffers (peer-to-peer between GPUs), then
// finishes the stage.  Send slots alternate between stages, so a pack never
// overwrites a slot a peer may still be reading.
int group_exchange(fdmap_gpu* const* hs, int n, bool main_stream) {
  for (int i = 0; i < n; ++i) {
    fdmap_gpu* h = hs[i];
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t bs = main_stream ? h->stream : boundary_stream(h);
    for (int k : h->part_ifaces) {
      const DevIface& I = h->hdom.ifc[k];
      const int rb = h->owns(I.im) ? I.ip : I.im;  // the block on a peer
      fdmap_gpu* p = nullptr;
      for (int j = 0; j < n; ++j)
        if (j != i && hs[j]->owns(rb) && hs[j]->partitioned()) p = hs[j];
      if (!p) return set_err(FDMAP_ERR_INVALID_ARG, "no handle of the group owns block " + std::to_string(rb));
      const DevIface& P = p->hdom.ifc[k];
      const size_t cnt = (size_t)h->nF * I.n;
      const double* src = P.send + (size_t)(p->xstage & 1) * cnt;
      double* dst = const_cast<double*>(I.rem_m ? I.rem_m : I.rem_p);
      CUDA_TRY(cudaStreamWaitEvent(bs, p->ev_packed, 0));
      if (p->device == h->device) CUDA_TRY(cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyDeviceToDevice, bs));
      else CUDA_TRY(cudaMemcpyPeerAsync(dst, h->device, src, p->device, cnt * sizeof(double), bs));
    }
  }
  return FDMAP_OK;
}

int check_group(fdmap_gpu* const* hs, int n) {
  if (!hs || n < 1) return set_err(FDMAP_ERR_INVALID_ARG, "empty group");
  for (int i = 0; i < n; ++i)
    if (!hs[i] || !hs[i]->partitioned()) return set_err(FDMAP_ERR_INVALID_ARG, "group members must be partitions");
  return FDMAP_OK;
}

}  // namespace

extern "C" {

int fdmap_gpu_create(const fdmap_desc* d, int device, int init_edges, fdmap_gpu** out) {
  return create_impl(d, device, init_edges, nullptr, out);
}

int fdmap_gpu_init_edges(fdmap_gpu* h, double t) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  const StageArgs a = init_edge_args(h, t);
  if (!h->part_ifaces.empty()) {
    // the peers' edge values first, through the exchange callback
    if (!h->exchange) return set_err(FDMAP_ERR_INVALID_ARG, "partitioned domain without an exchange callback");
    int rc = pack_partition_edges(h, a, h->stream);
    if (rc) return rc;
    rc = h->exchange(h->exchange_user, h->xstage, (void*)h->stream);
    if (rc) return set_err(FDMAP_ERR_CUDA, "edge exchange callback failed (" + std::to_string(rc) + ")");
    h->xstage++;
  }
  return launch_edges(h, a);
}

int fdmap_gpu_create_part(const fdmap_desc* d, int device, const int* owned, fdmap_gpu** out) {
  if (!owned) return set_err(FDMAP_ERR_INVALID_ARG, "null ownership list");
  return create_impl(d, device, 0, owned, out);
}

int fdmap_gpu_part_interfaces(fdmap_gpu* h, int* ifaces, int max) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  const int n = (int)h->part_ifaces.size();
  for (int q = 0; q < n && q < max && ifaces; ++q) ifaces[q] = h->part_ifaces[(size_t)q];
  return n;
}

int fdmap_gpu_part_buffers(fdmap_gpu* h, int iface, long long stage, double** send, double** recv, long long* count) {
  if (!h || iface < 0 || iface >= h->hdom.nifaces) return set_err(FDMAP_ERR_INVALID_ARG, "bad part_buffers arguments");
  const DevIface& I = h->hdom.ifc[iface];
  if (!I.send) return set_err(FDMAP_ERR_INVALID_ARG, "interface has no side on a peer GPU");
  const size_t cnt = (size_t)h->nF * I.n;
  if (send) *send = I.send + (size_t)(stage & 1) * cnt;
  if (recv) *recv = const_cast<double*>(I.rem_m ? I.rem_m : I.rem_p);
  if (count) *count = (long long)cnt;
  return FDMAP_OK;
}

int fdmap_gpu_set_exchange(fdmap_gpu* h, fdmap_exchange_fn fn, void* user) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  h->exchange = fn;
  h->exchange_user = user;
  return FDMAP_OK;
}

int fdmap_gpu_group_init_edges(fdmap_gpu* const* hs, int n, double t) {
  int rc = check_group(hs, n);
  if (rc) return rc;
  for (int i = 0; i < n; ++i) {
    CUDA_TRY(cudaSetDevice(hs[i]->device));
    if ((rc = pack_partition_edges(hs[i], init_edge_args(hs[i], t), hs[i]->stream))) return rc;
  }
  if ((rc = group_exchange(hs, n, true))) return rc;
  for (int i = 0; i < n; ++i) {
    hs[i]->xstage++;
    CUDA_TRY(cudaSetDevice(hs[i]->device));
    if ((rc = launch_edges(hs[i], init_edge_args(hs[i], t)))) return rc;
  }
  return FDMAP_OK;
}

int fdmap_gpu_group_time_step(fdmap_gpu* const* hs, int n, double t0, double dt, int final_step) {
  int rc = check_group(hs, n);
  if (rc) return rc;
  std::vector<std::vector<StageArgs>> args;
  for (int i = 0; i < n; ++i) args.push_back(step_args(hs[i], hs[i]->cur, t0, dt, final_step != 0));
  for (size_t s = 0; s < args[0].size(); ++s) {
    for (int i = 0; i < n; ++i) {
      CUDA_TRY(cudaSetDevice(hs[i]->device));
      if ((rc = stage_begin(hs[i], args[(size_t)i][s]))) return rc;
    }
    if ((rc = group_exchange(hs, n, false))) return rc;
    for (int i = 0; i < n; ++i) {
      hs[i]->xstage++;
      CUDA_TRY(cudaSetDevice(hs[i]->device));
      if ((rc = stage_end(hs[i], args[(size_t)i][s]))) return rc;
    }
  }
  for (int i = 0; i < n; ++i)
    if (!final_step && (hs[i]->rk.nstage & 1)) hs[i]->cur = 1 - hs[i]->cur;
  return FDMAP_OK;
}

int fdmap_gpu_group_run(fdmap_gpu* const* hs, int n, double t_start, double dt, int n_first, int n_last, int nt) {
  for (int k = n_first; k <= n_last; ++k) {
    int rc = fdmap_gpu_group_time_step(hs, n, t_start + (double)(k - 1) * dt, dt, k == nt);
    if (rc) return rc;
  }
  return FDMAP_OK;
}

int fdmap_gpu_time_step(fdmap_gpu* h, double t0, double dt, int final_step) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  int rc = output_before_step(h, h->out_next_n, t0);
  if (rc) return rc;
  if ((rc = forcing_load(h))) return rc;
  rc = issue_step(h, h->cur, t0, dt, final_step != 0, nullptr, h->out_next_n);
  if (rc) return rc;
  h->out_next_n += 1;
  if (!final_step && (step_swaps(h) & 1)) h->cur = 1 - h->cur;
  return FDMAP_OK;
}

int fdmap_gpu_run(fdmap_gpu* h, double t_start, double dt, int n_first, int n_last, int nt) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  h->launches = 0;
  int n_graph_last = std::min(n_last, nt - 1);  // the final step (n == nt) is issued directly
  if (h->use_graphs && !h->profiling && n_graph_last >= n_first) {
    if (h->graph_dt != dt || !h->step_graph[0]) {
      int rc = build_step_graphs(h, dt);
      if (rc) return rc;
    }
    set_step_clock<<<1, 1, 0, h->stream>>>(h->d_time, t_start, dt, (long long)n_first);
    h->launches++;
    CUDA_TRY(cudaGetLastError());
    for (int n = n_first; n <= n_graph_last; ++n) {
      int rc = output_before_step(h, n, t_start + (double)(n - 1) * dt);
      if (rc) return rc;
      if ((rc = forcing_load(h))) return rc;
      CUDA_TRY(cudaGraphLaunch(h->step_graph[h->cur], h->stream));
      h->launches += h->graph_launches;
      if (step_swaps(h) & 1) h->cur = 1 - h->cur;
    }
    n_first = n_graph_last + 1;
  }
  h->out_next_n = n_first;
  for (int n = n_first; n <= n_last; ++n) {
    int rc = fdmap_gpu_time_step(h, t_start + (double)(n - 1) * dt, dt, n == nt);
    if (rc) return rc;
  }
  h->out_next_n = (long long)n_last + 1;
  return FDMAP_OK;
}

int fdmap_gpu_synchronize(fdmap_gpu* h) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return FDMAP_OK;
}

int fdmap_gpu_get_fields(fdmap_gpu* h, double* F, double* DF) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  const int nF = h->nF;
  const long long NN = (long long)h->nx_g * h->ny_g;
  for (int which = 0; which < 2; ++which) {
    double* dst = which == 0 ? F : DF;
    if (!dst) continue;
    // padded block planes -> one contiguous global array on the device -> one copy
    for (int b = 0; b < h->hdom.nblocks; ++b) {
      if (!h->owns(b)) continue;  // body on a peer GPU
      const BlockGeom& g = h->geom[b];
      const double* src = which == 0 ? h->hdom.blk[b].F[h->cur] : h->hdom.blk[b].DF;
      dim3 grid((g.nx + 255) / 256, g.ny);
      gather_block<<<grid, 256, 0, h->stream>>>(src, h->d_global, h->nx_g, NN, g.mgx, g.mgy, g.nx, g.ny, g.pitch,
                                               g.plane, nF);
      CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaMemcpyAsync(dst, h->d_global, (size_t)NN * nF * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  return FDMAP_OK;
}

int fdmap_gpu_set_fields(fdmap_gpu* h, const double* F, const double* DF) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  const int nF = h->nF;
  const long long NN = (long long)h->nx_g * h->ny_g;
  for (int which = 0; which < 2; ++which) {
    const double* src = which == 0 ? F : DF;
    if (!src) continue;
    // one copy of the global array, then scattered into the padded block planes
    CUDA_TRY(cudaMemcpyAsync(h->d_global, src, (size_t)NN * nF * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    for (int b = 0; b < h->hdom.nblocks; ++b) {
      if (!h->owns(b)) continue;  // body on a peer GPU
      const BlockGeom& g = h->geom[b];
      double* dst = which == 0 ? h->hdom.blk[b].F[h->cur] : h->hdom.blk[b].DF;
      dim3 grid((g.pitch + 255) / 256, g.ny);
      scatter_block<<<grid, 256, 0, h->stream>>>(h->d_global, dst, h->nx_g, NN, g.mgx, g.mgy, g.nx, g.ny, g.pitch,
                                                g.plane, nF);
      CUDA_TRY(cudaGetLastError());
    }
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return FDMAP_OK;
}

int fdmap_gpu_time_params(fdmap_gpu* h, double* params, int* nt) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  if (params)
    for (int q = 0; q < 5; ++q) params[q] = h->tp[q];
  if (nt) *nt = h->tp_nt;
  return FDMAP_OK;
}

int fdmap_gpu_get_metric(fdmap_gpu* h, int which, double* out) {
  if (!h || !out || which < FDMAP_METRIC_XQ || which > FDMAP_METRIC_J)
    return set_err(FDMAP_ERR_INVALID_ARG, "bad get_metric arguments");
  CUDA_TRY(cudaSetDevice(h->device));
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    const DevBlock& B = h->hdom.blk[b];
    const double* planes[6] = {B.xq, B.xr, B.yq, B.yr, B.Ji, B.J};
    if (!planes[which]) return set_err(FDMAP_ERR_INVALID_ARG, "the Jacobian plane is kept for dissipative blocks only");
  }
  const long long NN = (long long)h->nx_g * h->ny_g;
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    const DevBlock& B = h->hdom.blk[b];
    const double* planes[6] = {B.xq, B.xr, B.yq, B.yr, B.Ji, B.J};
    const BlockGeom& g = h->geom[b];
    dim3 grid((g.pitch + 255) / 256, g.ny);
    gather_block<<<grid, 256, 0, h->stream>>>(planes[which], h->d_global, h->nx_g, NN, g.mgx, g.mgy, g.nx, g.ny,
                                              g.pitch, g.plane, 1);
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaMemcpyAsync(out, h->d_global, (size_t)NN * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return FDMAP_OK;
}

namespace {
// planes `which` of every block (body displacement U / DU, nU planes; peak pgv / pga, 1 plane)
// between the host's global layout and the device
int body_planes(fdmap_gpu* h, int which, double* out, const double* in) {
  const int nU = h->mode == 2 ? 2 : 1;
  const int np = which <= 1 ? nU : 1;
  const long long NN = (long long)h->nx_g * h->ny_g;
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    const DevBlock& B = h->hdom.blk[b];
    double* const planes[4] = {B.U, B.DU, B.pgv, B.pga};
    if (!planes[which])
      return set_err(FDMAP_ERR_INVALID_ARG, which <= 1 ? "the domain does not track the body displacement"
                                                       : "the domain does not track peak motion");
  }
  CUDA_TRY(cudaSetDevice(h->device));
  if (in) CUDA_TRY(cudaMemcpyAsync(h->d_global, in, (size_t)NN * np * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    const DevBlock& B = h->hdom.blk[b];
    double* const planes[4] = {B.U, B.DU, B.pgv, B.pga};
    const BlockGeom& g = h->geom[b];
    dim3 grid((g.pitch + 255) / 256, g.ny);
    if (in)
      scatter_block<<<grid, 256, 0, h->stream>>>(h->d_global, planes[which], h->nx_g, NN, g.mgx, g.mgy, g.nx, g.ny,
                                                 g.pitch, g.plane, np);
    else
      gather_block<<<grid, 256, 0, h->stream>>>(planes[which], h->d_global, h->nx_g, NN, g.mgx, g.mgy, g.nx, g.ny,
                                                g.pitch, g.plane, np);
    CUDA_TRY(cudaGetLastError());
  }
  if (out)
    CUDA_TRY(cudaMemcpyAsync(out, h->d_global, (size_t)NN * np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return FDMAP_OK;
}
}  // namespace

int fdmap_gpu_get_energy(fdmap_gpu* h, double* E) {
  if (!h || !E) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  if (!h->d_energy) return set_err(FDMAP_ERR_INVALID_ARG, "the domain does not track the energy");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CUDA_TRY(cudaMemcpy(E, h->d_energy, (size_t)(h->hdom.nblocks + 1) * sizeof(double), cudaMemcpyDeviceToHost));
  return FDMAP_OK;
}

int fdmap_gpu_get_displacement(fdmap_gpu* h, double* U, double* DU) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  int rc = FDMAP_OK;
  if (U && (rc = body_planes(h, 0, U, nullptr))) return rc;
  if (DU && (rc = body_planes(h, 1, DU, nullptr))) return rc;
  return FDMAP_OK;
}

int fdmap_gpu_set_displacement(fdmap_gpu* h, const double* U, const double* DU) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  int rc = FDMAP_OK;
  if (U && (rc = body_planes(h, 0, nullptr, U))) return rc;
  if (DU && (rc = body_planes(h, 1, nullptr, DU))) return rc;
  return FDMAP_OK;
}

int fdmap_gpu_get_peak(fdmap_gpu* h, double* pgv, double* pga) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  int rc = FDMAP_OK;
  if (pgv && (rc = body_planes(h, 2, pgv, nullptr))) return rc;
  if (pga && (rc = body_planes(h, 3, pga, nullptr))) return rc;
  return FDMAP_OK;
}

int fdmap_gpu_set_peak(fdmap_gpu* h, const double* pgv, const double* pga) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  int rc = FDMAP_OK;
  if (pgv && (rc = body_planes(h, 2, nullptr, pgv))) return rc;
  if (pga && (rc = body_planes(h, 3, nullptr, pga))) return rc;
  return FDMAP_OK;
}

// PML field Wx (which = 0) or Wy (1) in the global (nx,ny,nF) layout
int fdmap_gpu_get_pml(fdmap_gpu* h, int which, double* out) {
  if (!h || !out || which < 0 || which > 1) return set_err(FDMAP_ERR_INVALID_ARG, "bad get_pml arguments");
  CUDA_TRY(cudaSetDevice(h->device));
  const int nF = h->nF;
  const long long NN = (long long)h->nx_g * h->ny_g;
  CUDA_TRY(cudaMemsetAsync(h->d_global, 0, (size_t)NN * nF * sizeof(double), h->stream));
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    const double* W = which == 0 ? h->hdom.blk[b].Wx : h->hdom.blk[b].Wy;
    if (!W) continue;
    const BlockGeom& g = h->geom[b];
    dim3 grid((g.pitch + 255) / 256, g.ny);
    gather_block<<<grid, 256, 0, h->stream>>>(W, h->d_global, h->nx_g, NN, g.mgx, g.mgy, g.nx, g.ny, g.pitch, g.plane,
                                              nF);
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaMemcpyAsync(out, h->d_global, (size_t)NN * nF * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return FDMAP_OK;
}

int fdmap_gpu_set_pml(fdmap_gpu* h, int which, const double* in) {
  if (!h || !in || which < 0 || which > 1) return set_err(FDMAP_ERR_INVALID_ARG, "bad set_pml arguments");
  CUDA_TRY(cudaSetDevice(h->device));
  const int nF = h->nF;
  const long long NN = (long long)h->nx_g * h->ny_g;
  CUDA_TRY(cudaMemcpyAsync(h->d_global, in, (size_t)NN * nF * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    double* W = which == 0 ? h->hdom.blk[b].Wx : h->hdom.blk[b].Wy;
    if (!W) continue;
    const BlockGeom& g = h->geom[b];
    dim3 grid((g.pitch + 255) / 256, g.ny);
    scatter_block<<<grid, 256, 0, h->stream>>>(h->d_global, W, h->nx_g, NN, g.mgx, g.mgy, g.nx, g.ny, g.pitch, g.plane,
                                               nF);
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return FDMAP_OK;
}

int fdmap_gpu_get_side_displacement(fdmap_gpu* h, int b, int s, double* U, double* DU) {
  if (!h || b < 0 || b >= h->hdom.nblocks || s < 0 || s > 3)
    return set_err(FDMAP_ERR_INVALID_ARG, "bad get_side_displacement arguments");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  const DevSide& S = h->hdom.blk[b].side[s];
  const size_t nu = (size_t)S.n * (h->mode == 2 ? 2 : 1);
  if (U) CUDA_TRY(cudaMemcpy(U, S.U, nu * sizeof(double), cudaMemcpyDeviceToHost));
  if (DU) CUDA_TRY(cudaMemcpy(DU, S.DU, nu * sizeof(double), cudaMemcpyDeviceToHost));
  return FDMAP_OK;
}

int fdmap_gpu_set_side_displacement(fdmap_gpu* h, int b, int s, const double* U, const double* DU) {
  if (!h || b < 0 || b >= h->hdom.nblocks || s < 0 || s > 3)
    return set_err(FDMAP_ERR_INVALID_ARG, "bad set_side_displacement arguments");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  const DevSide& S = h->hdom.blk[b].side[s];
  const size_t nu = (size_t)S.n * (h->mode == 2 ? 2 : 1);
  if (U) CUDA_TRY(cudaMemcpy(S.U, U, nu * sizeof(double), cudaMemcpyHostToDevice));
  if (DU) CUDA_TRY(cudaMemcpy(S.DU, DU, nu * sizeof(double), cudaMemcpyHostToDevice));
  return FDMAP_OK;
}

int fdmap_gpu_get_side_impedance(fdmap_gpu* h, int b, int s, double* out) {
  if (!h || !out || b < 0 || b >= h->hdom.nblocks || s < 0 || s > 3)
    return set_err(FDMAP_ERR_INVALID_ARG, "bad get_side_impedance arguments");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  const DevSide& S = h->hdom.blk[b].side[s];
  CUDA_TRY(cudaMemcpy(out, S.M, (size_t)S.n * 5 * sizeof(double), cudaMemcpyDeviceToHost));
  return FDMAP_OK;
}

int fdmap_gpu_get_fault(fdmap_gpu* h, int iface, int field, double* out) {
  if (!h || !out || iface < 0 || iface >= h->hdom.nifaces || field < 0 || field >= FDMAP_FAULT_NFIELDS)
    return set_err(FDMAP_ERR_INVALID_ARG, "bad get_fault arguments");
  if (!h->iface_fric[iface]) return set_err(FDMAP_ERR_INVALID_ARG, "interface is not frictional");
  CUDA_TRY(cudaSetDevice(h->device));
  int n = h->iface_n[iface];
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CUDA_TRY(cudaMemcpy(out, h->hdom.ifc[iface].fr.st + (size_t)field * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  return FDMAP_OK;
}

int fdmap_gpu_set_fault(fdmap_gpu* h, int iface, int field, const double* in) {
  if (!h || !in || iface < 0 || iface >= h->hdom.nifaces || field < 0 || field >= FDMAP_FAULT_NFIELDS)
    return set_err(FDMAP_ERR_INVALID_ARG, "bad set_fault arguments");
  if (!h->iface_fric[iface]) return set_err(FDMAP_ERR_INVALID_ARG, "interface is not frictional");
  CUDA_TRY(cudaSetDevice(h->device));
  int n = h->iface_n[iface];
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CUDA_TRY(cudaMemcpy(h->hdom.ifc[iface].fr.st + (size_t)field * n, in, n * sizeof(double), cudaMemcpyHostToDevice));
  return FDMAP_OK;
}

int fdmap_gpu_get_fhat(fdmap_gpu* h, int b, int s, double* out) {
  if (!h || !out || b < 0 || b >= h->hdom.nblocks || s < 0 || s > 3)
    return set_err(FDMAP_ERR_INVALID_ARG, "bad get_fhat arguments");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CUDA_TRY(cudaMemcpy(out, h->dev_fhat[b][s], (size_t)h->side_n[b][s] * h->nF * sizeof(double),
                      cudaMemcpyDeviceToHost));
  return FDMAP_OK;
}

int fdmap_gpu_status(fdmap_gpu* h, long long* newton_failures) {
  long long counts[2] = {0, 0};
  const int rc = fdmap_gpu_newton_counts(h, counts);
  if (newton_failures) *newton_failures = counts[0];
  return rc;
}

int fdmap_gpu_newton_counts(fdmap_gpu* h, long long* counts) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  unsigned long long st[4];
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CUDA_TRY(cudaMemcpy(st, h->d_status, sizeof(st), cudaMemcpyDeviceToHost));
  if (counts) {
    counts[0] = (long long)st[0];
    counts[1] = (long long)st[3];
  }
  if (st[1] & 2ull) return set_err(FDMAP_ERR_TIMEOUT, "a bounded device wait gave up");
  if (st[3]) return set_err(FDMAP_ERR_NEWTON_NOCONV, std::to_string(st[3]) + " Newton solves failed twice");
  return FDMAP_OK;
}

int fdmap_gpu_clear_status(fdmap_gpu* h) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CUDA_TRY(cudaMemset(h->d_status, 0, 4 * sizeof(unsigned long long)));
  return FDMAP_OK;
}

int fdmap_gpu_trace(fdmap_gpu* h, int capacity) {
  if (!h || capacity < 0) return set_err(FDMAP_ERR_INVALID_ARG, "bad trace arguments");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  TraceBuf& T = h->hdom.trace;
  if (capacity > 0 && (unsigned)capacity > T.cap) {
    unsigned long long* rec = nullptr;
    unsigned int* n = nullptr;
    int rc;
    if ((rc = h->alloc(&rec, (size_t)capacity * 3)) || (rc = h->alloc(&n, 1))) return rc;
    h->trace_rec = rec;
    T.n = n;
    T.cap = (unsigned)capacity;
  }
  if (capacity == 0) {
    T.rec = nullptr;  // off; the records taken so far stay readable
  } else {
    T.rec = h->trace_rec;
    CUDA_TRY(cudaMemset(T.n, 0, sizeof(unsigned int)));
  }
  CUDA_TRY(cudaMemcpy(h->ddom, &h->hdom, sizeof(DevDomain), cudaMemcpyHostToDevice));
  for (auto& ge : h->step_graph)  // the graphs carry the domain by value
    if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  h->graph_dt = 0.0;
  return FDMAP_OK;
}

int fdmap_gpu_trace_read(fdmap_gpu* h, unsigned long long* records, int max) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  const TraceBuf& T = h->hdom.trace;
  if (!T.n) return 0;
  const unsigned long long* rec = h->trace_rec;
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  unsigned int n = 0;
  CUDA_TRY(cudaMemcpy(&n, T.n, sizeof(n), cudaMemcpyDeviceToHost));
  n = std::min<unsigned>(n, T.cap);
  const int k = std::min<int>((int)n, max);
  if (records && k > 0) CUDA_TRY(cudaMemcpy(records, rec, (size_t)k * 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return (int)n;
}

int fdmap_gpu_set_tile(fdmap_gpu* h, int tile) {
  if (!h || tile < 0 || tile >= MARCH_SHAPES) return set_err(FDMAP_ERR_INVALID_ARG, "tile must be 0..3");
  return march_set_shape(h, tile);
}

int fdmap_gpu_get_tile(fdmap_gpu* h, int* tile, int* mw, int* mr) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  if (!h->use_march) return set_err(FDMAP_ERR_UNSUPPORTED, "the domain uses the tiled interior kernel");
  if (tile) *tile = h->march_shape;
  if (mw) *mw = shape_mw(h->march_shape);
  if (mr) *mr = shape_mr(h->march_shape);
  return FDMAP_OK;
}

int fdmap_gpu_tune(fdmap_gpu* h, double dt, int steps, int* best_tile, double* best_ms) {
  if (!h || steps < 1) return set_err(FDMAP_ERR_INVALID_ARG, "bad tune arguments");
  if (!h->use_march) return set_err(FDMAP_ERR_UNSUPPORTED, "the domain uses the tiled interior kernel");
  if (h->partitioned()) return set_err(FDMAP_ERR_UNSUPPORTED, "a partition is not tuned on its own");
  if (output_is_open(h)) return set_err(FDMAP_ERR_INVALID_ARG, "tune before opening the outputs");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  std::vector<void*> saved;
  int rc = state_snapshot(h, saved, h->stream);
  if (rc) return rc;
  const int cur0 = h->cur, shape0 = h->march_shape;
  const bool pairs0 = h->use_pairs;
  const long long out0 = h->out_next_n;
  int best = shape0;
  bool best_pairs = pairs0;
  float best_t = -1.f;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  auto set_pairs = [&](bool on) {
    if (h->use_pairs == on) return;
    h->use_pairs = on;
    for (auto& ge : h->step_graph)
      if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  };
  // every tile shape, with two-stage passes on and off where the domain can
  // take them (small, L2-resident domains step faster stage by stage)
  for (int k = 0; k < (h->pair_ok ? 2 : 1) * MARCH_SHAPES && rc == FDMAP_OK; ++k) {
    const int sh = k % MARCH_SHAPES;
    const bool pv = h->pair_ok ? k < MARCH_SHAPES : pairs0;
    set_pairs(pv);
    rc = march_set_shape(h, sh);
    if (rc == FDMAP_ERR_UNSUPPORTED) { rc = FDMAP_OK; continue; }
    if (rc) break;
    // warm-up step (captures the graphs), then two timed repetitions; the faster counts
    if ((rc = fdmap_gpu_run(h, 0.0, dt, 1, 1, 1 << 30))) break;
    float ms = -1.f;
    for (int rep = 0; rep < 2 && rc == FDMAP_OK; ++rep) {
      cudaEventRecord(t0, h->stream);
      if ((rc = fdmap_gpu_run(h, 0.0, dt, 2, 1 + steps, 1 << 30))) break;
      cudaEventRecord(t1, h->stream);
      if (cudaEventSynchronize(t1) != cudaSuccess) { rc = set_err(FDMAP_ERR_CUDA, "tuning run failed"); break; }
      float m = 0.f;
      cudaEventElapsedTime(&m, t0, t1);
      if (ms < 0.f || m < ms) ms = m;
    }
    if (rc == FDMAP_OK && (best_t < 0.f || ms < best_t)) { best_t = ms; best = sh; best_pairs = pv; }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  const int rr = state_restore(h, saved, h->stream);
  h->cur = cur0;
  h->out_next_n = out0;
  if (rc) { set_pairs(pairs0); march_set_shape(h, shape0); return rc; }
  if (rr) return rr;
  set_pairs(best_pairs);
  if ((rc = march_set_shape(h, best))) return rc;
  if (best_tile) *best_tile = best;
  if (best_ms) *best_ms = best_t / steps;
  return FDMAP_OK;
}

int fdmap_gpu_set_newton_limit(fdmap_gpu* h, int imax) {
  if (!h || imax < 1 || imax > 99) return set_err(FDMAP_ERR_INVALID_ARG, "Newton iteration limit must be 1..99");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->hdom.newton_imax = imax;
  CUDA_TRY(cudaMemcpy(h->ddom, &h->hdom, sizeof(DevDomain), cudaMemcpyHostToDevice));
  // the step graphs carry the domain by value: capture them again
  for (auto& ge : h->step_graph)
    if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  h->graph_dt = 0.0;
  return FDMAP_OK;
}

int fdmap_gpu_test_wait_timeout(fdmap_gpu* h, double limit_s) {
  if (!h || !(limit_s > 0.0) || limit_s > 10.0) return set_err(FDMAP_ERR_INVALID_ARG, "limit must be in (0, 10] s");
  CUDA_TRY(cudaSetDevice(h->device));
  wait_timeout_probe<<<1, 32, 0, h->stream>>>(h->d_status, (unsigned long long)(limit_s * 1e9));
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return FDMAP_OK;
}

int fdmap_gpu_check_finite(fdmap_gpu* h, long long* count) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  unsigned long long* d_count = h->d_status + 2;  // scratch word of the status block
  CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), h->stream));
  for (int b = 0; b < h->hdom.nblocks; ++b) {
    if (!h->owns(b)) continue;  // body on a peer GPU
    const DevBlock& B = h->hdom.blk[b];
    const long long n = (long long)h->nF * B.ny * B.nx;
    count_nonfinite_block<<<(int)std::min<long long>((n + 255) / 256, 4 * 148), 256, 0, h->stream>>>(
        B.F[h->cur], B.nx, B.ny, B.pitch, B.plane, h->nF, d_count);
    CUDA_TRY(cudaGetLastError());
  }
  for (int i = 0; i < h->hdom.nifaces; ++i) {
    const DevIface& I = h->hdom.ifc[i];
    if (I.coupling != FDMAP_COUPLING_FRICTION) continue;
    const int fields[3] = {ST_V, ST_S, ST_PSI};
    for (int f : fields) {
      count_nonfinite_block<<<(I.n + 255) / 256, 256, 0, h->stream>>>(I.fr.st + (size_t)f * I.n, I.n, 1, I.n, I.n, 1,
                                                                      d_count);
      CUDA_TRY(cudaGetLastError());
    }
  }
  unsigned long long c = 0;
  CUDA_TRY(cudaMemcpyAsync(&c, d_count, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (count) *count = (long long)c;
  return c ? set_err(FDMAP_ERR_NONFINITE, std::to_string(c) + " non-finite values") : FDMAP_OK;
}

int fdmap_gpu_set_stream(fdmap_gpu* h, void* stream) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return FDMAP_OK;
}

int fdmap_gpu_profile(fdmap_gpu* h, int enable) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  h->drain_events();
  h->profiling = enable != 0;
  for (int k = 0; k < 5; ++k) { h->prof_ms[k] = 0.0; h->prof_n[k] = 0; }
  return FDMAP_OK;
}

int fdmap_gpu_profile_read_kinds(fdmap_gpu* h, int n, double* ms, long long* count) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  if (n < 0 || n > 5) return set_err(FDMAP_ERR_INVALID_ARG, "at most 5 kernel kinds");
  CUDA_TRY(cudaSetDevice(h->device));
  h->drain_events();
  for (int k = 0; k < n; ++k) {
    if (ms) ms[k] = h->prof_ms[k];
    if (count) count[k] = h->prof_n[k];
  }
  return FDMAP_OK;
}

int fdmap_gpu_set_pairs(fdmap_gpu* h, int enable) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  if (enable && !h->pair_ok) return set_err(FDMAP_ERR_UNSUPPORTED, "the domain cannot run two-stage passes");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (h->use_pairs != (enable != 0)) {
    h->use_pairs = enable != 0;
    for (auto& ge : h->step_graph)
      if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  }
  return FDMAP_OK;
}

int fdmap_gpu_get_pairs(fdmap_gpu* h) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  return h->use_pairs ? 1 : 0;
}

int fdmap_gpu_profile_read(fdmap_gpu* h, double* ms, long long* count) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  CUDA_TRY(cudaSetDevice(h->device));
  h->drain_events();
  for (int k = 0; k < 3; ++k) {
    if (ms) ms[k] = h->prof_ms[k];
    if (count) count[k] = h->prof_n[k];
  }
  return FDMAP_OK;
}

long long fdmap_gpu_launch_count(fdmap_gpu* h) { return h ? h->launches : -1; }

long long fdmap_gpu_device_bytes(fdmap_gpu* h) { return h ? h->bytes : -1; }

void fdmap_gpu_destroy(fdmap_gpu* h) { delete h; }

const char* fdmap_gpu_strerror(int code) {
  switch (code) {
    case FDMAP_OK: return "ok";
    case FDMAP_ERR_INVALID_ARG: return "invalid argument";
    case FDMAP_ERR_CUDA: return "CUDA error";
    case FDMAP_ERR_NONFINITE: return "non-finite value detected";
    case FDMAP_ERR_NEWTON_NOCONV: return "friction Newton solver did not converge";
    case FDMAP_ERR_TIMEOUT: return "device wait timed out";
    case FDMAP_ERR_UNSUPPORTED: return "unsupported configuration";
    case FDMAP_ERR_IO: return "I/O error";
    case FDMAP_ERR_NOMEM: return "out of memory";
  }
  return "unknown error";
}

const char* fdmap_gpu_last_error(void) { return g_err.c_str(); }

}  // extern "C"
