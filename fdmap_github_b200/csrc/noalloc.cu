// fdmap_gpu_fault_max_noalloc: max |field| along one interface, computed on
// the device with no memory allocation of any kind during the call.
//
// Why: a driver that monitors the rupture every step (the maximum slip rate
// against a nucleation or arrest threshold) calls this in its time loop.
// Such callers cannot allocate there: cudaMalloc / cudaFree synchronise the
// device and would stall the asynchronous step pipeline, and a driver whose
// HBM is fully reserved by its domains (large ensembles) has no room to hand
// out.  The existing path, fdmap_gpu_get_fault, copies the whole field to the
// host instead.
//
// Scratch: the per-CTA partial maxima and the result live in a file-scope
// static device array of NOALLOC_MAX_PARTIALS + 1 doubles (8 KiB + 8 B); the
// completion counter is a static device word.  Limits and rules:
//  - at most NOALLOC_MAX_PARTIALS CTAs of NOALLOC_PER_CTA nodes each, i.e.
//    faults of up to 1,048,576 nodes; longer ones are rejected
//    (FDMAP_ERR_UNSUPPORTED) before anything is launched;
//  - the completion counter must be zero when a call starts: every call
//    clears it with cudaMemsetAsync on its stream before the launch (a memset
//    allocates nothing), so a counter left over by an earlier call that never
//    finished cannot make a CTA mistake itself for the last one;
//  - a NaN anywhere in the field makes the result NaN (the maximum does not
//    skip it the way fmax would), so a blown-up slip rate is not reported as
//    a finite maximum;
//  - the partials need no initial value: each CTA writes its own slot before
//    it counts itself done;
//  - the scratch is shared by every handle on a device: two calls that overlap
//    in time on the same device (from two host threads, or on two streams)
//    race on it.  Calls on one device must not overlap;
//  - the first call on a device looks up the scratch address
//    (cudaGetSymbolAddress) and caches it; make that first call before any
//    stream capture begins.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.h"
#include "fdmap_gpu.h"

namespace {

constexpr int NOALLOC_MAX_PARTIALS = 1024;
constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_PER_THREAD = 4;
constexpr int NOALLOC_PER_CTA = NOALLOC_THREADS * NOALLOC_PER_THREAD;
constexpr int NOALLOC_MAX_DEVICES = 64;

// [0, NOALLOC_MAX_PARTIALS): per-CTA partial maxima; [NOALLOC_MAX_PARTIALS]: result
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_PARTIALS + 1];
// CTAs finished in the current call; zero between calls
static __device__ __align__(256) unsigned int g_noalloc_done;

struct ScratchPtrs {
  double* partials = nullptr;
  unsigned int* done = nullptr;
};
ScratchPtrs g_ptrs[NOALLOC_MAX_DEVICES];
std::mutex g_ptrs_mutex;

// once per device, with that device current
int scratch_for(int device, ScratchPtrs* out) {
  if (device < 0 || device >= NOALLOC_MAX_DEVICES) return set_err(FDMAP_ERR_UNSUPPORTED, "device index too large");
  std::lock_guard<std::mutex> lock(g_ptrs_mutex);
  ScratchPtrs& p = g_ptrs[device];
  if (!p.partials) {
    cudaError_t e = cudaGetSymbolAddress((void**)&p.partials, g_noalloc_scratch);
    if (e != cudaSuccess) {
      p.partials = nullptr;
      return set_err(FDMAP_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    }
    e = cudaGetSymbolAddress((void**)&p.done, g_noalloc_done);
    if (e != cudaSuccess) {
      p.partials = nullptr;
      p.done = nullptr;
      return set_err(FDMAP_ERR_CUDA, std::string("cudaGetSymbolAddress(counter): ") + cudaGetErrorString(e));
    }
  }
  *out = p;
  return FDMAP_OK;
}

// maximum that propagates NaN: a NaN operand wins (fmax would drop it)
__device__ __forceinline__ double max_nan(double a, double b) { return (b != b || b > a) ? b : a; }

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max_nan(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// max |x[0..n)|: each CTA reduces NOALLOC_PER_CTA nodes into partials[cta];
// the last CTA to finish folds the partials into partials[NOALLOC_MAX_PARTIALS].
__global__ void __launch_bounds__(NOALLOC_THREADS) fault_absmax_kernel(const double* __restrict__ x, int n,
                                                                       double* partials, unsigned int* done) {
  __shared__ double warp_part[NOALLOC_THREADS / 32];
  __shared__ bool last;
  double m = 0.0;
  const int base = blockIdx.x * NOALLOC_PER_CTA + threadIdx.x;
#pragma unroll
  for (int q = 0; q < NOALLOC_PER_THREAD; ++q) {
    const int k = base + q * NOALLOC_THREADS;
    if (k < n) m = max_nan(m, fabs(x[k]));
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < NOALLOC_THREADS / 32 ? warp_part[threadIdx.x] : 0.0;
    v = warp_max(v);
    if (threadIdx.x == 0) {
      partials[blockIdx.x] = v;
      __threadfence();
      last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (!last) return;
  // last CTA: every other CTA's partial is visible (written before its count)
  __threadfence();
  double v = 0.0;
  for (int c = threadIdx.x; c < (int)gridDim.x; c += NOALLOC_THREADS)
    v = max_nan(v, ((volatile double*)partials)[c]);
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < NOALLOC_THREADS / 32; ++w) r = max_nan(r, warp_part[w]);
    partials[NOALLOC_MAX_PARTIALS] = r;
  }
}

}  // namespace

extern "C" int fdmap_gpu_fault_max_noalloc(fdmap_gpu* h, int iface, int field, double* out) {
  if (!h || !out) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  if (iface < 0 || iface >= h->hdom.nifaces) return set_err(FDMAP_ERR_INVALID_ARG, "interface index out of range");
  if (field < 0 || field >= FDMAP_FAULT_NFIELDS) return set_err(FDMAP_ERR_INVALID_ARG, "fault field out of range");
  const DevIface& I = h->hdom.ifc[iface];
  if (!I.fr.st) return set_err(FDMAP_ERR_INVALID_ARG, "interface has no friction state (locked coupling)");
  const int n = I.n;
  const long long ctas = ((long long)n + NOALLOC_PER_CTA - 1) / NOALLOC_PER_CTA;
  if (ctas > NOALLOC_MAX_PARTIALS)
    return set_err(FDMAP_ERR_UNSUPPORTED, "fault longer than 1,048,576 nodes: beyond the static scratch of fdmap_gpu_fault_max_noalloc");
  CUDA_TRY(cudaSetDevice(h->device));
  ScratchPtrs sp;
  int rc = scratch_for(h->device, &sp);
  if (rc) return rc;
  if (n == 0) {
    *out = 0.0;
    return FDMAP_OK;
  }
  const double* x = I.fr.st + (size_t)field * n;
  CUDA_TRY(cudaMemsetAsync(sp.done, 0, sizeof(unsigned int), h->stream));
  fault_absmax_kernel<<<(int)ctas, NOALLOC_THREADS, 0, h->stream>>>(x, n, sp.partials, sp.done);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(out, sp.partials + NOALLOC_MAX_PARTIALS, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return FDMAP_OK;
}
