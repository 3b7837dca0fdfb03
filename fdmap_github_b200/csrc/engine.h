// Internal header of the engine: the handle behind include/fdmap_gpu.h and
// the launchers that other translation units of the library (ensemble,
// adjoint) call.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "device_common.cuh"
#include "fdmap_gpu.h"
#include "sbp_tables.h"

namespace fdmap {

int set_err(int code, const std::string& msg);
extern thread_local std::string g_err;

#define CUDA_TRY(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return ::fdmap::set_err(FDMAP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct BlockGeom {
  int mgx, mgy, nx, ny, pitch;
  long long plane;
};

struct OutputState;  // device-side output (output.cu)
struct TmapPair;     // tensor maps of the two-stage march (march_pair.cuh)
void output_destroy(fdmap_gpu* h);

__global__ void advance_step(TimeState* ts);
void pair_free(fdmap_gpu* h);  // releases the two-stage march's host-side maps (march_pair.cu)
__global__ void set_step_clock(TimeState* ts, double t_start, double dt, long long n);

}  // namespace fdmap

using namespace fdmap;  // internal header: the handle below is written in the engine's namespace terms

struct fdmap_gpu {
  int device = 0;
  cudaStream_t stream = nullptr;
  DevDomain hdom{};
  DevDomain* ddom = nullptr;
  std::vector<void*> allocs;
  std::vector<size_t> alloc_sizes;  // bytes of each allocation (state snapshots for the autotuner)
  long long bytes = 0;
  int cur = 0;
  int mode = 2, nF = 6, pI = 2, het = 0;
  RkTable rk{};
  int nx_g = 0, ny_g = 0;
  std::vector<BlockGeom> geom;
  std::vector<int> iface_n;
  std::vector<int> iface_fric;
  int total_tiles = 0, edge_threads = 0;
  long long closure_threads = 0;
  long long march_units = 0;
  int march_grid = 0;
  int use_march = 1;
  int march_shape = 0;      // tile shape of the march (shape_mw / shape_mr)
  int march_ext = 0;        // march variant: 0 plain, 1 dissipation / forcing / body extras, 2 PML (+ forcing, extras)
  bool dissipation = false;  // some block has Cdiss > 0 (tiled interior kernel)
  bool pml = false;  // some block has a perfectly matched layer (tiled interior kernel)
  bool forcing = false;  // tsunami forcing or forcing from file (tiled interior kernel)
  bool extras = false;   // body displacement or peak motion tracked (tiled interior kernel)
  double* d_energy = nullptr;  // [nblocks + 1] stage-1 energies (energy_balance = T)
  double* d_epart = nullptr;   // their partial sums
  std::FILE* frc_file = nullptr;  // forcing frames, one (nx,ny,nF) frame per step
  std::vector<double> frc_host;   // the frame being loaded
  bool body_on_device = false;  // body built by build_body (fdmap_desc.body)
  double tp[5] = {0, 0, 0, 0, 0};  // t0, dt, CFL, hmin, hmax (set_dt)
  int tp_nt = 0;
  int fused = 0;  // boundary kernel handles interface solves and closure strips in one launch
  // two-stage passes (march_pair.cuh): stages 2k+1, 2k+2 of a step in one
  // interior pass; available for homogeneous plain domains (pair_ok), used
  // when also enabled (use_pairs)
  bool pair_ok = false;
  bool use_pairs = false;
  TmapPair* tmaps_pair = nullptr;
  long long pair_units = 0;
  int pair_grid = 0;
  long long band_threads = 0;
  // CUDA graphs of one full step, one per starting F buffer, replayed by fdmap_gpu_run
  TimeState* d_time = nullptr;
  cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
  double graph_dt = 0.0;
  long long graph_launches = 0;
  bool use_graphs = true;
  double* met_base[MAX_BLOCKS] = {};
  double* het_base[MAX_BLOCKS] = {};
  TmapSet* tmaps = nullptr;  // host copy, passed by value to the march kernel
  double* d_global = nullptr;  // one field set in FDMAP's global layout: get/set_fields staging
  unsigned long long* d_status = nullptr;
  long long launches = 0;
  double* dev_fhat[MAX_BLOCKS][4] = {};
  int side_n[MAX_BLOCKS][4] = {};
  cudaStream_t own_stream = nullptr;
  // device-side output (fdmap_gpu_output_*): open state and the next step index
  OutputState* out = nullptr;
  long long out_next_n = 1;
  // boundary work (interface solves, closure strips) runs on a low-priority
  // side stream beside the interior march of the same stage
  bool overlap = false;
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // block-aligned partition (fdmap_gpu_create_part): the blocks this handle
  // steps; the other blocks' body arrays live on peer GPUs
  std::vector<char> owned;
  std::vector<int> part_ifaces;       // interfaces with exactly one side here
  fdmap_exchange_fn exchange = nullptr;
  void* exchange_user = nullptr;
  long long xstage = 0;               // stages issued (selects the send slot)
  unsigned long long* trace_rec = nullptr;  // timeline records (fdmap_gpu_trace), kept while tracing is off
  cudaEvent_t ev_packed = nullptr;    // the stage's edge values are packed
  bool owns(int b) const { return owned.empty() || owned[(size_t)b] != 0; }
  bool partitioned() const { return !owned.empty(); }
  // per-kernel event timing (fdmap_gpu_profile)
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;  // kind, (start, stop)
  // kinds: 0 interior march, 1 closure strips, 2 interface solves, 3 two-stage march, 4 band
  double prof_ms[5] = {0, 0, 0, 0, 0};
  long long prof_n[5] = {0, 0, 0, 0, 0};

  template <typename T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    size_t bytes_ = count * sizeof(T);
    if (bytes_ == 0) bytes_ = 16;
    cudaError_t e = cudaMalloc(&q, bytes_);
    if (e != cudaSuccess) return set_err(FDMAP_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(q);
    alloc_sizes.push_back(bytes_);
    bytes += (long long)bytes_;
    *p = (T*)q;
    return FDMAP_OK;
  }
  // field arrays: PADL doubles of front padding so halo bulk copies may start
  // before column 0; every plane carries PADTAIL doubles of slack after its last row
  int alloc_planes(double** base, int nplanes, long long plane) {
    double* raw = nullptr;
    int rc = alloc(&raw, (size_t)PADL + (size_t)nplanes * plane);
    if (rc) return rc;
    CUDA_TRY(cudaMemset(raw, 0, ((size_t)PADL + (size_t)nplanes * plane) * sizeof(double)));
    *base = raw + PADL;
    return FDMAP_OK;
  }
  int upload(double** dst, const double* src, size_t count) {
    int rc = alloc(dst, count);
    if (rc) return rc;
    if (src) CUDA_TRY(cudaMemcpy(*dst, src, count * sizeof(double), cudaMemcpyHostToDevice));
    return FDMAP_OK;
  }
  // global (nx_g, ny_g) plane -> padded block plane on the device
  int upload_plane(double* dst, const double* src, const BlockGeom& g) {
    std::vector<double> tmp((size_t)g.plane, 0.0);
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i)
        tmp[(size_t)j * g.pitch + i] = src[(size_t)(g.mgx - 1 + i) + (size_t)nx_g * (size_t)(g.mgy - 1 + j)];
    CUDA_TRY(cudaMemcpy(dst, tmp.data(), tmp.size() * sizeof(double), cudaMemcpyHostToDevice));
    return FDMAP_OK;
  }
  cudaEvent_t take_event() {
    cudaEvent_t e;
    if (!ev_pool.empty()) { e = ev_pool.back(); ev_pool.pop_back(); }
    else cudaEventCreate(&e);
    return e;
  }
  // folds finished event pairs into the totals (blocking on the last one)
  void drain_events() {
    for (auto& p : ev_pending) {
      cudaEventSynchronize(p.second.second);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, p.second.first, p.second.second);
      prof_ms[p.first] += ms;
      prof_n[p.first] += 1;
      ev_pool.push_back(p.second.first);
      ev_pool.push_back(p.second.second);
    }
    ev_pending.clear();
  }
  ~fdmap_gpu() {
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (frc_file) std::fclose(frc_file);
    for (auto& p : ev_pending) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
    for (auto e : ev_pool) cudaEventDestroy(e);
    for (void* p : allocs) cudaFree(p);
    if (own_stream) cudaStreamDestroy(own_stream);
    if (side_stream) cudaStreamDestroy(side_stream);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_packed) cudaEventDestroy(ev_packed);
    output_destroy(this);
    delete tmaps;
    pair_free(this);
    for (auto& ge : step_graph)
      if (ge) cudaGraphExecDestroy(ge);
  }
};

namespace fdmap {

// device-side output hooks (output.cu)
bool output_is_open(const fdmap_gpu* h);
int output_before_step(fdmap_gpu* h, long long n, double t);
int output_gather(fdmap_gpu* h, const TimeState* ts, long long n, int cur);

// Launchers over a batch of independent domains (one DevDomain per instance,
// in device memory).  `proto` supplies the compile-time variant (mode, SBP
// order, heterogeneity); every instance must share it.
struct BatchPlan {
  const DevDomain* doms;          // [ninst] device copies of each instance's domain
  const TmapSet* tmaps;           // [ninst] device copies of each instance's tensor maps
  const long long* unit_begin;    // [ninst+1] march units, prefix over instances
  const int* closure_cta_begin;   // [ninst+1] closure CTAs, prefix over instances
  const int* edge_cta_begin;      // [ninst+1] interface CTAs, prefix over instances
  int ninst;
  long long units;
  int march_grid;
  int closure_ctas, closure_tpb;
  int edge_ctas, edge_tpb;
};
// Stage-1 mechanical energy of every block into h->d_energy (energy.cu), from
// the fields of buffer `cur`.
int launch_energy(fdmap_gpu* h, int cur);
int energy_scratch_size(int nblocks);

// Builds the body of a domain whose descriptor carries fdmap_desc.body
// (body_init.cu) into the already allocated block planes and side arrays, and
// finishes set_dt into h->tp / h->tp_nt and each block's scaled Cdiss.
int build_body(fdmap_gpu* h, const fdmap_desc* d, const SbpOperator& op);

// One RK stage of a single domain (boundary + interior kernels) on h->stream.
int engine_stage(fdmap_gpu* h, const StageArgs& a);

int batch_march(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s);

// The interior march for tile shape 0..3 (march_s<N>.cu): configure sets the
// unit decomposition, tensor maps and grid for that shape (FDMAP_ERR_UNSUPPORTED
// when the shape cannot serve the handle's variant); launch issues one stage.
int march_configure_s0(fdmap_gpu* h);
int march_configure_s1(fdmap_gpu* h);
int march_configure_s2(fdmap_gpu* h);
int march_configure_s3(fdmap_gpu* h);
int march_launch_s0(fdmap_gpu* h, const StageArgs& a);
int march_launch_s1(fdmap_gpu* h, const StageArgs& a);
int march_launch_s2(fdmap_gpu* h, const StageArgs& a);
int march_launch_s3(fdmap_gpu* h, const StageArgs& a);
int march_batch_s0(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s);
int march_batch_s1(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s);
int march_batch_s2(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s);
int march_batch_s3(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s);
// configure for `shape` and publish the domain (device copy, step graphs dropped)
int march_set_shape(fdmap_gpu* h, int shape);

// Two-stage passes (march_pair.cu).  pair_configure checks whether the
// handle's domain can use them (homogeneous material, plain split form, SBP2
// or SBP4, blocks wider than two bands), allocates the scratch field buffer
// F[2] and the second rate buffer, builds the band table and the tensor maps,
// and sets h->pair_ok; it leaves the handle unchanged when the domain does
// not qualify.  pair_launch issues the interior pass of stages a0, a1;
// band_launch the band kernel of the second stage.
int pair_configure(fdmap_gpu* h);
int pair_launch(fdmap_gpu* h, const StageArgs& a0, const StageArgs& a1, int dfr, int dfw);
int band_launch(fdmap_gpu* h, const StageArgs& a);

// Two-stage passes over a batch of instances (ensemble.cu): the pass walks the
// concatenated units of every instance, the band kernel the concatenated bands.
struct PairBatch {
  const DevDomain* doms;           // [ninst] device copies of each instance's domain
  const TmapPair* tmaps;           // [ninst] device copies of each instance's pass tensor maps
  const long long* unit_begin;     // [ninst+1] pass units, prefix over instances
  const int* band_cta_begin;       // [ninst+1] band CTAs (128 threads), prefix over instances
  int ninst;
  long long units;
  int grid;
  int band_ctas;
};
int pair_batch(const fdmap_gpu* proto, const StageArgs& a0, const StageArgs& a1, int dfr, int dfw,
               const PairBatch& p, cudaStream_t s);
int band_batch(const fdmap_gpu* proto, const StageArgs& a, const PairBatch& p, cudaStream_t s);

// Copy of every device allocation of a handle (its whole state), to put the
// state back after timing runs; `out` receives the copies (freed by restore).
int state_snapshot(fdmap_gpu* h, std::vector<void*>& out, cudaStream_t s);
int state_restore(fdmap_gpu* h, std::vector<void*>& saved, cudaStream_t s);
int batch_closure(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s);
int batch_edges(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s);

}  // namespace fdmap
