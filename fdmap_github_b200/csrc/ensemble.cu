// Batched ensemble: many independent FDMAP domains (instances of uneven
// grid sizes and their own prestress) advanced together.  Every stage is one
// launch per kernel kind for ALL instances:
//   - the persistent interior march walks the concatenated row-group units of
//     every block of every instance (one CTA per SM, balanced partition);
//   - one interface launch covers every fault node of every instance;
//   - one closure launch covers every SBP boundary strip of every instance.
// Per-node arithmetic is the single-domain kernels' own, so every instance
// reproduces its plain single-domain run bit for bit.  Each step is captured
// once as a CUDA graph and replayed.  Launch shapes (thread-block sizes of the
// boundary kernels, boundary/interior overlap) are picked by a timing-based
// autotuner (fdmap_gpu_ensemble_tune).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "engine.h"
#include "fdmap_gpu.h"
#include "march_kernel.cuh"
#include "march_pair.cuh"

using namespace fdmap;

struct fdmap_ensemble {
  int device = 0;
  int ninst = 0;
  std::vector<fdmap_gpu*> inst;
  fdmap_gpu* proto = nullptr;  // instance 0: compile-time variant of all
  cudaStream_t stream = nullptr, side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  DevDomain* d_doms = nullptr;
  TmapSet* d_tmaps = nullptr;
  long long* d_unit_begin = nullptr;
  int* d_closure_begin = nullptr;
  int* d_edge_begin = nullptr;
  TimeState* d_time = nullptr;
  std::vector<long long> closure_threads, edge_threads;
  BatchPlan plan{};
  // two-stage passes over every instance (all instances able to take them)
  TmapPair* d_pmaps = nullptr;
  long long* d_pair_begin = nullptr;
  int* d_band_begin = nullptr;
  PairBatch pplan{};
  bool pair_ok = false;
  bool pairs = false;
  bool pairs_wanted = true;  // the caller's (or the tuner's) choice; used when pair_ok
  int overlap = 1;
  int cur = 0;
  RkTable rk{};
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double graph_dt = 0.0;
  long long graph_launches = 0;
  long long launches = 0;

  void free_graphs() {
    for (auto& g : graph)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  }
  ~fdmap_ensemble() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    free_graphs();
    for (fdmap_gpu* h : inst) fdmap_gpu_destroy(h);
    cudaFree(d_doms);
    cudaFree(d_tmaps);
    cudaFree(d_unit_begin);
    cudaFree(d_closure_begin);
    cudaFree(d_edge_begin);
    cudaFree(d_pmaps);
    cudaFree(d_pair_begin);
    cudaFree(d_band_begin);
    cudaFree(d_time);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// CTA prefix over instances for a boundary kernel of `tpb` threads per CTA
int cta_prefix(const std::vector<long long>& threads, int tpb, std::vector<int>& begin) {
  begin.assign(threads.size() + 1, 0);
  long long c = 0;
  for (size_t k = 0; k < threads.size(); ++k) {
    begin[k] = (int)c;
    c += (threads[k] + tpb - 1) / tpb;
  }
  begin[threads.size()] = (int)c;
  return (int)c;
}

int apply_shapes(fdmap_ensemble* e, int closure_tpb, int edge_tpb, int overlap) {
  if (closure_tpb != 64 && closure_tpb != 128 && closure_tpb != 256)
    return set_err(FDMAP_ERR_INVALID_ARG, "closure block size must be 64, 128 or 256");
  if (edge_tpb != 32 && edge_tpb != 64 && edge_tpb != 128)
    return set_err(FDMAP_ERR_INVALID_ARG, "interface block size must be 32, 64 or 128");
  std::vector<int> cb, eb;
  e->plan.closure_ctas = cta_prefix(e->closure_threads, closure_tpb, cb);
  e->plan.edge_ctas = cta_prefix(e->edge_threads, edge_tpb, eb);
  e->plan.closure_tpb = closure_tpb;
  e->plan.edge_tpb = edge_tpb;
  CUDA_TRY(cudaMemcpy(e->d_closure_begin, cb.data(), cb.size() * sizeof(int), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(e->d_edge_begin, eb.data(), eb.size() * sizeof(int), cudaMemcpyHostToDevice));
  e->overlap = overlap != 0;
  e->free_graphs();
  return FDMAP_OK;
}

int ens_stage(fdmap_ensemble* e, const StageArgs& a) {
  const BatchPlan& p = e->plan;
  int rc;
  if (e->overlap) {
    CUDA_TRY(cudaEventRecord(e->ev_fork, e->stream));
    CUDA_TRY(cudaStreamWaitEvent(e->side, e->ev_fork, 0));
    if ((rc = batch_march(e->proto, a, p, e->stream))) return rc;
    if ((rc = batch_edges(e->proto, a, p, e->side))) return rc;
    if ((rc = batch_closure(e->proto, a, p, e->side))) return rc;
    CUDA_TRY(cudaEventRecord(e->ev_join, e->side));
    CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_join, 0));
  } else {
    if ((rc = batch_edges(e->proto, a, p, e->stream))) return rc;
    if ((rc = batch_closure(e->proto, a, p, e->stream))) return rc;
    if ((rc = batch_march(e->proto, a, p, e->stream))) return rc;
  }
  e->launches += (p.edge_ctas ? 1 : 0) + (p.closure_ctas ? 1 : 0) + 1;
  return FDMAP_OK;
}

// Two stages a0, a1 of every instance as one interior pass (the single
// domain's launch_pair over the batch): the pass beside the first stage's
// interface solves and closure strips and the second stage's interface
// solves, then the bands.
int ens_pair(fdmap_ensemble* e, const StageArgs& a0, const StageArgs& a1, int dfr, int dfw) {
  const BatchPlan& p = e->plan;
  StageArgs c0 = a0;
  c0.out = 2;
  c0.dfr = dfr;
  c0.dfw = dfw;
  StageArgs e1 = a1;
  e1.in = 2;
  e1.dfr = dfw;
  e1.dfw = dfw;
  int rc;
  cudaStream_t bs = e->overlap ? e->side : e->stream;
  if (e->overlap) {
    CUDA_TRY(cudaEventRecord(e->ev_fork, e->stream));
    CUDA_TRY(cudaStreamWaitEvent(e->side, e->ev_fork, 0));
  }
  if ((rc = pair_batch(e->proto, a0, a1, dfr, dfw, e->pplan, e->stream))) return rc;
  if ((rc = batch_edges(e->proto, c0, p, bs))) return rc;
  if ((rc = batch_closure(e->proto, c0, p, bs))) return rc;
  if ((rc = batch_edges(e->proto, e1, p, bs))) return rc;
  if (e->overlap) {
    CUDA_TRY(cudaEventRecord(e->ev_join, e->side));
    CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_join, 0));
  }
  if ((rc = band_batch(e->proto, e1, e->pplan, e->stream))) return rc;
  e->launches += 2 * (p.edge_ctas ? 1 : 0) + (p.closure_ctas ? 1 : 0) + 1 + (e->pplan.band_ctas ? 1 : 0);
  return FDMAP_OK;
}

// F buffer swaps of one (non-final) step: one per stage, or one per pass
int ens_swaps(const fdmap_ensemble* e) {
  return e->pairs ? e->rk.nstage / 2 + (e->rk.nstage & 1) : e->rk.nstage;
}

// all stages of one step of every instance (final step: stage 1 only); with
// two-stage passes, stages (1,2), (3,4), ... as pairs and an odd last stage
// alone, the rate buffers alternating as in the single domain's issue_step
int ens_issue_step(fdmap_ensemble* e, int cur, double t0, double dt, bool final_step, const TimeState* ts) {
  const int npairs = (e->pairs && !final_step) ? e->rk.nstage / 2 : 0;
  auto args = [&](int s, int in) {
    StageArgs a{};
    a.A = e->rk.A[s];
    a.Bdt = e->rk.B[s] * dt;
    a.t = t0 + e->rk.C[s] * dt;
    a.C = e->rk.C[s];
    a.ts = ts;
    a.in = in;
    a.out = 1 - in;
    a.scale = 1;
    a.update = final_step ? 0 : 1;
    return a;
  };
  for (int s = 0; s < e->rk.nstage; ++s) {
    int rc;
    const StageArgs a = args(s, cur);
    if (s < 2 * npairs) {
      const int p = s / 2;
      const int dfw = ((npairs - 1 - p) & 1) ? 1 : 0;
      const int dfr = p == 0 ? 0 : 1 - dfw;
      if ((rc = ens_pair(e, a, args(s + 1, cur), dfr, dfw))) return rc;
      ++s;
    } else if ((rc = ens_stage(e, a))) {
      return rc;
    }
    if (final_step) return FDMAP_OK;
    cur = 1 - cur;
  }
  return FDMAP_OK;
}

int ens_build_graphs(fdmap_ensemble* e, double dt) {
  e->free_graphs();
  long long before = e->launches;
  int rc = FDMAP_OK;
  for (int c = 0; c < 2 && rc == FDMAP_OK; ++c) {
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return set_err(FDMAP_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
    long long l0 = e->launches;
    rc = ens_issue_step(e, c, 0.0, dt, false, e->d_time);
    if (rc == FDMAP_OK) advance_step<<<1, 1, 0, e->stream>>>(e->d_time);
    e->graph_launches = e->launches - l0 + 1;
    ce = cudaStreamEndCapture(e->stream, &g);
    if (rc == FDMAP_OK && ce != cudaSuccess) rc = set_err(FDMAP_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ce));
    if (rc == FDMAP_OK) {
      ce = cudaGraphInstantiate(&e->graph[c], g, cudaGraphInstantiateFlagUseNodePriority);
      if (ce != cudaSuccess) rc = set_err(FDMAP_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ce));
    }
    if (g) cudaGraphDestroy(g);
  }
  e->launches = before;
  if (rc == FDMAP_OK) e->graph_dt = dt;
  return rc;
}

// per-instance device descriptors and tensor maps and the prefix of march
// units over instances, for the instances' current march tile shape
int ens_fill_plan(fdmap_ensemble* e) {
  const int ninst = e->ninst;
  std::vector<DevDomain> doms(ninst);
  std::vector<TmapSet> maps(ninst);
  std::vector<long long> ub(ninst + 1, 0);
  long long units = 0;
  int grid = 0;
  for (int k = 0; k < ninst; ++k) {
    fdmap_gpu* h = e->inst[k];
    if (h->march_shape != e->proto->march_shape)
      return set_err(FDMAP_ERR_INVALID_ARG, "ensemble instances must share the march tile shape");
    doms[k] = h->hdom;
    maps[k] = *h->tmaps;
    ub[k] = units;
    units += h->march_units;
    grid = std::max(grid, h->march_grid);
  }
  ub[ninst] = units;
  CUDA_TRY(cudaMemcpy(e->d_doms, doms.data(), sizeof(DevDomain) * ninst, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(e->d_tmaps, maps.data(), sizeof(TmapSet) * ninst, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(e->d_unit_begin, ub.data(), sizeof(long long) * (ninst + 1), cudaMemcpyHostToDevice));
  e->plan.units = units;
  // CTAs per SM as the shape allows (the ring fills shared memory), never more CTAs than units
  e->plan.march_grid = (int)std::min<long long>(grid, units);
  // two-stage passes when every instance can take them
  e->pair_ok = true;
  for (fdmap_gpu* h : e->inst) e->pair_ok = e->pair_ok && h->pair_ok;
  if (e->pair_ok) {
    std::vector<TmapPair> pm(ninst);
    std::vector<long long> pb(ninst + 1, 0);
    std::vector<int> bb(ninst + 1, 0);
    long long pu = 0;
    int bc = 0, pgrid = 0;
    for (int k = 0; k < ninst; ++k) {
      fdmap_gpu* h = e->inst[k];
      pm[k] = *h->tmaps_pair;
      pb[k] = pu;
      pu += h->pair_units;
      bb[k] = bc;
      bc += (int)((h->band_threads + 127) / 128);
      pgrid = std::max(pgrid, h->pair_grid);
    }
    pb[ninst] = pu;
    bb[ninst] = bc;
    if (!e->d_pmaps) {
      CUDA_TRY(cudaMalloc(&e->d_pmaps, sizeof(TmapPair) * ninst));
      CUDA_TRY(cudaMalloc(&e->d_pair_begin, sizeof(long long) * (ninst + 1)));
      CUDA_TRY(cudaMalloc(&e->d_band_begin, sizeof(int) * (ninst + 1)));
    }
    CUDA_TRY(cudaMemcpy(e->d_pmaps, pm.data(), sizeof(TmapPair) * ninst, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(e->d_pair_begin, pb.data(), sizeof(long long) * (ninst + 1), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(e->d_band_begin, bb.data(), sizeof(int) * (ninst + 1), cudaMemcpyHostToDevice));
    e->pplan = PairBatch{e->d_doms, e->d_pmaps, e->d_pair_begin, e->d_band_begin, ninst, pu,
                         (int)std::min<long long>(pgrid, pu), bc};
  }
  e->pairs = e->pair_ok && e->pairs_wanted;
  e->free_graphs();
  return FDMAP_OK;
}

// every instance to march tile `tile`, then the plan (FDMAP_ERR_UNSUPPORTED,
// with the previous tile restored, if some instance cannot take it)
int ens_set_tile(fdmap_ensemble* e, int tile) {
  const int keep = e->proto->march_shape;
  int rc = FDMAP_OK;
  for (fdmap_gpu* h : e->inst)
    if ((rc = march_set_shape(h, tile))) break;
  if (rc) {
    const std::string msg = g_err;
    for (fdmap_gpu* h : e->inst) march_set_shape(h, keep);
    ens_fill_plan(e);
    g_err = msg;
    return rc;
  }
  return ens_fill_plan(e);
}

int ens_check_cur(fdmap_ensemble* e) {
  for (fdmap_gpu* h : e->inst)
    if (h->cur != e->cur) return set_err(FDMAP_ERR_INVALID_ARG, "an instance was stepped outside its ensemble");
  return FDMAP_OK;
}

void ens_sync_cur(fdmap_ensemble* e) {
  for (fdmap_gpu* h : e->inst) h->cur = e->cur;
}

}  // namespace

extern "C" {

int fdmap_gpu_ensemble_create(const fdmap_desc* const* descs, int ninst, int device, int init_edges,
                              fdmap_ensemble** out) {
  if (!out) return set_err(FDMAP_ERR_INVALID_ARG, "null ensemble pointer");
  *out = nullptr;
  if (!descs || ninst < 1) return set_err(FDMAP_ERR_INVALID_ARG, "an ensemble needs at least one instance");
  fdmap_ensemble* e = new (std::nothrow) fdmap_ensemble();
  if (!e) return set_err(FDMAP_ERR_NOMEM, "out of host memory");
  e->device = device;
  e->ninst = ninst;
  auto fail = [&](int rc) {
    std::string keep = g_err;
    delete e;
    g_err = keep;
    return rc;
  };
  int rc;
  for (int k = 0; k < ninst; ++k) {
    fdmap_gpu* h = nullptr;
    if ((rc = fdmap_gpu_create(descs[k], device, init_edges, &h))) return fail(rc);
    e->inst.push_back(h);
  }
  fdmap_gpu* p = e->inst[0];
  e->proto = p;
  for (fdmap_gpu* h : e->inst) {
    if (h->mode != p->mode || h->pI != p->pI || h->het != p->het || h->rk.nstage != p->rk.nstage)
      return fail(set_err(FDMAP_ERR_INVALID_ARG, "ensemble instances must share mode, FD method, RK order and material kind"));
    for (int s = 0; s < h->rk.nstage; ++s)
      if (h->rk.A[s] != p->rk.A[s] || h->rk.B[s] != p->rk.B[s] || h->rk.C[s] != p->rk.C[s])
        return fail(set_err(FDMAP_ERR_INVALID_ARG, "ensemble instances must share the RK table"));
    if (h->d_energy)
      return fail(set_err(FDMAP_ERR_UNSUPPORTED, "ensembles do not track the energy balance"));
    if (!h->use_march)
      return fail(set_err(FDMAP_ERR_UNSUPPORTED, "ensembles need the marching interior kernel (homogeneous mode II or any mode III)"));
    if (h->cur != 0) return fail(set_err(FDMAP_ERR_INVALID_ARG, "instance buffer state"));
  }
  e->rk = p->rk;
  if ((rc = [&]() -> int {
        CUDA_TRY(cudaSetDevice(device));
        int lo = 0, hi = 0;
        CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        CUDA_TRY(cudaStreamCreateWithPriority(&e->stream, cudaStreamNonBlocking, hi));
        CUDA_TRY(cudaStreamCreateWithPriority(&e->side, cudaStreamNonBlocking, lo));
        CUDA_TRY(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
        for (int k = 0; k < ninst; ++k) {
          e->closure_threads.push_back(e->inst[k]->closure_threads);
          e->edge_threads.push_back(e->inst[k]->edge_threads);
        }
        CUDA_TRY(cudaMalloc(&e->d_doms, sizeof(DevDomain) * ninst));
        CUDA_TRY(cudaMalloc(&e->d_tmaps, sizeof(TmapSet) * ninst));
        CUDA_TRY(cudaMalloc(&e->d_unit_begin, sizeof(long long) * (ninst + 1)));
        CUDA_TRY(cudaMalloc(&e->d_closure_begin, sizeof(int) * (ninst + 1)));
        CUDA_TRY(cudaMalloc(&e->d_edge_begin, sizeof(int) * (ninst + 1)));
        CUDA_TRY(cudaMalloc(&e->d_time, sizeof(TimeState)));
        CUDA_TRY(cudaMemset(e->d_time, 0, sizeof(TimeState)));
        e->plan.doms = e->d_doms;
        e->plan.tmaps = e->d_tmaps;
        e->plan.unit_begin = e->d_unit_begin;
        e->plan.closure_cta_begin = e->d_closure_begin;
        e->plan.edge_cta_begin = e->d_edge_begin;
        e->plan.ninst = ninst;
        // instances read and write through the ensemble stream
        for (fdmap_gpu* h : e->inst) {
          CUDA_TRY(cudaStreamSynchronize(h->stream));
          h->stream = e->stream;
        }
        return ens_fill_plan(e);
      }()))
    return fail(rc);
  if ((rc = apply_shapes(e, 128, 64, 1))) return fail(rc);
  *out = e;
  return FDMAP_OK;
}

int fdmap_gpu_ensemble_instance(fdmap_ensemble* e, int k, fdmap_gpu** h) {
  if (!e || !h) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  if (k < 0 || k >= e->ninst) return set_err(FDMAP_ERR_INVALID_ARG, "instance index out of range");
  *h = e->inst[k];
  return FDMAP_OK;
}

int fdmap_gpu_ensemble_size(fdmap_ensemble* e) { return e ? e->ninst : -1; }

int fdmap_gpu_ensemble_time_step(fdmap_ensemble* e, double t0, double dt, int final_step) {
  if (!e) return set_err(FDMAP_ERR_INVALID_ARG, "null ensemble");
  CUDA_TRY(cudaSetDevice(e->device));
  int rc = ens_check_cur(e);
  if (rc) return rc;
  if ((rc = ens_issue_step(e, e->cur, t0, dt, final_step != 0, nullptr))) return rc;
  if (!final_step && (ens_swaps(e) & 1)) e->cur = 1 - e->cur;
  ens_sync_cur(e);
  return FDMAP_OK;
}

int fdmap_gpu_ensemble_run(fdmap_ensemble* e, double t_start, double dt, int n_first, int n_last, int nt) {
  if (!e) return set_err(FDMAP_ERR_INVALID_ARG, "null ensemble");
  CUDA_TRY(cudaSetDevice(e->device));
  int rc = ens_check_cur(e);
  if (rc) return rc;
  e->launches = 0;
  const int n_graph_last = std::min(n_last, nt - 1);  // the final step (n == nt) is issued directly
  if (n_graph_last >= n_first) {
    if (e->graph_dt != dt || !e->graph[0]) {
      if ((rc = ens_build_graphs(e, dt))) return rc;
    }
    set_step_clock<<<1, 1, 0, e->stream>>>(e->d_time, t_start, dt, (long long)n_first);
    e->launches++;
    CUDA_TRY(cudaGetLastError());
    for (int n = n_first; n <= n_graph_last; ++n) {
      CUDA_TRY(cudaGraphLaunch(e->graph[e->cur], e->stream));
      e->launches += e->graph_launches;
      if (ens_swaps(e) & 1) e->cur = 1 - e->cur;
    }
    n_first = n_graph_last + 1;
  }
  ens_sync_cur(e);
  for (int n = n_first; n <= n_last; ++n)
    if ((rc = fdmap_gpu_ensemble_time_step(e, t_start + (double)(n - 1) * dt, dt, n == nt))) return rc;
  return FDMAP_OK;
}

int fdmap_gpu_ensemble_synchronize(fdmap_ensemble* e) {
  if (!e) return set_err(FDMAP_ERR_INVALID_ARG, "null ensemble");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return FDMAP_OK;
}

int fdmap_gpu_ensemble_set_shape(fdmap_ensemble* e, const int* shape) {
  if (!e || !shape) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return apply_shapes(e, shape[0], shape[1], shape[2]);
}

int fdmap_gpu_ensemble_get_shape(fdmap_ensemble* e, int* shape) {
  if (!e || !shape) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  shape[0] = e->plan.closure_tpb;
  shape[1] = e->plan.edge_tpb;
  shape[2] = e->overlap;
  return FDMAP_OK;
}

// Autotuner: times `steps` graph-replayed steps (best of two repetitions),
// first for every march tile shape (strip width x rows per group) the
// instances can take, then on the fastest tile for every launch shape of the
// boundary kernels (closure block size x interface block size x
// boundary/interior overlap); keeps the fastest and leaves it applied.  Every
// instance's device state is saved before and restored after, so tuning does
// not advance the ensemble.
int fdmap_gpu_ensemble_tune(fdmap_ensemble* e, double dt, int steps, int* best_shape, double* best_ms) {
  if (!e) return set_err(FDMAP_ERR_INVALID_ARG, "null ensemble");
  if (steps < 1) return set_err(FDMAP_ERR_INVALID_ARG, "steps must be positive");
  CUDA_TRY(cudaSetDevice(e->device));
  int rc = ens_check_cur(e);
  if (rc) return rc;
  // snapshot of every instance's whole device state
  std::vector<std::vector<void*>> saved(e->inst.size());
  for (size_t k = 0; k < e->inst.size() && rc == FDMAP_OK; ++k) rc = state_snapshot(e->inst[k], saved[k], e->stream);
  auto cleanup = [&]() {
    for (auto& v : saved) {
      for (void* p : v) cudaFree(p);
      v.clear();
    }
  };
  if (rc) { cleanup(); return rc; }
  const int cur0 = e->cur;
  const int ctpb[3] = {64, 128, 256}, etpb[3] = {32, 64, 128};
  int best[4] = {e->plan.closure_tpb, e->plan.edge_tpb, e->overlap, e->proto->march_shape};
  float best_t = -1.f;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  // warm-up step (also builds the graphs), then two timed repetitions; the faster counts
  auto time_shape = [&](float& ms) -> int {
    int r = fdmap_gpu_ensemble_run(e, 0.0, dt, 1, 1, 1 << 30);
    if (r) return r;
    ms = -1.f;
    for (int rep = 0; rep < 2; ++rep) {
      cudaEventRecord(t0, e->stream);
      if ((r = fdmap_gpu_ensemble_run(e, 0.0, dt, 2, 1 + steps, 1 << 30))) return r;
      cudaEventRecord(t1, e->stream);
      if (cudaEventSynchronize(t1) != cudaSuccess) return set_err(FDMAP_ERR_CUDA, "tuning run failed");
      float m = 0.f;
      cudaEventElapsedTime(&m, t0, t1);
      if (ms < 0.f || m < ms) ms = m;
    }
    return FDMAP_OK;
  };
  // 1. the march tile shape, with two-stage passes on and off where every
  // instance can take them, with the boundary launch shapes as they are
  const bool pairs0 = e->pairs;
  bool best_pairs = pairs0;
  for (int k = 0; k < (e->pair_ok ? 2 : 1) * MARCH_SHAPES && rc == FDMAP_OK; ++k) {
    const int tile = k % MARCH_SHAPES;
    rc = ens_set_tile(e, tile);
    if (rc == FDMAP_ERR_UNSUPPORTED) { rc = FDMAP_OK; continue; }
    e->pairs = e->pair_ok ? k < MARCH_SHAPES : pairs0;  // after ens_set_tile, which resets it
    e->free_graphs();
    float ms = 0.f;
    if (rc || (rc = time_shape(ms))) break;
    if (best_t < 0.f || ms < best_t) { best_t = ms; best[3] = tile; best_pairs = e->pairs; }
  }
  // 2. closure and interface block sizes and the overlap, on the best tile
  if (rc == FDMAP_OK) rc = ens_set_tile(e, best[3]);
  if (rc == FDMAP_OK) {
    e->pairs = best_pairs;
    e->free_graphs();
  }
  for (int ov = 0; ov < 2 && rc == FDMAP_OK; ++ov)
    for (int ci = 0; ci < 3 && rc == FDMAP_OK; ++ci)
      for (int ei = 0; ei < 3 && rc == FDMAP_OK; ++ei) {
        if ((rc = apply_shapes(e, ctpb[ci], etpb[ei], ov))) break;
        float ms = 0.f;
        if ((rc = time_shape(ms))) break;
        if (ms < best_t) {
          best_t = ms;
          best[0] = ctpb[ci]; best[1] = etpb[ei]; best[2] = ov;
        }
      }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  // restore the state and the buffer parity
  for (size_t k = 0; k < e->inst.size(); ++k) {
    const int rr = state_restore(e->inst[k], saved[k], e->stream);
    if (rr && !rc) rc = rr;
  }
  cleanup();
  e->cur = cur0;
  ens_sync_cur(e);
  if (rc) {
    e->pairs = pairs0;
    e->free_graphs();
    return rc;
  }
  e->pairs_wanted = best_pairs;
  if ((rc = ens_set_tile(e, best[3]))) return rc;
  if ((rc = apply_shapes(e, best[0], best[1], best[2]))) return rc;
  if (best_shape) { best_shape[0] = best[0]; best_shape[1] = best[1]; best_shape[2] = best[2]; }
  if (best_ms) *best_ms = best_t / steps;
  return FDMAP_OK;
}

int fdmap_gpu_ensemble_set_pairs(fdmap_ensemble* e, int enable) {
  if (!e) return set_err(FDMAP_ERR_INVALID_ARG, "null ensemble");
  if (enable && !e->pair_ok) return set_err(FDMAP_ERR_UNSUPPORTED, "some instance cannot run two-stage passes");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  e->pairs_wanted = enable != 0;
  if (e->pairs != (enable != 0)) {
    e->pairs = enable != 0;
    e->free_graphs();
  }
  return FDMAP_OK;
}

int fdmap_gpu_ensemble_get_pairs(fdmap_ensemble* e) {
  if (!e) return set_err(FDMAP_ERR_INVALID_ARG, "null ensemble");
  return e->pairs ? 1 : 0;
}

int fdmap_gpu_ensemble_set_tile(fdmap_ensemble* e, int tile) {
  if (!e || tile < 0 || tile >= MARCH_SHAPES) return set_err(FDMAP_ERR_INVALID_ARG, "tile must be 0..3");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return ens_set_tile(e, tile);
}

int fdmap_gpu_ensemble_get_tile(fdmap_ensemble* e, int* tile) {
  if (!e || !tile) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  *tile = e->proto->march_shape;
  return FDMAP_OK;
}

long long fdmap_gpu_ensemble_launch_count(fdmap_ensemble* e) { return e ? e->launches : -1; }

void fdmap_gpu_ensemble_destroy(fdmap_ensemble* e) { delete e; }

}  // extern "C"
