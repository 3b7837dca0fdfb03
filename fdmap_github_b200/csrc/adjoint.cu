// Forward/backward pair for gradients of a receiver-seismogram misfit with
// respect to the density and shear-modulus fields of a heterogeneous mode III
// domain (SBP-SAT wave solve, LS-RK time stepping) and, with frictional
// interfaces, the shear prestress of every fault node.  The reference has no
// adjoint; the forward pass is the engine's own time step (time_step_LS,
// time_step.f90:71-167), so the misfit is that of the production path.
//
// Every block's stage runs as interior tiles (adj_stage_tma) beside its band
// (adj_band_kernel).  Several blocks or interfaces take the general path:
// after the blocks, the fault nodes run through adj_fault_kernel
// (adjoint_fault.cuh); the state variable of each fault node is stored beside
// the fields at every stage and the fault registers in every checkpoint.
//
//   forward : steps 1..nt-1 as replayed graphs; vz sampled at the receivers at
//             every step start (n = 1..nt, the reference's stage-1 output
//             point, time_step.f90:129); the fields are checkpointed every
//             `checkpoint_every` steps.
//   backward: segments in reverse; each is recomputed from its checkpoint with
//             every stage input stored, then reversed stage by stage with the
//             discrete adjoint (adjoint_kernel.cuh), injecting the receiver
//             residuals dJ/dU^n = vz - d at every step start.
//   resident segments: with a store budget, the forward run with data keeps
//             the stage inputs of its last R segments in device memory (the
//             whole 2000-step trajectory of an 801 x 801 block is 157 GB),
//             and the backward reverses those without recomputing them; the
//             others are recomputed into one more segment store after them.
//             The stored inputs are the recomputed ones bit for bit.
// J = 1/2 sum_n sum_r (vz_r(U^n) - d_r^n)^2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <new>
#include <string>
#include <vector>

#include "adjoint_fault.cuh"
#include "adjoint_kernel.cuh"
#include "engine.h"
#include "fdmap_gpu.h"

using namespace fdmap;

struct fdmap_adjoint {
  fdmap_gpu* h = nullptr;
  int K = 45;                        // steps per checkpoint segment
  int nrec = 0;
  int N = 0;                         // samples of the last forward (nt)
  double t_start = 0.0, dt = 0.0;
  std::vector<long long> rec_host;   // block-local linear node index of each receiver
  long long* rec = nullptr;
  // distinct receiver nodes and the receivers on each (CSR), for the residual injection
  int nnode = 0;
  long long* node = nullptr;
  int* rstart = nullptr;
  int* rlist = nullptr;
  std::vector<long long> nband;       // per block: nodes within nbnd of a side
  cudaStream_t side = nullptr;        // band kernel beside the interior adjoint kernel (high priority)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t copy = nullptr;        // stage-input copies beside the recomputed stage
  cudaEvent_t ev_cfork = nullptr, ev_cjoin = nullptr;
  std::vector<AdjMaps> maps;          // per block: TMA descriptors of the interior adjoint tiles
  double* init_F = nullptr;          // initial fields (3 planes)
  double* init_DF = nullptr;
  double* ckpt = nullptr;            // checkpoints, 3 planes each
  int nckpt_alloc = 0;
  double* store = nullptr;           // stage inputs: store_segs segments of K*nstage slots
  int store_segs = 1;                // segment stores allocated (the resident ones, then the recomputed one)
  long long store_budget = 0;        // bytes for resident segments: 0 none, < 0 all free device memory
  int plan_nseg = -1;                // segments and budget the present store was sized for
  long long plan_budget = 0;
  int plan_R = 0;                    // resident segments of that plan
  int resident = 0;                  // last segments of the last forward with data held in the store
  double* ub[2] = {nullptr, nullptr};
  double* qp[2] = {nullptr, nullptr};
  double* grho = nullptr;
  double* gG = nullptr;
  std::vector<double*> geo;          // edge geometry factors, 4 sides per block
  // general path (several blocks or interfaces)
  bool general = false;
  int nb = 1;
  long long boff[MAX_BLOCKS] = {};   // block offsets in the concatenated 3-plane layout
  long long goff[MAX_BLOCKS] = {};   // and in the concatenated gradient planes
  long long total = 0;               // 3-plane layout doubles of all blocks
  long long gtotal = 0;              // gradient-plane doubles of all blocks
  int nfault = 0;                    // fault nodes of all interfaces
  std::vector<AdjIfaceInfo> info_host;
  AdjIfaceInfo* info = nullptr;
  std::vector<long long> st_off;     // fault-register offset of each frictional interface in a checkpoint
  long long st_total = 0;
  double* init_st = nullptr;
  double* psib[2] = {nullptr, nullptr};   // Psibar, qbar'_Psi per fault node (ubar parity)
  double* qpsib[2] = {nullptr, nullptr};
  double* gS0 = nullptr;
  const double** recp[2] = {nullptr, nullptr};  // per receiver: vz in F[parity]
  std::vector<std::pair<int, long long>> rec_gen;  // (block, local index) per receiver
  double* traces = nullptr;          // N*nrec
  double* resid = nullptr;           // N*nrec
  int trace_alloc = 0;
  AdjClock* clock = nullptr;
  bool have_resid = false;
  // graphs: forward step, forward step that also stores its stage inputs,
  // recompute step (each by F parity), adjoint step (by ubar parity)
  cudaGraphExec_t g_fwd[2] = {nullptr, nullptr}, g_fst[2] = {nullptr, nullptr}, g_rec[2] = {nullptr, nullptr},
                  g_adj[2] = {nullptr, nullptr};
  double graph_dt = -1.0, graph_t0 = 0.0;
  std::vector<void*> mem;

  long long stride() const { return 3 * h->hdom.blk[0].plane; }
  // a stage slot: every block's 3 planes, then Psi and the converged slip rate
  // of the fault nodes, each padded to an even count (the 4-D store map needs
  // 16-byte slot strides)
  long long fault_pad() const { return (nfault + 1) & ~1; }
  long long slot_stride() const { return general ? total + 2 * fault_pad() : stride(); }
  long long ckpt_stride() const { return general ? total + st_total : stride(); }
  size_t segment_bytes() const { return (size_t)K * h->rk.nstage * slot_stride() * sizeof(double); }
  void free_graphs() {
    for (auto* set : {g_fwd, g_fst, g_rec, g_adj})
      for (int q = 0; q < 2; ++q)
        if (set[q]) { cudaGraphExecDestroy(set[q]); set[q] = nullptr; }
    graph_dt = -1.0;
  }
  ~fdmap_adjoint() {
    if (h) {
      cudaSetDevice(h->device);
      cudaStreamSynchronize(h->stream);
    }
    free_graphs();
    for (void* p : mem) cudaFree(p);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_cfork) cudaEventDestroy(ev_cfork);
    if (ev_cjoin) cudaEventDestroy(ev_cjoin);
    if (side) cudaStreamDestroy(side);
    if (copy) cudaStreamDestroy(copy);
    if (h) fdmap_gpu_destroy(h);
  }
  template <typename T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16)) != cudaSuccess)
      return set_err(FDMAP_ERR_NOMEM, "adjoint: out of device memory");
    mem.push_back(q);
    *p = (T*)q;
    return FDMAP_OK;
  }
  void release(void* p) {
    if (!p) return;
    auto it = std::find(mem.begin(), mem.end(), p);
    if (it != mem.end()) mem.erase(it);
    cudaFree(p);
  }
};

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// 3-D FP64 map over `nplanes` planes of the block layout, box {bx, by, bz};
// halo boxes start off the 256-byte lines, so no L2 promotion (sector fetches)
int adj_encode(EncodeTiledFn enc, CUtensorMap* map, const double* base, const BlockGeom& g, long long nplanes, int bx,
               int by, int bz) {
  cuuint64_t dims[3] = {(cuuint64_t)g.pitch, (cuuint64_t)g.ny, (cuuint64_t)nplanes};
  cuuint64_t strides[2] = {(cuuint64_t)g.pitch * 8, (cuuint64_t)g.plane * 8};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_err(FDMAP_ERR_CUDA, "adjoint tensor map (" + std::to_string((int)r) + ")");
  return FDMAP_OK;
}

// 4-D FP64 map over the stage store of one block: (x, y, plane 0..2, slot),
// slots `slot_stride` doubles apart; box {bx, by, 3, 1}
int adj_encode_store(EncodeTiledFn enc, CUtensorMap* map, const double* base, const BlockGeom& g, long long slot_stride,
                     long long nslots, int bx, int by) {
  cuuint64_t dims[4] = {(cuuint64_t)g.pitch, (cuuint64_t)g.ny, 3, (cuuint64_t)nslots};
  cuuint64_t strides[3] = {(cuuint64_t)g.pitch * 8, (cuuint64_t)g.plane * 8, (cuuint64_t)slot_stride * 8};
  cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 3, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_err(FDMAP_ERR_CUDA, "adjoint store tensor map (" + std::to_string((int)r) + ")");
  return FDMAP_OK;
}

template <int PI_>
int adj_maps_for(fdmap_adjoint* a) {
  using T = AdjTile<PI_>;
  fdmap_gpu* h = a->h;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult qr;
  CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr));
  if (!fn || qr != cudaDriverEntryPointSuccess) return set_err(FDMAP_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  EncodeTiledFn enc = (EncodeTiledFn)fn;
  int rc;
  a->maps.assign(a->nb, AdjMaps{});
  for (int b = 0; b < a->nb; ++b) {
    const BlockGeom& g = h->geom[b];
    AdjMaps& m = a->maps[b];
    for (int q = 0; q < 2; ++q) {
      if ((rc = adj_encode(enc, &m.ub[q], a->ub[q] + a->boff[b], g, 3, T::WX, T::WY, 3))) return rc;
      if ((rc = adj_encode(enc, &m.qp[q], a->qp[q] + a->boff[b], g, 3, T::WX, T::WY, 3))) return rc;
    }
    if ((rc = adj_encode_store(enc, &m.st, a->store + a->boff[b], g, a->slot_stride(),
                               (long long)a->store_segs * a->K * h->rk.nstage, T::WX, T::WY)))
      return rc;
    if ((rc = adj_encode(enc, &m.met, h->met_base[b], g, 5, T::WX, T::WY, 5))) return rc;
    if ((rc = adj_encode(enc, &m.het, h->het_base[b], g, 2, T::WX, T::WY, 2))) return rc;
  }
  CUDA_TRY(cudaFuncSetAttribute(adj_stage_tma<PI_>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM + 128));
  return FDMAP_OK;
}

int adj_maps(fdmap_adjoint* a) {
  const int pI = a->h->pI;
  return pI == 1 ? adj_maps_for<1>(a) : (pI == 2 ? adj_maps_for<2>(a) : adj_maps_for<3>(a));
}

// one block's adjoint stage: interior tiles on the main stream, the band on
// the side stream (disjoint nodes, same inputs); the caller forks and joins
int adj_block_launch(fdmap_adjoint* a, const AdjStage& p, int q) {
  fdmap_gpu* h = a->h;
  const int b = p.blk;
  const DevBlock& B = h->hdom.blk[b];
  dim3 blk(ATX * ATY), grid((B.nx + ATX - 1) / ATX, (B.ny + ATY - 1) / ATY);
  const long long nb = a->nband[b];
  const int bgrid = (int)((nb + BAND_NODES - 1) / BAND_NODES);
  const AdjMaps& m = a->maps[b];
  // the latency-bound band kernel goes first, at high priority, so its few CTAs
  // are placed before the interior tiles fill the SMs
  if (h->pI == 1) {
    adj_band_kernel<1><<<bgrid, 2 * BAND_NODES, 0, a->side>>>(h->hdom, p, nb);
    adj_stage_tma<1><<<grid, blk, AdjTile<1>::SMEM + 128, h->stream>>>(h->hdom, p, m, q);
  } else if (h->pI == 2) {
    adj_band_kernel<2><<<bgrid, 2 * BAND_NODES, 0, a->side>>>(h->hdom, p, nb);
    adj_stage_tma<2><<<grid, blk, AdjTile<2>::SMEM + 128, h->stream>>>(h->hdom, p, m, q);
  } else {
    adj_band_kernel<3><<<bgrid, 2 * BAND_NODES, 0, a->side>>>(h->hdom, p, nb);
    adj_stage_tma<3><<<grid, blk, AdjTile<3>::SMEM + 128, h->stream>>>(h->hdom, p, m, q);
  }
  CUDA_TRY(cudaGetLastError());
  return FDMAP_OK;
}

int adj_fork(fdmap_adjoint* a) {
  CUDA_TRY(cudaEventRecord(a->ev_fork, a->h->stream));
  CUDA_TRY(cudaStreamWaitEvent(a->side, a->ev_fork, 0));
  return FDMAP_OK;
}

int adj_join(fdmap_adjoint* a) {
  CUDA_TRY(cudaEventRecord(a->ev_join, a->side));
  CUDA_TRY(cudaStreamWaitEvent(a->h->stream, a->ev_join, 0));
  return FDMAP_OK;
}

// single block: interior tiles and band, joined before the next stage; q = ubar / qbar' parity
int adj_stage_launch(fdmap_adjoint* a, const AdjStage& p, int q) {
  int rc;
  if ((rc = adj_fork(a)) || (rc = adj_block_launch(a, p, q)) || (rc = adj_join(a))) return rc;
  return FDMAP_OK;
}

// forward stage sequence of one step from buffer `cur` (the engine's time_step_LS body)
int forward_step_stages(fdmap_adjoint* a, int cur, double dt, bool stash) {
  fdmap_gpu* h = a->h;
  const long long slot = a->slot_stride();
  for (int s = 0; s < h->rk.nstage; ++s) {
    if (stash) {
      // the stage only reads F[cur]; the copy of it runs beside the stage and
      // joins before the next stage overwrites that buffer
      if (s > 0) CUDA_TRY(cudaStreamWaitEvent(h->stream, a->ev_cjoin, 0));
      if (a->nfault > 0) {
        // the stage updates Psi in place: its copy goes first, on the stage's stream
        adj_stash_psi<<<(a->nfault + 127) / 128, 128, 0, h->stream>>>(
            h->hdom, a->info, (int)a->info_host.size(), a->nfault, a->store, slot, a->total, a->total + a->fault_pad(),
            &a->clock->rel, s, h->rk.nstage, 1);
        CUDA_TRY(cudaGetLastError());
      }
      CUDA_TRY(cudaEventRecord(a->ev_cfork, h->stream));
      CUDA_TRY(cudaStreamWaitEvent(a->copy, a->ev_cfork, 0));
      for (int b = 0; b < a->nb; ++b) {
        const DevBlock& B = h->hdom.blk[b];
        adj_stash<<<296, 256, 0, a->copy>>>(B.F[cur], a->store + a->boff[b], slot, &a->clock->rel, s, h->rk.nstage,
                                            3 * B.plane);
        CUDA_TRY(cudaGetLastError());
      }
      CUDA_TRY(cudaEventRecord(a->ev_cjoin, a->copy));
    }
    StageArgs st{};
    st.A = h->rk.A[s];
    st.Bdt = h->rk.B[s] * dt;
    st.C = h->rk.C[s];
    st.ts = h->d_time;
    st.in = cur;
    st.out = 1 - cur;
    st.scale = 1;
    st.update = 1;
    int rc = engine_stage(h, st);
    if (rc) return rc;
    cur = 1 - cur;
  }
  if (stash && a->nfault > 0) {
    // the slip rate the last stage converged to
    adj_stash_psi<<<(a->nfault + 127) / 128, 128, 0, h->stream>>>(
        h->hdom, a->info, (int)a->info_host.size(), a->nfault, a->store, slot, a->total, a->total + a->fault_pad(),
        &a->clock->rel, h->rk.nstage - 1, h->rk.nstage, 0);
    CUDA_TRY(cudaGetLastError());
  }
  if (stash) CUDA_TRY(cudaStreamWaitEvent(h->stream, a->ev_cjoin, 0));
  return FDMAP_OK;
}

int capture(fdmap_adjoint* a, cudaGraphExec_t* out, const std::function<int()>& body) {
  cudaStream_t s = a->h->stream;
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = body();
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc == FDMAP_OK && e != cudaSuccess) rc = set_err(FDMAP_ERR_CUDA, std::string("adjoint capture: ") + cudaGetErrorString(e));
  if (rc == FDMAP_OK) {
    e = cudaGraphInstantiate(out, g, cudaGraphInstantiateFlagUseNodePriority);
    if (e != cudaSuccess) rc = set_err(FDMAP_ERR_CUDA, std::string("adjoint instantiate: ") + cudaGetErrorString(e));
  }
  if (g) cudaGraphDestroy(g);
  return rc;
}

// one adjoint stage of the general path: every block (tiles and band), then
// the fault nodes
int gen_stage_launch(fdmap_adjoint* a, int s, double dt, int q) {
  fdmap_gpu* h = a->h;
  int rc = adj_fork(a);
  if (rc) return rc;
  for (int b = 0; b < a->nb; ++b) {
    AdjStage p{};
    p.A = h->rk.A[s];
    p.Bdt = h->rk.B[s] * dt;
    p.s = s;
    p.nstage = h->rk.nstage;
    p.ub_in = a->ub[q] + a->boff[b];
    p.qp_in = a->qp[q] + a->boff[b];
    p.ub_out = a->ub[1 - q] + a->boff[b];
    p.qp_out = a->qp[1 - q] + a->boff[b];
    p.store = a->store + a->boff[b];
    p.stride = a->slot_stride();
    p.rel = &a->clock->rel;
    p.grho = a->grho + a->goff[b];
    p.gG = a->gG + a->goff[b];
    p.blk = b;
    if ((rc = adj_block_launch(a, p, q))) return rc;
  }
  if (a->nfault == 0) return adj_join(a);
  AdjFaultArgs f{};
  f.A = h->rk.A[s];
  f.Bdt = h->rk.B[s] * dt;
  f.C = h->rk.C[s];
  f.t_start = a->t_start;
  f.dt = dt;
  f.s = s;
  f.nstage = h->rk.nstage;
  f.ub_in = a->ub[q];
  f.qp_in = a->qp[q];
  f.ub_out = a->ub[1 - q];
  f.store = a->store;
  f.slot_stride = a->slot_stride();
  f.psi_off = a->total;
  f.v_off = a->total + a->fault_pad();
  f.ck = a->clock;
  f.psib_in = a->psib[q];
  f.qpsib_in = a->qpsib[q];
  f.psib_out = a->psib[1 - q];
  f.qpsib_out = a->qpsib[1 - q];
  f.grho = a->grho;
  f.gG = a->gG;
  f.gS0 = a->gS0;
  f.info = a->info;
  f.nifc = (int)a->info_host.size();
  f.nfault = a->nfault;
  for (int b = 0; b < a->nb; ++b) {
    f.boff[b] = a->boff[b];
    f.goff[b] = a->goff[b];
  }
  // on the side stream after the band kernels: the fault nodes write only
  // edge nodes, which no interior tile touches
  const long long thr = (long long)a->nfault * FAULT_LANES;
  adj_fault_kernel<<<(int)((thr + 127) / 128), 128, 0, a->side>>>(h->hdom, f);
  CUDA_TRY(cudaGetLastError());
  return adj_join(a);
}

int build_graphs(fdmap_adjoint* a, double dt) {
  a->free_graphs();
  fdmap_gpu* h = a->h;
  const long long saved = h->launches;
  const DevBlock& B = h->hdom.blk[0];
  int rc = FDMAP_OK;
  for (int c = 0; c < 2 && rc == FDMAP_OK; ++c) {
    // forward step: the stages, then vz at the receivers of the new state;
    // the storing variant also puts every stage input into the store and
    // advances the store's step index
    for (int keep = 0; keep < 2 && rc == FDMAP_OK; ++keep)
      rc = capture(a, keep ? &a->g_fst[c] : &a->g_fwd[c], [&]() -> int {
        int r = forward_step_stages(a, c, dt, keep != 0);
        if (r) return r;
        const int last = (h->rk.nstage & 1) ? 1 - c : c;  // buffer holding the new state
        AdjClock* ck = keep ? a->clock : nullptr;
        if (a->general)
          adj_sample_advance_ptr<<<1, 128, 0, h->stream>>>(a->recp[last], a->nrec, h->d_time, a->traces,
                                                           a->trace_alloc, ck);
        else
          adj_sample_advance<<<1, 128, 0, h->stream>>>(B.F[last], a->rec, a->nrec, h->d_time, a->traces,
                                                       a->trace_alloc, ck);
        return (int)FDMAP_OK;
      });
    if (rc) break;
    // recomputed step: every stage input goes to the segment store
    rc = capture(a, &a->g_rec[c], [&]() -> int {
      int r = forward_step_stages(a, c, dt, true);
      if (r) return r;
      adj_forward_advance<<<1, 1, 0, h->stream>>>(h->d_time, a->clock);
      return (int)FDMAP_OK;
    });
    if (rc) break;
    // adjoint step: stages in reverse from ubar parity c, then the residual at this step start
    rc = capture(a, &a->g_adj[c], [&]() -> int {
      int q = c;
      for (int s = h->rk.nstage - 1; s >= 0 && a->general; --s) {
        int r = gen_stage_launch(a, s, dt, q);
        if (r) return r;
        q = 1 - q;
      }
      for (int s = h->rk.nstage - 1; s >= 0 && !a->general; --s) {
        AdjStage p{};
        p.A = h->rk.A[s];
        p.Bdt = h->rk.B[s] * dt;
        p.s = s;
        p.nstage = h->rk.nstage;
        p.ub_in = a->ub[q];
        p.qp_in = a->qp[q];
        p.ub_out = a->ub[1 - q];
        p.qp_out = a->qp[1 - q];
        p.store = a->store;
        p.stride = a->stride();
        p.rel = &a->clock->rel;
        p.grho = a->grho;
        p.gG = a->gG;
        int r = adj_stage_launch(a, p, q);
        if (r) return r;
        q = 1 - q;
      }
      adj_inject<<<1, 128, 0, h->stream>>>(a->ub[q], a->node, a->rstart, a->rlist, a->nnode, a->nrec, a->resid,
                                           a->clock, 1);
      return (int)FDMAP_OK;
    });
  }
  h->launches = saved;
  if (rc == FDMAP_OK) a->graph_dt = dt;
  return rc;
}

// global (nx, ny) plane -> device block plane and back
int to_block(fdmap_adjoint* a, double* dst, const double* src, int b = 0) {
  fdmap_gpu* h = a->h;
  return h->upload_plane(dst, src, h->geom[b]);
}

int from_block(fdmap_adjoint* a, double* dst, const double* src, int b = 0) {
  fdmap_gpu* h = a->h;
  const BlockGeom& g = h->geom[b];
  std::vector<double> tmp((size_t)g.plane);
  CUDA_TRY(cudaMemcpy(tmp.data(), src, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int j = 0; j < g.ny; ++j)
    std::memcpy(dst + (size_t)(g.mgy - 1 + j) * h->nx_g + (g.mgx - 1), tmp.data() + (size_t)j * g.pitch,
                g.nx * sizeof(double));
  return FDMAP_OK;
}

int ensure_trace_buffers(fdmap_adjoint* a, int N) {
  if (N <= a->trace_alloc) return FDMAP_OK;
  a->release(a->traces);
  a->release(a->resid);
  a->traces = a->resid = nullptr;
  int rc;
  if ((rc = a->alloc(&a->traces, (size_t)N * a->nrec))) return rc;
  if ((rc = a->alloc(&a->resid, (size_t)N * a->nrec))) return rc;
  a->trace_alloc = N;
  a->free_graphs();  // graphs hold the buffer pointers
  return FDMAP_OK;
}

// fields of every block into F[0] (and, given `st`, the fault registers)
// from a checkpoint layout: blocks at boff, fault registers after them
int restore_state(fdmap_adjoint* a, const double* src, const double* st) {
  fdmap_gpu* h = a->h;
  for (int b = 0; b < a->nb; ++b)
    CUDA_TRY(cudaMemcpyAsync(h->hdom.blk[b].F[0], src + a->boff[b], 3 * h->hdom.blk[b].plane * sizeof(double),
                             cudaMemcpyDeviceToDevice, h->stream));
  for (size_t i = 0; i < a->st_off.size(); ++i) {
    if (a->st_off[i] < 0) continue;
    const double* from = st ? st + (a->st_off[i] - a->total) : src + a->st_off[i];
    CUDA_TRY(cudaMemcpyAsync(h->hdom.ifc[i].fr.st, from, (size_t)FDMAP_FAULT_NFIELDS * h->hdom.ifc[i].n * sizeof(double),
                             cudaMemcpyDeviceToDevice, h->stream));
  }
  return FDMAP_OK;
}

int save_state(fdmap_adjoint* a, double* dst) {
  fdmap_gpu* h = a->h;
  for (int b = 0; b < a->nb; ++b)
    CUDA_TRY(cudaMemcpyAsync(dst + a->boff[b], h->hdom.blk[b].F[h->cur], 3 * h->hdom.blk[b].plane * sizeof(double),
                             cudaMemcpyDeviceToDevice, h->stream));
  for (size_t i = 0; i < a->st_off.size(); ++i) {
    if (a->st_off[i] < 0) continue;
    CUDA_TRY(cudaMemcpyAsync(dst + a->st_off[i], h->hdom.ifc[i].fr.st,
                             (size_t)FDMAP_FAULT_NFIELDS * h->hdom.ifc[i].n * sizeof(double), cudaMemcpyDeviceToDevice,
                             h->stream));
  }
  return FDMAP_OK;
}

// Size the stage store for a forward with data over `nseg` segments: R
// resident segments (the last ones) as the budget and the free device memory
// allow, less a 2 GiB margin, and one segment store more for recomputing the
// others when R < nseg.  The plan is kept while nseg and the budget stay the
// same, so repeated forward runs reuse the store, its maps and the graphs.
int ensure_store(fdmap_adjoint* a, int nseg) {
  if (a->plan_nseg == nseg && a->plan_budget == a->store_budget) return FDMAP_OK;
  const size_t seg = a->segment_bytes();
  int R = 0;
  if (a->store_budget != 0) {
    size_t freeb = 0, totalb = 0;
    CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
    const size_t margin = (size_t)2 << 30;
    const size_t have = freeb + (size_t)a->store_segs * seg;  // the present store is given back first
    size_t avail = have > margin ? have - margin : 0;
    if (a->store_budget > 0) avail = std::min(avail, (size_t)a->store_budget);
    const long long fit = (long long)(avail / seg);
    R = fit >= nseg ? nseg : (int)std::max(0LL, fit - 1);
  }
  const int segs = R < nseg ? R + 1 : R;
  if (segs != a->store_segs) {
    a->free_graphs();  // graphs and maps hold the store
    CUDA_TRY(cudaStreamSynchronize(a->h->stream));
    a->release(a->store);
    a->store = nullptr;
    a->store_segs = 0;  // no store: the next forward with data sizes it again
    a->resident = 0;
    if (a->alloc(&a->store, (size_t)segs * seg / sizeof(double)) != FDMAP_OK) {
      // fall back to checkpointing alone (and clear the failed allocation's error)
      cudaGetLastError();
      R = 0;
      int rc = a->alloc(&a->store, seg / sizeof(double));
      if (rc) {
        cudaGetLastError();
        a->plan_nseg = -1;
        return rc;
      }
      a->store_segs = 1;
    } else {
      a->store_segs = segs;
    }
    int rc = adj_maps(a);
    if (rc) return rc;
  }
  a->plan_nseg = nseg;
  a->plan_budget = a->store_budget;
  a->plan_R = R;
  return FDMAP_OK;
}

int ensure_checkpoints(fdmap_adjoint* a, int nck) {
  if (nck <= a->nckpt_alloc) return FDMAP_OK;
  a->release(a->ckpt);
  a->ckpt = nullptr;
  int rc = a->alloc(&a->ckpt, (size_t)nck * a->ckpt_stride());
  if (rc) return rc;
  a->nckpt_alloc = nck;
  return FDMAP_OK;
}

}  // namespace

extern "C" {

int fdmap_gpu_adjoint_create(const fdmap_desc* d, int device, int nrec, const int* rec_i, const int* rec_j,
                             int checkpoint_every, fdmap_adjoint** out) {
  if (!out) return set_err(FDMAP_ERR_INVALID_ARG, "null adjoint pointer");
  *out = nullptr;
  if (!d) return set_err(FDMAP_ERR_INVALID_ARG, "null descriptor");
  if (d->mode != 3 || !d->heterogeneous)
    return set_err(FDMAP_ERR_UNSUPPORTED, "the adjoint covers heterogeneous mode III domains");
  if (d->displacement || d->peak || d->energy_balance)
    return set_err(FDMAP_ERR_UNSUPPORTED, "the adjoint does not track displacement or peak motion");
  for (int b = 0; b < d->nblocks; ++b)
    if (d->blocks[b].Cdiss > 0.0)
      return set_err(FDMAP_ERR_UNSUPPORTED, "the adjoint does not cover artificial dissipation");
  if (d->src.gauss_forcing || d->src.forcing_filename)
    return set_err(FDMAP_ERR_UNSUPPORTED, "the adjoint covers the point source only");
  for (int b = 0; b < d->nblocks; ++b)
    for (int s = 0; s < 4; ++s) {
      const int bc = d->blocks[b].side[s].bc;
      if (bc == FDMAP_BC_NONE) {
        // an interface side must be covered by interfaces over its whole length
        const int len = s < 2 ? d->blocks[b].pgy - d->blocks[b].mgy + 1 : d->blocks[b].pgx - d->blocks[b].mgx + 1;
        int cov = 0;
        for (int i = 0; i < d->nifaces; ++i) {
          const fdmap_iface& fi = d->ifaces[i];
          const int sm = fi.direction == 0 ? 1 : 3, sp = fi.direction == 0 ? 0 : 2;
          if ((fi.iblockm == b && sm == s) || (fi.iblockp == b && sp == s)) cov += fi.p - fi.m + 1;
        }
        if (cov != len) return set_err(FDMAP_ERR_UNSUPPORTED, "adjoint: a side without a boundary condition is not an interface");
      } else if (bc != FDMAP_BC_ABSORBING && bc != FDMAP_BC_FREE && bc != FDMAP_BC_RIGID) {
        return set_err(FDMAP_ERR_UNSUPPORTED, "adjoint sides must be absorbing, free or rigid");
      }
    }
  for (int i = 0; i < d->nifaces; ++i) {
    const fdmap_iface& fi = d->ifaces[i];
    if (fi.coupling == FDMAP_COUPLING_LOCKED) continue;
    const fdmap_friction& fr = fi.fr;
    // the smooth laws: the slip-weakening kink has no derivative
    if (fr.law == FDMAP_FR_SW)
      return set_err(FDMAP_ERR_UNSUPPORTED, "the adjoint covers locked and rate-and-state interfaces, not slip weakening");
    if (fr.force || fr.reg)
      return set_err(FDMAP_ERR_UNSUPPORTED, "the adjoint does not cover forced rupture or regularised normal stress");
  }
  if (nrec < 1 || !rec_i || !rec_j) return set_err(FDMAP_ERR_INVALID_ARG, "receivers required");
  if (checkpoint_every < 1) return set_err(FDMAP_ERR_INVALID_ARG, "checkpoint interval must be positive");
  fdmap_adjoint* a = new (std::nothrow) fdmap_adjoint();
  if (!a) return set_err(FDMAP_ERR_NOMEM, "out of host memory");
  auto fail = [&](int rc) {
    std::string keep = g_err;
    delete a;
    g_err = keep;
    return rc;
  };
  int rc = fdmap_gpu_create(d, device, 1, &a->h);
  if (rc) return fail(rc);
  fdmap_gpu* h = a->h;
  a->K = checkpoint_every;
  a->nrec = nrec;
  a->general = d->nblocks > 1 || d->nifaces > 0;
  a->nb = d->nblocks;
  const BlockGeom& g = h->geom[0];
  const int nbnd = h->hdom.nbnd;
  for (int b = 0; b < a->nb; ++b) {
    const BlockGeom& gb = h->geom[b];
    if (gb.nx < 2 * nbnd + 1 || gb.ny < 2 * nbnd + 1)
      return fail(set_err(FDMAP_ERR_UNSUPPORTED, "block too small for the adjoint band decomposition"));
    a->boff[b] = a->total;
    a->goff[b] = a->gtotal;
    a->total += 3 * gb.plane;
    a->gtotal += gb.plane;
  }
  for (int b = 0; b < a->nb; ++b)
    a->nband.push_back(2LL * nbnd * h->geom[b].nx + 2LL * nbnd * (h->geom[b].ny - 2 * nbnd));
  for (int i = 0; i < d->nifaces; ++i) {
    const fdmap_iface& fi = d->ifaces[i];
    const int n = fi.p - fi.m + 1;
    a->info_host.push_back(AdjIfaceInfo{i, a->nfault, nullptr, nullptr});
    a->nfault += n;
    if (fi.coupling == FDMAP_COUPLING_LOCKED) {
      a->st_off.push_back(-1);
    } else {
      a->st_off.push_back(a->total + a->st_total);
      a->st_total += (long long)FDMAP_FAULT_NFIELDS * n;
      // the background shear stress term is always read, so the prestress can be set
      h->hdom.ifc[i].fr.has_bsS0 = 1;
    }
  }
  {
    int lo = 0, hi = 0;
    if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&a->side, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&a->copy, cudaStreamNonBlocking, lo) != cudaSuccess ||
        cudaEventCreateWithFlags(&a->ev_cfork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&a->ev_cjoin, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&a->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&a->ev_join, cudaEventDisableTiming) != cudaSuccess)
      return fail(set_err(FDMAP_ERR_CUDA, "adjoint stream setup"));
  }
  for (int r = 0; r < nrec; ++r) {
    int b = 0;
    while (b < a->nb && !(rec_i[r] >= h->geom[b].mgx && rec_i[r] < h->geom[b].mgx + h->geom[b].nx &&
                          rec_j[r] >= h->geom[b].mgy && rec_j[r] < h->geom[b].mgy + h->geom[b].ny))
      ++b;
    if (b == a->nb) return fail(set_err(FDMAP_ERR_INVALID_ARG, "receiver outside the domain"));
    const BlockGeom& gb = h->geom[b];
    const long long local = (long long)(rec_j[r] - gb.mgy) * gb.pitch + (rec_i[r] - gb.mgx);
    a->rec_host.push_back(a->boff[b] + local);  // vz of the node in the concatenated layout
    a->rec_gen.push_back({b, local});
  }
  const long long S = a->total;
  if ((rc = a->alloc(&a->rec, nrec)) || (rc = a->alloc(&a->init_F, S)) || (rc = a->alloc(&a->init_DF, S)) ||
      (rc = a->alloc(&a->store, (size_t)a->K * h->rk.nstage * a->slot_stride())) || (rc = a->alloc(&a->ub[0], S)) ||
      (rc = a->alloc(&a->ub[1], S)) || (rc = a->alloc(&a->qp[0], S)) || (rc = a->alloc(&a->qp[1], S)) ||
      (rc = a->alloc(&a->grho, a->gtotal)) || (rc = a->alloc(&a->gG, a->gtotal)) || (rc = a->alloc(&a->clock, 1)))
    return fail(rc);
  if (a->general) {
    if ((rc = a->alloc(&a->init_st, std::max<long long>(a->st_total, 1))) ||
        (rc = a->alloc(&a->psib[0], std::max(a->nfault, 1))) || (rc = a->alloc(&a->qpsib[0], std::max(a->nfault, 1))) ||
        (rc = a->alloc(&a->psib[1], std::max(a->nfault, 1))) || (rc = a->alloc(&a->qpsib[1], std::max(a->nfault, 1))) ||
        (rc = a->alloc(&a->gS0, std::max(a->nfault, 1))) || (rc = a->alloc(&a->recp[0], nrec)) ||
        (rc = a->alloc(&a->recp[1], nrec)))
      return fail(rc);
    for (int c = 0; c < 2; ++c) {
      std::vector<const double*> ptr(nrec);
      for (int r = 0; r < nrec; ++r) ptr[r] = h->hdom.blk[a->rec_gen[r].first].F[c] + a->rec_gen[r].second;
      if (cudaMemcpy(a->recp[c], ptr.data(), nrec * sizeof(double*), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_err(FDMAP_ERR_CUDA, "receiver upload"));
    }
  }
  if (cudaMemcpy(a->rec, a->rec_host.data(), nrec * sizeof(long long), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(set_err(FDMAP_ERR_CUDA, "receiver upload"));
  {
    // distinct receiver nodes in first-appearance order, receivers listed per node
    std::vector<long long> nodes;
    std::vector<std::vector<int>> members;
    for (int r = 0; r < nrec; ++r) {
      auto it = std::find(nodes.begin(), nodes.end(), a->rec_host[r]);
      if (it == nodes.end()) { nodes.push_back(a->rec_host[r]); members.push_back({r}); }
      else members[it - nodes.begin()].push_back(r);
    }
    std::vector<int> rstart(1, 0), rlist;
    for (auto& m : members) {
      rlist.insert(rlist.end(), m.begin(), m.end());
      rstart.push_back((int)rlist.size());
    }
    a->nnode = (int)nodes.size();
    if ((rc = a->alloc(&a->node, nodes.size())) || (rc = a->alloc(&a->rstart, rstart.size())) ||
        (rc = a->alloc(&a->rlist, rlist.size())))
      return fail(rc);
    if (cudaMemcpy(a->node, nodes.data(), nodes.size() * sizeof(long long), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(a->rstart, rstart.data(), rstart.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(a->rlist, rlist.data(), rlist.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(set_err(FDMAP_ERR_CUDA, "receiver upload"));
  }
  for (int b = 0; b < a->nb; ++b) {
    const DevBlock& B = h->hdom.blk[b];
    if (cudaMemcpy(a->init_F + a->boff[b], B.F[h->cur], 3 * B.plane * sizeof(double), cudaMemcpyDeviceToDevice) !=
            cudaSuccess ||
        cudaMemcpy(a->init_DF + a->boff[b], B.DF, 3 * B.plane * sizeof(double), cudaMemcpyDeviceToDevice) !=
            cudaSuccess)
      return fail(set_err(FDMAP_ERR_CUDA, "initial state copy"));
  }
  for (int i = 0; i < d->nifaces; ++i)
    if (a->st_off[i] >= 0 &&
        cudaMemcpy(a->init_st + (a->st_off[i] - a->total), h->hdom.ifc[i].fr.st,
                   (size_t)FDMAP_FAULT_NFIELDS * h->hdom.ifc[i].n * sizeof(double), cudaMemcpyDeviceToDevice) != cudaSuccess)
      return fail(set_err(FDMAP_ERR_CUDA, "initial fault state copy"));
  // edge geometry factors H00i*|grad|/J (init_edges, domain.f90:1349-1459)
  SbpOperator op;
  sbp_operator(d->fd_method, &op);
  a->geo.assign(4 * a->nb, nullptr);
  for (int b = 0; b < a->nb; ++b) {
    const fdmap_block& fb = d->blocks[b];
    const BlockGeom& gb = h->geom[b];
    for (int s = 0; s < 4; ++s) {
      const int n = (s < 2) ? gb.ny : gb.nx;
      if ((rc = a->alloc(&a->geo[4 * b + s], n))) return fail(rc);
      if (d->body) {
        // body built on the device: the factors come from its metric planes
        adj_edge_geometry<<<(n + 127) / 128, 128, 0, h->stream>>>(h->hdom.blk[b], s, n, op.H00i, a->geo[4 * b + s]);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess)
          return fail(set_err(FDMAP_ERR_CUDA, "edge geometry"));
        continue;
      }
      std::vector<double> geo(n);
      for (int k = 0; k < n; ++k) {
        int i, j;
        if (s == 0) { i = fb.mgx; j = fb.mgy + k; }
        else if (s == 1) { i = fb.pgx; j = fb.mgy + k; }
        else if (s == 2) { i = fb.mgx + k; j = fb.mgy; }
        else { i = fb.mgx + k; j = fb.pgy; }
        const size_t q = (size_t)(i - 1) + (size_t)d->nx * (size_t)(j - 1);
        const double mag = (s < 2) ? std::sqrt(d->xr[q] * d->xr[q] + d->yr[q] * d->yr[q])
                                   : std::sqrt(d->xq[q] * d->xq[q] + d->yq[q] * d->yq[q]);
        geo[k] = op.H00i * mag / d->J[q];
      }
      if (cudaMemcpy(a->geo[4 * b + s], geo.data(), n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_err(FDMAP_ERR_CUDA, "geometry upload"));
    }
  }
  if (a->general && !a->info_host.empty()) {
    for (auto& inf : a->info_host) {
      const DevIface& I = h->hdom.ifc[inf.iface];
      inf.geom = a->geo[4 * I.im + (I.direction == 0 ? 1 : 3)];
      inf.geop = a->geo[4 * I.ip + (I.direction == 0 ? 0 : 2)];
    }
    if ((rc = a->alloc(&a->info, a->info_host.size()))) return fail(rc);
    if (cudaMemcpy(a->info, a->info_host.data(), a->info_host.size() * sizeof(AdjIfaceInfo), cudaMemcpyHostToDevice) !=
        cudaSuccess)
      return fail(set_err(FDMAP_ERR_CUDA, "interface table upload"));
  }
  if ((rc = adj_maps(a))) return fail(rc);
  *out = a;
  return FDMAP_OK;
}

int fdmap_gpu_adjoint_set_material(fdmap_adjoint* a, const double* rho, const double* G) {
  if (!a || !rho || !G) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  fdmap_gpu* h = a->h;
  a->resident = 0;  // stored stage inputs belong to the old model: a backward recomputes
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (size_t q = 0; q < (size_t)h->nx_g * h->ny_g; ++q)
    if (!(rho[q] > 0.0) || !(G[q] > 0.0)) return set_err(FDMAP_ERR_INVALID_ARG, "density and shear modulus must be positive");
  int rc;
  for (int b = 0; b < a->nb; ++b) {
    DevBlock& B = h->hdom.blk[b];
    const BlockGeom& gb = h->geom[b];
    if ((rc = to_block(a, B.rho, rho, b))) return rc;
    if ((rc = to_block(a, B.G, G, b))) return rc;
    for (int s = 0; s < 4; ++s) {
      const DevSide& S = B.side[s];
      adj_edge_material<<<(S.n + 127) / 128, 128, 0, h->stream>>>(S, B.rho, B.G, a->geo[4 * b + s], s, gb.nx, gb.ny,
                                                                  gb.pitch);
      CUDA_TRY(cudaGetLastError());
    }
  }
  for (auto& inf : a->info_host) {
    const DevIface& I = h->hdom.ifc[inf.iface];
    const DevSide& Sm = h->hdom.blk[I.im].side[I.direction == 0 ? 1 : 3];
    const DevSide& Sp = h->hdom.blk[I.ip].side[I.direction == 0 ? 0 : 2];
    adj_iface_material<<<(I.n + 127) / 128, 128, 0, h->stream>>>(I, Sm, Sp);
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return FDMAP_OK;
}

int fdmap_gpu_adjoint_forward(fdmap_adjoint* a, double t_start, double dt, int nt, const double* data, double* traces,
                              double* misfit) {
  if (!a) return set_err(FDMAP_ERR_INVALID_ARG, "null adjoint");
  if (nt < 2) return set_err(FDMAP_ERR_INVALID_ARG, "nt must be at least 2");
  fdmap_gpu* h = a->h;
  CUDA_TRY(cudaSetDevice(h->device));
  // until this run has finished, there is nothing to take a backward pass over
  a->have_resid = false;
  a->resident = 0;
  int rc;
  if ((rc = ensure_trace_buffers(a, nt))) return rc;
  const int nck = (nt - 1 + a->K - 1) / a->K;
  if ((rc = ensure_checkpoints(a, nck))) return rc;
  // a run with data precedes a backward: its last R segments keep their stage inputs
  if (data && (rc = ensure_store(a, nck))) return rc;
  const int R = data ? a->plan_R : 0;
  a->N = nt;
  a->t_start = t_start;
  a->dt = dt;
  if (a->graph_dt != dt || a->graph_t0 != t_start || !a->g_fwd[0]) {
    if ((rc = build_graphs(a, dt))) return rc;
    a->graph_t0 = t_start;
  }
  // reset to the initial state
  DevBlock& B = h->hdom.blk[0];
  h->cur = 0;
  if ((rc = restore_state(a, a->init_F, a->init_st))) return rc;
  for (int b = 0; b < a->nb; ++b)
    CUDA_TRY(cudaMemcpyAsync(h->hdom.blk[b].DF, a->init_DF + a->boff[b], 3 * h->hdom.blk[b].plane * sizeof(double),
                             cudaMemcpyDeviceToDevice, h->stream));
  set_step_clock<<<1, 1, 0, h->stream>>>(h->d_time, t_start, dt, 1);
  // sample 1: the initial state; each replayed step samples the state it produces
  if (a->general)
    adj_sample_ptr<<<(a->nrec + 127) / 128, 128, 0, h->stream>>>(a->recp[0], a->nrec, h->d_time, a->traces, nt);
  else
    adj_sample<<<(a->nrec + 127) / 128, 128, 0, h->stream>>>(B.F[0], a->rec, a->nrec, h->d_time, a->traces, nt);
  CUDA_TRY(cudaGetLastError());
  const int first = nck - R;  // first resident segment
  for (int n = 1; n <= nt - 1; ++n) {
    const int seg = (n - 1) / a->K;
    if ((n - 1) % a->K == 0) {
      if ((rc = save_state(a, a->ckpt + (size_t)seg * a->ckpt_stride()))) return rc;
      if (R > 0 && seg == first) {
        // resident segment r, step k: store step index r*K + k
        AdjClock c0{0, nt};
        CUDA_TRY(cudaMemcpyAsync(a->clock, &c0, sizeof(c0), cudaMemcpyHostToDevice, h->stream));
      }
    }
    CUDA_TRY(cudaGraphLaunch(seg >= first ? a->g_fst[h->cur] : a->g_fwd[h->cur], h->stream));
    if (h->rk.nstage & 1) h->cur = 1 - h->cur;
  }
  std::vector<double> tr((size_t)nt * a->nrec);
  CUDA_TRY(cudaMemcpyAsync(tr.data(), a->traces, tr.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (traces) std::memcpy(traces, tr.data(), tr.size() * sizeof(double));
  if (data) {
    double J = 0.0;
    for (size_t q = 0; q < tr.size(); ++q) {
      const double r = tr[q] - data[q];
      tr[q] = r;
      J += 0.5 * r * r;
    }
    if (misfit) *misfit = J;
    CUDA_TRY(cudaMemcpy(a->resid, tr.data(), tr.size() * sizeof(double), cudaMemcpyHostToDevice));
    a->have_resid = true;
    a->resident = R;
  }
  return FDMAP_OK;
}

int fdmap_gpu_adjoint_backward(fdmap_adjoint* a, double* grad_rho, double* grad_G) {
  if (!a) return set_err(FDMAP_ERR_INVALID_ARG, "null adjoint");
  if (!a->have_resid) return set_err(FDMAP_ERR_INVALID_ARG, "backward needs a forward run with data");
  fdmap_gpu* h = a->h;
  CUDA_TRY(cudaSetDevice(h->device));
  const long long S = a->total;
  const int N = a->N;
  const size_t plane_bytes = (size_t)a->gtotal * sizeof(double);
  for (int q = 0; q < 2; ++q) {
    CUDA_TRY(cudaMemsetAsync(a->ub[q], 0, S * sizeof(double), h->stream));
    CUDA_TRY(cudaMemsetAsync(a->qp[q], 0, S * sizeof(double), h->stream));
  }
  CUDA_TRY(cudaMemsetAsync(a->grho, 0, plane_bytes, h->stream));
  CUDA_TRY(cudaMemsetAsync(a->gG, 0, plane_bytes, h->stream));
  if (a->nfault > 0) {
    for (int q = 0; q < 2; ++q) {
      CUDA_TRY(cudaMemsetAsync(a->psib[q], 0, a->nfault * sizeof(double), h->stream));
      CUDA_TRY(cudaMemsetAsync(a->qpsib[q], 0, a->nfault * sizeof(double), h->stream));
    }
    CUDA_TRY(cudaMemsetAsync(a->gS0, 0, a->nfault * sizeof(double), h->stream));
  }
  // dJ/dU^N at the receivers
  AdjClock ck{0, N};
  CUDA_TRY(cudaMemcpyAsync(a->clock, &ck, sizeof(ck), cudaMemcpyHostToDevice, h->stream));
  adj_inject<<<1, 128, 0, h->stream>>>(a->ub[0], a->node, a->rstart, a->rlist, a->nnode, a->nrec, a->resid, a->clock,
                                       0);
  CUDA_TRY(cudaGetLastError());
  int p = 0;  // ubar parity
  const int nseg = (N - 1 + a->K - 1) / a->K;
  const int R = a->resident, first = nseg - R;
  // recomputed segments go to the store after the resident ones
  const long long rbase = (long long)R * a->K;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int n0 = seg * a->K + 1, n1 = std::min(n0 + a->K, N);  // steps n0 .. n1-1
    long long base = (long long)(seg - first) * a->K;
    if (seg < first) {
      h->cur = 0;
      int rc = restore_state(a, a->ckpt + (size_t)seg * a->ckpt_stride(), nullptr);
      if (rc) return rc;
      set_step_clock<<<1, 1, 0, h->stream>>>(h->d_time, a->t_start, a->dt, n0);
      ck.rel = rbase;
      ck.n = N;  // unused while recomputing
      CUDA_TRY(cudaMemcpyAsync(a->clock, &ck, sizeof(ck), cudaMemcpyHostToDevice, h->stream));
      for (int n = n0; n < n1; ++n) {
        CUDA_TRY(cudaGraphLaunch(a->g_rec[h->cur], h->stream));
        if (h->rk.nstage & 1) h->cur = 1 - h->cur;
      }
      base = rbase;
    }
    ck.rel = base + (n1 - 1 - n0);
    ck.n = n1 - 1;
    CUDA_TRY(cudaMemcpyAsync(a->clock, &ck, sizeof(ck), cudaMemcpyHostToDevice, h->stream));
    for (int n = n1 - 1; n >= n0; --n) {
      CUDA_TRY(cudaGraphLaunch(a->g_adj[p], h->stream));
      if (h->rk.nstage & 1) p = 1 - p;
    }
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (int b = 0; b < a->nb; ++b) {
    int rc;
    if (grad_rho && (rc = from_block(a, grad_rho, a->grho + a->goff[b], b))) return rc;
    if (grad_G && (rc = from_block(a, grad_G, a->gG + a->goff[b], b))) return rc;
  }
  return FDMAP_OK;
}

int fdmap_gpu_adjoint_fault_size(const fdmap_adjoint* a) { return a ? a->nfault : 0; }

int fdmap_gpu_adjoint_set_store_budget(fdmap_adjoint* a, long long bytes) {
  if (!a) return set_err(FDMAP_ERR_INVALID_ARG, "null adjoint");
  a->store_budget = bytes < 0 ? -1 : bytes;
  return FDMAP_OK;
}

long long fdmap_gpu_adjoint_segment_bytes(const fdmap_adjoint* a) { return a ? (long long)a->segment_bytes() : 0; }

int fdmap_gpu_adjoint_resident_segments(const fdmap_adjoint* a) { return a ? a->resident : 0; }

int fdmap_gpu_adjoint_time_params(fdmap_adjoint* a, double* params, int* nt) {
  if (!a) return set_err(FDMAP_ERR_INVALID_ARG, "null adjoint");
  return fdmap_gpu_time_params(a->h, params, nt);
}

int fdmap_gpu_adjoint_set_prestress(fdmap_adjoint* a, const double* S0) {
  if (!a || !S0) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  fdmap_gpu* h = a->h;
  a->resident = 0;
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (const auto& inf : a->info_host) {
    const DevIface& I = h->hdom.ifc[inf.iface];
    if (I.coupling == FDMAP_COUPLING_LOCKED) continue;
    CUDA_TRY(cudaMemcpy(I.fr.par + (size_t)PAR_BSS0 * I.n, S0 + inf.start, I.n * sizeof(double),
                        cudaMemcpyHostToDevice));
  }
  return FDMAP_OK;
}

int fdmap_gpu_adjoint_get_prestress(fdmap_adjoint* a, double* S0) {
  if (!a || !S0) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  fdmap_gpu* h = a->h;
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (const auto& inf : a->info_host) {
    const DevIface& I = h->hdom.ifc[inf.iface];
    if (I.coupling == FDMAP_COUPLING_LOCKED) {
      std::fill(S0 + inf.start, S0 + inf.start + I.n, 0.0);
      continue;
    }
    CUDA_TRY(cudaMemcpy(S0 + inf.start, I.fr.par + (size_t)PAR_BSS0 * I.n, I.n * sizeof(double),
                        cudaMemcpyDeviceToHost));
  }
  return FDMAP_OK;
}

int fdmap_gpu_adjoint_prestress_gradient(fdmap_adjoint* a, double* grad_S0) {
  if (!a || !grad_S0) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  if (a->nfault == 0) return FDMAP_OK;
  CUDA_TRY(cudaSetDevice(a->h->device));
  CUDA_TRY(cudaStreamSynchronize(a->h->stream));
  CUDA_TRY(cudaMemcpy(grad_S0, a->gS0, a->nfault * sizeof(double), cudaMemcpyDeviceToHost));
  return FDMAP_OK;
}

int fdmap_gpu_adjoint_fields(fdmap_adjoint* a, double* F) {
  if (!a) return set_err(FDMAP_ERR_INVALID_ARG, "null adjoint");
  return fdmap_gpu_get_fields(a->h, F, nullptr);
}

void fdmap_gpu_adjoint_destroy(fdmap_adjoint* a) { delete a; }

}  // extern "C"
