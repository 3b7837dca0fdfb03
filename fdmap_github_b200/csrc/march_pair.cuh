// Two-stage march: two consecutive stages s, s+1 of the low-storage RK step
// (time_step_LS, time_step.f90:96-165) in one pass over HBM, for blocks with
// homogeneous material and the plain split form.
//
// Why: one stage moves every node's fields, rates and metric terms through
// HBM (224 B per node in mode II) for about 150 FP64 operations, so a stage
// is bound by HBM bandwidth.  Stage s+1 at a node needs stage s only within
// PI nodes of it, so a tile that computes stage s on its core plus a PI-wide
// halo can go on to stage s+1 on the core without writing stage s out: the
// pass reads F, DF and the metric terms once and writes F and DF once for
// two stages.
//
// What crosses the edges.  Stage s+1 at a node needs stage s at its
// neighbours, and stage s near a block edge needs the interface solve of
// stage s (the SAT at the edge node) and the one-sided closure rows.  Those
// are left to the boundary kernels, so the pass splits the nodes of a block
// by their distance d from its nearest edge:
//   - d >= nbst + PI: both stages here (every neighbour stage s needs is an
//     interior node, computed here from the stage's input alone);
//   - nbst <= d < nbst + 2 PI: stage s here; its values are written to the
//     scratch buffer F[2] (and its rates, where d < nbst + PI, to the pass's
//     rate buffer) for the band kernel;
//   - d < nbst: stage s by the closure kernel (into F[2]), after the
//     interface solve of stage s.
// The interface solve of stage s+1 reads F[2] at the edge nodes, and the band
// kernel (band_kernel below) then does stage s+1 at every node with
// d < nbst + PI.
//
// Buffers.  F goes from F[in] to F[out] (in != out) across the pair; the
// rates go from one rate buffer (DF or DFalt, read only where A != 0) to the
// other: a tile reads the input rates of its halo while the neighbouring
// tile already writes its result, so neither may be updated in place.
//
// Tile: 128 threads across (the extended columns of stage s) x 2 rows; the
// core is the middle 128 - 2 PI columns.  Row groups stream through
// shared-memory rings filled by 3-D TMA boxes (no multicast) that all start
// at column i0 - 2 PI (an even column, so every box starts on 16 bytes):
//   - input ring (6 slots): the rate fields and yr, xr, yq, xq, Ji of a row
//     group, {128 + 2 PI, 2, NR} and {128 + 2 PI, 2, 5};
//   - centre ring (3 slots): the stage-s input rates (A != 0) and szz;
//   - stage-s ring (4 slots): the rate fields after stage s, read by stage
//     s+1 at the neighbours; each thread keeps its own node's stage-s rates
//     and szz in registers for stage s+1 two iterations later.
// Stage s runs two row groups ahead of stage s+1, so within one iteration
// the two stages touch disjoint data and one barrier per iteration suffices;
// a ring slot is refilled after that barrier, once every thread has left the
// iteration that last read it.  Every mbarrier wait is bounded in time; a CTA
// whose wait gives up stops, drains its copies and leaves (status word ->
// FDMAP_ERR_TIMEOUT).
#pragma once

#include "march_kernel.cuh"

namespace fdmap {

template <int MODE, int PI_>
struct PairLayout {
  static constexpr int MWX = 128;             // threads across: extended columns of stage s
  static constexpr int MWC = MWX - 2 * PI_;   // core columns of a strip (stage s+1)
  static constexpr int MR = 2;                // rows of a row group
  static constexpr int THREADS = MWX * MR;
  static constexpr int WB = MWX + 2 * PI_;    // box width: columns i0 - 2 PI .. i0 + MWC + 2 PI - 1
  static constexpr int NGS = 6, NCS = 3, N1S = 4;
  static constexpr int NR = RDef<MODE>::NR;
  // input slot: rate fields [NR][MR][WB], yr, xr, yq, xq, Ji [5][MR][WB]
  static constexpr size_t F_OFF = 0;
  static constexpr size_t M_OFF = align128((size_t)NR * MR * WB * 8);
  static constexpr size_t GSLOT = align128(M_OFF + (size_t)5 * MR * WB * 8);
  // centre slot: stage-s input rates [NR][MR][WB], szz [MR][WB] (mode II)
  static constexpr size_t DF_OFF = 0;
  static constexpr size_t F6_OFF = align128((size_t)NR * MR * WB * 8);
  static constexpr size_t CSLOT = align128(F6_OFF + (MODE == 2 ? (size_t)MR * WB * 8 : 0));
  // stage-s slot: rate fields after stage s [NR][MR][MWX]
  static constexpr size_t S1SLOT = align128((size_t)NR * MR * MWX * 8);
  static constexpr size_t C_BASE = (size_t)NGS * GSLOT;
  static constexpr size_t S1_BASE = C_BASE + (size_t)NCS * CSLOT;
  static constexpr size_t BARS_OFF = S1_BASE + (size_t)N1S * S1SLOT;
  static constexpr size_t BYTES = BARS_OFF + (NGS + NCS) * 8 + 128;  // + alignment slack
  static constexpr unsigned NB_BYTES = (unsigned)((size_t)(NR + 5) * MR * WB * 8);
  static_assert(PI_ <= MR, "PI rows must fit in one row group");
  static_assert((N1S & (N1S - 1)) == 0, "the stage-s ring index wraps by masking");
};

// TMA descriptors of the two-stage march, every box {WB, MR, planes}
struct TmapPair {
  CUtensorMap F[MAX_BLOCKS][2];   // rate fields of F[0], F[1]
  CUtensorMap F6[MAX_BLOCKS][2];  // szz plane (mode II)
  CUtensorMap DF[MAX_BLOCKS][2];  // rate fields of DF, DFalt
  CUtensorMap MT[MAX_BLOCKS];     // yr, xr, yq, xq, Ji
};

struct PairPlan {
  long long units;               // strips of MWC columns x row groups, all blocks (all instances)
  const TmapPair* tms;           // batched instances: per-instance maps in device memory, else NULL
  const long long* unit_begin;   // batched instances: prefix of units over instances
  int ninst;
  int dfr, dfw;                  // rate buffer read by stage s / written by both stages (0 DF, 1 DFalt)
};

// distance of block-local node (i, j) from the block's nearest edge
__device__ __forceinline__ int edge_distance(int i, int j, int nx, int ny) {
  return min(min(i, nx - 1 - i), min(j, ny - 1 - j));
}

// 168 registers a thread (no spills): two warps of the pass take 10.5K of a
// sub-partition's 16K registers, so a boundary warp (128 registers a
// thread) fits beside them
template <int MODE, int PI_>
__global__ void __maxnreg__(168)
    march_pair_kernel(const DevDomain* __restrict__ doms, StageArgs a0, StageArgs a1, PairPlan plan,
                      const __grid_constant__ TmapPair tm) {
  using L = PairLayout<MODE, PI_>;
  constexpr int MWX = L::MWX, MWC = L::MWC, MR = L::MR, WB = L::WB;
  constexpr int NR = L::NR;
  constexpr int NF = MODE == 2 ? 6 : 3;
  constexpr int NGS = L::NGS, NCS = L::NCS, N1S = L::N1S;
  extern __shared__ unsigned char smem_dyn[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  unsigned long long* nbar = reinterpret_cast<unsigned long long*>(smem + L::BARS_OFF);
  unsigned long long* cbar = nbar + NGS;

  const int tid = threadIdx.x;
  const int cx = tid % MWX, ry = tid / MWX;
  const unsigned long long t_in = (tid == 0 && doms[0].trace.rec) ? globaltimer_ns() : 0ull;
  const long long ubeg = plan.units * blockIdx.x / gridDim.x;
  const long long uend = plan.units * (blockIdx.x + 1) / gridDim.x;
  const bool load_df = a0.A != 0.0;  // A = 0 (first stage of a step): the input rates are not read
  const unsigned cbytes = (unsigned)((load_df ? (size_t)NR * MR * WB * 8 : 0) + (MODE == 2 ? (size_t)MR * WB * 8 : 0));

  long long u = ubeg;
  while (u < uend) {
    int inst = 0;
    long long base = 0;
    if (plan.ninst > 1) {
      int lo = 0, hi = plan.ninst - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (plan.unit_begin[mid] <= u) lo = mid;
        else hi = mid - 1;
      }
      inst = lo;
      base = plan.unit_begin[inst];
    }
    const DevDomain& D = doms[inst];
    const TmapPair& tmi = plan.tms ? plan.tms[inst] : tm;
    // segment: consecutive row groups of one strip
    int b = 0;
    while (b + 1 < D.nblocks && u - base >= D.blk[b + 1].pair_unit_begin) ++b;
    const DevBlock& B = D.blk[b];
    const int groups = (B.ny + MR - 1) / MR;
    const long long local = u - base - B.pair_unit_begin;
    const int sx = (int)(local / groups);
    const int jr0 = (int)(local % groups) * MR;
    const long long strip_end = base + B.pair_unit_begin + (long long)(sx + 1) * groups;
    const long long seg_end = uend < strip_end ? uend : strip_end;
    const int nx = B.nx, ny = B.ny;
    const long long pitch = B.pitch, plane = B.plane;
    const int jr1 = min(ny, (int)(jr0 + (seg_end - u) * MR));
    const int ngroups = (jr1 - jr0 + MR - 1) / MR;
    const int i0 = sx * MWC;      // first core column
    const int xb = i0 - 2 * PI_;  // first column of every box (even)
    // stage s on row groups ks0..ks1: the core groups and one more on each
    // side inside the block; input groups gmin..gmax around them
    const int ks0 = jr0 > 0 ? -1 : 0;
    const int ks1 = ngroups - 1 + (jr1 < ny ? 1 : 0);
    const int gmin = max(ks0 - 1, -(jr0 / MR));
    const int gmax = min(ks1 + 1, (ny - 1 - jr0) / MR);
    const CUtensorMap* mF = &tmi.F[b][a0.in];
    const CUtensorMap* mF6 = &tmi.F6[b][a0.in];
    const CUtensorMap* mDF = &tmi.DF[b][plan.dfr];

    if (tid == 0) {
      for (int s = 0; s < NGS + NCS; ++s) mbar_init(&nbar[s], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    int nb_next = gmin, c_next = ks0;  // next input / centre group to be filled (thread 0)
    auto fill_nb = [&](int k) {
      nb_next = k + 1;
      const int sl = (k - gmin) % NGS;
      unsigned char* g = smem + (size_t)sl * L::GSLOT;
      const int row = jr0 + k * MR;
      mbar_arrive_tx(&nbar[sl], L::NB_BYTES);
      tma_load_3d(g + L::F_OFF, mF, xb, row, 0, &nbar[sl]);
      tma_load_3d(g + L::M_OFF, &tmi.MT[b], xb, row, 0, &nbar[sl]);
    };
    auto fill_c = [&](int k) {
      c_next = k + 1;
      const int sl = (k - ks0) % NCS;
      unsigned char* g = smem + L::C_BASE + (size_t)sl * L::CSLOT;
      const int row = jr0 + k * MR;
      mbar_arrive_tx(&cbar[sl], cbytes);
      if (load_df) tma_load_3d(g + L::DF_OFF, mDF, xb, row, 0, &cbar[sl]);
      if (MODE == 2) tma_load_3d(g + L::F6_OFF, mF6, xb, row, 5, &cbar[sl]);
    };
    if (tid == 0) {
      fence_proxy_async();
      for (int k = gmin; k <= min(gmax, gmin + NGS - 1); ++k) fill_nb(k);
      for (int k = ks0; k <= min(ks1, ks0 + NCS - 1); ++k) fill_c(k);
    }

    double cf[PI_ + 1][3];
#pragma unroll
    for (int s = 1; s <= PI_; ++s)
#pragma unroll
      for (int q = 0; q < 3; ++q) cf[s][q] = B.coef[s][q];
    NodeMat m;
    m.rho = B.rho_b; m.G = B.G_b; m.M = B.M_b; m.gamma = B.gamma_b; m.nu = B.nu_b; m.rinv = 0.0;
    double* __restrict__ DFw = plan.dfw ? B.DFalt : B.DF;
    double* __restrict__ Fout = B.F[a1.out];
    double* __restrict__ Fband = B.F[2];
    const int nbst = D.nbst;
    const bool forces = D.src.use_gravity || (D.src.use_singular && B.src_ok);
    const double t0s = forces ? stage_time(a0) : 0.0;
    const double t1s = forces ? stage_time(a1) : 0.0;
    const int i = i0 - PI_ + cx;                           // this thread's column
    const bool core = cx >= PI_ && cx < PI_ + MWC && i < nx;  // a column of this strip's core
    const int pc = cx + PI_;                               // its position in a box row

    // group offset and row, within the ring, of row ry + dr of a row group
    // (ry and dr compile-time below: every shared-memory address is a slot
    // pointer of the iteration plus a constant)
    auto goff = [](int rr) { return rr >= 0 ? rr / MR : -((MR - 1 - rr) / MR); };

    // this thread's node, stage s, from the last two iterations (its rates
    // and szz; the other fields are in the stage-s ring): [0] group t-2, [1] t-1
    double hdf[2][NF], hf6[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      hf6[q] = 0.0;
#pragma unroll
      for (int l = 0; l < NF; ++l) hdf[q][l] = 0.0;
    }
    int aborted_at = -1;
    // iteration t: stage s at row group t, stage s+1 at row group t-2, one
    // barrier; the second stage reads only what earlier iterations wrote, so
    // the two are independent within an iteration
    // ring slots of input group t-3, stage-s group t-3 and centre group t,
    // advanced with t (a group outside the CTA's range maps to some slot: no
    // node that is computed reads it)
    int gi = ((ks0 - 3 - gmin) % NGS + NGS) % NGS;
    int si = (ks0 - 3 - ks0) & (N1S - 1);
    int ci = 0;
    for (int t = ks0; t <= ngroups + 1; ++t) {
      bool ok = true;
      // input groups t-3 .. t+1 (stage s at t needs t-1..t+1, stage s+1 at t-2
      // needs t-3..t-1): all of them on the first iteration, then the new one
      for (int k = (t == ks0 ? gmin : t + 1); k <= min(gmax, t + 1); ++k)
        ok = mbar_wait_bounded(&nbar[(k - gmin) % NGS], (unsigned)(((k - gmin) / NGS) & 1), D.status) && ok;
      if (t <= ks1) ok = mbar_wait_bounded(&cbar[ci], (unsigned)(((t - ks0) / NCS) & 1), D.status) && ok;
      if (__syncthreads_or(!ok)) {
        aborted_at = t;
        break;
      }
      // every thread is past iteration t-1: input group t-4 and centre group
      // t-1 are free; their slots take groups t+2
      if (tid == 0) {
        fence_proxy_async();
        if (t - 4 >= gmin && t + 2 <= gmax) fill_nb(t + 2);
        if (t - 1 >= ks0 && t + 2 <= ks1) fill_c(t + 2);
      }
      // this iteration's slots, offset by this thread's box column: input
      // groups t-3 .. t+1, stage-s groups t-3 .. t, the centre group t (a
      // group outside the CTA's range gets slot 0: no node that is computed
      // reads it)
      const double* gp[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        const int sl = gi + q >= NGS ? gi + q - NGS : gi + q;
        gp[q] = reinterpret_cast<const double*>(smem + (size_t)sl * L::GSLOT) + pc;
      }
      double* sp[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        sp[q] = reinterpret_cast<double*>(smem + L::S1_BASE + (size_t)((si + q) & (N1S - 1)) * L::S1SLOT) + cx;
      const double* cp = reinterpret_cast<const double*>(smem + L::C_BASE + (size_t)ci * L::CSLOT) + pc;
      gi = gi + 1 == NGS ? 0 : gi + 1;
      si = (si + 1) & (N1S - 1);
      ci = ci + 1 == NCS ? 0 : ci + 1;
      constexpr int FO = (int)(L::F_OFF / 8), MO = (int)(L::M_OFF / 8), DO = (int)(L::DF_OFF / 8),
                    SO = (int)(L::F6_OFF / 8);
      const int js = jr0 + t * MR + ry;
      const bool s_on = t <= ks1 && i >= nbst && i <= nx - 1 - nbst && js >= nbst && js <= ny - 1 - nbst;
      const int k2 = t - 2;
      const int j2 = jr0 + k2 * MR + ry;
      const bool s2_on = k2 >= 0 && core && j2 < jr1 && edge_distance(i, j2, nx, ny) >= nbst + PI_;
      double cdf[NF], cf6 = 0.0;
#pragma unroll
      for (int l = 0; l < NF; ++l) cdf[l] = 0.0;
      // the row within the group is warp-uniform: one body per row value
      auto body = [&](auto ryc) {
        constexpr int RY = decltype(ryc)::value;
        // ---- stage s+1 at row group t-2 (core nodes at least nbst + PI from every edge)
        if (s2_on) {
          double acc[NF];
#pragma unroll
          for (int l = 0; l < NR; ++l) acc[l] = a1.A != 0.0 ? a1.A * hdf[0][l] : 0.0;
          if (MODE == 2) acc[5] = 0.0;
          double Fc[NF];
#pragma unroll
          for (int l = 0; l < NR; ++l) Fc[l] = sp[1][(l * MR + RY) * MWX];
          if (MODE == 2) Fc[5] = hf6[0];
          const double Ji = gp[1][MO + (4 * MR + RY) * WB];
          split_rates<MODE, PI_, false>(
              acc, m, cf, D.DI, Ji, [&](int l, int s) { return sp[1][(l * MR + RY) * MWX + s]; },
              [&](int l, int s) {
                const int go = goff(RY + s);
                return sp[1 + go][(l * MR + (RY + s - go * MR)) * MWX];
              },
              [&](int k, int s) { return gp[1][MO + (k * MR + RY) * WB + s]; },
              [&](int k, int s) {
                const int go = goff(RY + s);
                return gp[1 + go][MO + ((2 + k) * MR + (RY + s - go * MR)) * WB];
              });
          if (MODE == 2) acc[5] = m.nu * (acc[2] + acc[4]);
          if (forces) body_forces<MODE>(D, B, i, j2, t1s, a1, acc);
          const long long c = (long long)j2 * pitch + i;
#pragma unroll
          for (int l = 0; l < NF; ++l) DFw[l * plane + c] = acc[l];
#pragma unroll
          for (int l = 0; l < NF; ++l) Fout[l * plane + c] = Fc[l] + a1.Bdt * acc[l];
        }
        // ---- stage s at row group t (interior nodes of the extended tile)
        if (s_on) {
          double acc[NF];
          if (load_df) {
#pragma unroll
            for (int l = 0; l < NR; ++l) acc[l] = a0.A * cp[DO + (l * MR + RY) * WB];
          } else {
#pragma unroll
            for (int l = 0; l < NR; ++l) acc[l] = 0.0;
          }
          if (MODE == 2) acc[5] = 0.0;
          double Fc[NF];
#pragma unroll
          for (int l = 0; l < NR; ++l) Fc[l] = gp[3][FO + (l * MR + RY) * WB];
          if (MODE == 2) Fc[5] = cp[SO + RY * WB];
          const double Ji = gp[3][MO + (4 * MR + RY) * WB];
          split_rates<MODE, PI_, false>(
              acc, m, cf, D.DI, Ji, [&](int l, int s) { return gp[3][FO + (l * MR + RY) * WB + s]; },
              [&](int l, int s) {
                const int go = goff(RY + s);
                return gp[3 + go][FO + (l * MR + (RY + s - go * MR)) * WB];
              },
              [&](int k, int s) { return gp[3][MO + (k * MR + RY) * WB + s]; },
              [&](int k, int s) {
                const int go = goff(RY + s);
                return gp[3 + go][MO + ((2 + k) * MR + (RY + s - go * MR)) * WB];
              });
          if (MODE == 2) acc[5] = m.nu * (acc[2] + acc[4]);
          if (forces) body_forces<MODE>(D, B, i, js, t0s, a0, acc);
          double F1[NF];
#pragma unroll
          for (int l = 0; l < NF; ++l) {
            cdf[l] = acc[l];
            F1[l] = Fc[l] + a0.Bdt * acc[l];
          }
          if (MODE == 2) cf6 = F1[5];
#pragma unroll
          for (int l = 0; l < NR; ++l) sp[3][(l * MR + RY) * MWX] = F1[l];
          // values the band kernel reads: stage s within nbst + 2 PI of an edge
          const int d = edge_distance(i, js, nx, ny);
          if (core && js >= jr0 && js < jr1 && d < nbst + 2 * PI_) {
            const long long c = (long long)js * pitch + i;
#pragma unroll
            for (int l = 0; l < NF; ++l) Fband[l * plane + c] = F1[l];
            if (d < nbst + PI_) {
#pragma unroll
              for (int l = 0; l < NF; ++l) DFw[l * plane + c] = cdf[l];
            }
          }
        }
      };
      if (ry == 0) body(std::integral_constant<int, 0>{});
      else body(std::integral_constant<int, 1>{});
#pragma unroll
      for (int l = 0; l < NF; ++l) { hdf[0][l] = hdf[1][l]; hdf[1][l] = cdf[l]; }
      hf6[0] = hf6[1];
      hf6[1] = cf6;
    }
    if (aborted_at >= 0) {
      // wait (bounded again) for every copy this CTA may still have in flight
      // into its shared memory, then end the CTA
      if (tid == 0) {
        const int t = aborted_at;
        for (int k = max(gmin, t - 3); k < nb_next; ++k)
          mbar_wait_bounded(&nbar[(k - gmin) % NGS], (unsigned)(((k - gmin) / NGS) & 1), D.status);
        for (int k = max(ks0, t); k < c_next; ++k)
          mbar_wait_bounded(&cbar[(k - ks0) % NCS], (unsigned)(((k - ks0) / NCS) & 1), D.status);
      }
      __syncthreads();
      return;
    }
    __syncthreads();
    u = seg_end;
  }
  if (tid == 0) trace_record(doms[0].trace, TRACE_PAIR, t_in);
}

// Stage of an interior node read through the cache from global memory: the
// march's per-node work (scale, split-form rates, szz, point source and
// gravity, update) with the same routine, so the node gets the bits the
// march would give it.
template <int MODE, int PI_>
__device__ __forceinline__ void interior_node_global(const DevDomain& D, const DevBlock& B, int i, int j,
                                                     const StageArgs& a) {
  constexpr int NR = RDef<MODE>::NR;
  constexpr int NF = MODE == 2 ? 6 : 3;
  const long long pitch = B.pitch, plane = B.plane;
  const long long c = (long long)j * pitch + i;
  const double* __restrict__ Fin = B.F[a.in];
  const double* __restrict__ DFr = a.dfr ? B.DFalt : B.DF;
  double acc[NF];
  const bool load_df = a.scale && a.A != 0.0;
#pragma unroll
  for (int l = 0; l < NR; ++l) acc[l] = load_df ? a.A * DFr[l * plane + c] : 0.0;
  if (MODE == 2) acc[5] = 0.0;
  double Fc[NF];
#pragma unroll
  for (int l = 0; l < NF; ++l) Fc[l] = Fin[l * plane + c];
  double cf[PI_ + 1][3];
#pragma unroll
  for (int s = 1; s <= PI_; ++s)
#pragma unroll
    for (int q = 0; q < 3; ++q) cf[s][q] = B.coef[s][q];
  NodeMat m;
  m.rho = B.rho_b; m.G = B.G_b; m.M = B.M_b; m.gamma = B.gamma_b; m.nu = B.nu_b; m.rinv = 0.0;
  const double* qm[2] = {B.yr, B.xr};
  const double* rm[2] = {B.yq, B.xq};
  split_rates<MODE, PI_, false>(
      acc, m, cf, D.DI, B.Ji[c], [&](int l, int s) { return Fin[l * plane + c + s]; },
      [&](int l, int s) { return Fin[l * plane + c + (long long)s * pitch]; },
      [&](int k, int s) { return qm[k][c + s]; }, [&](int k, int s) { return rm[k][c + (long long)s * pitch]; });
  if (MODE == 2) acc[5] = m.nu * (acc[2] + acc[4]);
  if (D.src.use_gravity || (D.src.use_singular && B.src_ok)) body_forces<MODE>(D, B, i, j, stage_time(a), a, acc);
  double* __restrict__ DFw = a.dfw ? B.DFalt : B.DF;
#pragma unroll
  for (int l = 0; l < NF; ++l) DFw[l * plane + c] = acc[l];
  if (a.update) {
    double* __restrict__ Fout = B.F[a.out];
#pragma unroll
    for (int l = 0; l < NF; ++l) Fout[l * plane + c] = Fc[l] + a.Bdt * acc[l];
  }
}

// band item -> block-local node; returns the block (bands of width nbw along
// the bottom, top, left and right of every block, like closure_item)
__device__ __forceinline__ int band_item(const DevDomain& D, long long tid, int& i, int& j) {
  int sg = 0;
  while (tid >= D.bstart[sg + 1]) ++sg;
  const int b = sg >> 2, strip = sg & 3;
  const DevBlock& B = D.blk[b];
  const int w = D.nbw, nx = B.nx, ny = B.ny;
  const long long k = tid - D.bstart[sg];
  if (strip == 0) { j = (int)(k / nx); i = (int)(k % nx); }
  else if (strip == 1) { j = ny - w + (int)(k / nx); i = (int)(k % nx); }
  else if (strip == 2) { j = w + (int)(k / w); i = (int)(k % w); }
  else { j = w + (int)(k / w); i = nx - w + (int)(k % w); }
  return b;
}

// Second stage of a two-stage pass at every node within nbst + PI of a block
// edge: the closure nodes as closure_kernel does them (after the stage's
// interface solve), the rest as the march does them.
template <int MODE, int PI_>
__global__ void __launch_bounds__(128) band_kernel(const __grid_constant__ DevDomain D, StageArgs a) {
  const unsigned long long t_in = (threadIdx.x == 0 && D.trace.rec) ? globaltimer_ns() : 0ull;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid < D.bstart[4 * D.nblocks]) {
    int i, j;
    const int b = band_item(D, tid, i, j);
    const DevBlock& B = D.blk[b];
    if (edge_distance(i, j, B.nx, B.ny) < D.nbst) closure_node<MODE, PI_, false, true>(D, B, i, j, a, -1, nullptr);
    else interior_node_global<MODE, PI_>(D, B, i, j, a);
  }
  if (threadIdx.x == 0) trace_record(D.trace, TRACE_BAND, t_in);
}

// Bands of a batch of independent instances in one launch.
template <int MODE, int PI_>
__global__ void __launch_bounds__(128)
    band_kernel_batch(const DevDomain* __restrict__ doms, const int* __restrict__ cta_begin, int ninst, StageArgs a) {
  const int k = batch_instance(cta_begin, ninst, blockIdx.x);
  const DevDomain& D = doms[k];
  const long long tid = (long long)(blockIdx.x - cta_begin[k]) * blockDim.x + threadIdx.x;
  if (tid >= D.bstart[4 * D.nblocks]) return;
  int i, j;
  const int b = band_item(D, tid, i, j);
  const DevBlock& B = D.blk[b];
  if (edge_distance(i, j, B.nx, B.ny) < D.nbst) closure_node<MODE, PI_, false, true>(D, B, i, j, a, -1, nullptr);
  else interior_node_global<MODE, PI_>(D, B, i, j, a);
}

}  // namespace fdmap
