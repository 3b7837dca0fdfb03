// Persistent "march" stage kernel: the same per-node work as stencil_kernel
// (fused scale + SAT + SBP rates + szz + sources + RK update), organised for
// HBM streaming on sm_100a.
//
// Work: every block is cut into strips of MW columns; the strip-rows of all
// blocks form one sequence of row groups (MR rows) that is split into equal
// contiguous ranges, one per resident CTA (grid = SMs x CTAs per SM), so
// every CTA streams the same amount of data and consecutive CTAs hold
// vertically adjacent rows (their halo rows are shared through L2).  The tile
// MW x MR is a template parameter (128 x 4, 128 x 2 with deep rings, 64 x 4,
// 128 x 2 with shallow rings and two CTAs per SM), chosen per domain by the
// host or the autotuner; one CTA has MW x MR threads.
//
// Data movement: each row group arrives through 3-D tiled TMA boxes
// (cp.async.bulk.tensor.3d ... mbarrier::complete_tx, no multicast) issued by
// one thread ahead of use, into two shared-memory rings with one mbarrier per
// slot:
//  - the neighbour ring (NGS slots: groups g-1, g, g+1 resident, the next
//    ones in flight) holds what the stencil reads at neighbours: the rate fields and
//    yr, xr with PI halo columns ({WH, MR, NR} and {WH, MR, 2} boxes), and
//    yq, xq, Ji ({MW, MR, 3});
//  - the centre ring (NCS slots) holds what only the node itself reads:
//    DF (skipped in a stage whose A is 0), szz and heterogeneous material.
// Neighbours along i come from a slot's halo columns, neighbours along j from
// the adjacent slots.  Boxes past the block edges are zero-filled by TMA.
// Every wait is bounded in time; a CTA whose wait gives up stops computing,
// drains its copies in flight and leaves (status word -> FDMAP_ERR_TIMEOUT).
#pragma once

#include <cuda.h>

#include <type_traits>

#include "stencil_kernel.cuh"

namespace fdmap {

// Tile shapes of the march: strip width MW (columns) x rows per row group MR.
// The host picks one per domain (the first whose rings fit in shared memory,
// or the autotuner's choice); the unit decomposition and the tensor-map boxes
// follow it.
constexpr int MARCH_SHAPES = 4;
__host__ __device__ constexpr int shape_mw(int sh) { return sh == 2 ? 64 : 128; }
__host__ __device__ constexpr int shape_mr(int sh) { return (sh == 1 || sh == 3) ? 2 : 4; }
// Ring depths: the neighbour ring holds groups g-1, g, g+1 and prefetches
// the rest; the centre ring holds group g and prefetches the rest.  Shape 1
// (2-row groups) gets deeper rings, so about as many rows are in flight per
// CTA as with 4-row groups; shape 3 (also 2-row groups) keeps the shallow
// rings, small enough for two CTAs per SM.
__host__ __device__ constexpr int shape_ngs(int sh) { return sh == 1 ? 6 : 4; }
__host__ __device__ constexpr int shape_ncs(int sh) { return sh == 1 ? 3 : 2; }

__host__ __device__ constexpr int even_halo(int h) { return (h + 1) & ~1; }
__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) / 128 * 128; }

// EXT: 0 the plain variant; 1 the variant for artificial dissipation (a J
// plane with halo columns in every neighbour slot), source forcing, body
// displacement and peak motion; 2 the variant for a perfectly matched layer
// (with forcing and body extras).  Forcing, displacement, peak motion and the
// PML's auxiliary fields are node-local: read and written by the node's own
// thread.
enum { MARCH_PLAIN = 0, MARCH_DISS = 1, MARCH_PML = 2 };

template <int MODE, int PI_, bool HET, int EXT, int SH>
struct MarchLayout {
  static constexpr int MW = shape_mw(SH);
  static constexpr int MR = shape_mr(SH);
  static constexpr int THREADS = MW * MR;
  static constexpr int NGS = shape_ngs(SH);
  static constexpr int NCS = shape_ncs(SH);
  static constexpr int NR = RDef<MODE>::NR;
  static constexpr int HP = even_halo(PI_);
  static constexpr int WH = MW + 2 * HP;                       // halo row length (doubles)
  static constexpr int NH = HET ? (MODE == 2 ? 5 : 2) : 0;     // heterogeneous material planes
  // neighbour group slot: rate fields [NR][MR][WH], yr,xr [2][MR][WH], yq,xq,Ji [3][MR][MW], (EXT) J [MR][WH]
  static constexpr size_t F_OFF = 0;
  static constexpr size_t MH_OFF = align128(F_OFF + (size_t)NR * MR * WH * 8);
  static constexpr size_t MC_OFF = align128(MH_OFF + (size_t)2 * MR * WH * 8);
  static constexpr size_t J_OFF = align128(MC_OFF + (size_t)3 * MR * MW * 8);
  static constexpr size_t GSLOT = align128(J_OFF + (EXT == MARCH_DISS ? (size_t)MR * WH * 8 : 0));
  // centre group slot: DF [NR][MR][MW], szz [1][MR][MW] (mode II), material [NH][MR][MW]
  static constexpr size_t DF_OFF = 0;
  static constexpr size_t F6_OFF = align128(DF_OFF + (size_t)NR * MR * MW * 8);
  static constexpr size_t HT_OFF = align128(F6_OFF + (MODE == 2 ? (size_t)MR * MW * 8 : 0));
  static constexpr size_t CSLOT = align128(HT_OFF + (size_t)NH * MR * MW * 8);
  static constexpr size_t BARS_OFF = NGS * GSLOT + NCS * CSLOT;
  static constexpr size_t BYTES = BARS_OFF + (NGS + NCS) * 8 + 128;  // + alignment slack
  static constexpr unsigned NB_BYTES = (unsigned)(((size_t)(NR + 2) * WH + 3 * MW) * MR * 8);
  static constexpr unsigned J_BYTES = (unsigned)((size_t)MR * WH * 8);
};

struct MarchPlan {
  int grid;          // CTAs launched
  long long units;   // total row groups over all strips of all blocks (of all instances)
  // batched instances: per-instance tensor maps in device memory and the
  // prefix of march units over instances; ninst == 1 uses the by-value maps
  const TmapSet* tms;
  const long long* unit_begin;
  int ninst;
};

// Interface node k of interface I, then the whole stage for the two edge nodes
// it couples (minus side, plus side), using the hat variables just solved.
template <int MODE, int PI_, bool HET>
__device__ __forceinline__ void iface_item(const DevDomain& D, const DevIface& I, int k, const StageArgs& a) {
  double Fhm[6], Fhp[6];
  d_iface_node<MODE>(D, I, k, a, Fhm, Fhp);
  const DevBlock& Bm = D.blk[I.im];
  const DevBlock& Bp = D.blk[I.ip];
  const int sm = I.direction == 0 ? 1 : 3, sp = I.direction == 0 ? 0 : 2;
  int im_, jm_, ip_, jp_;
  side_node_local(sm, I.offm + k, Bm.nx, Bm.ny, im_, jm_);
  side_node_local(sp, I.offp + k, Bp.nx, Bp.ny, ip_, jp_);
  closure_node<MODE, PI_, HET>(D, Bm, im_, jm_, a, sm, Fhm);
  closure_node<MODE, PI_, HET>(D, Bp, ip_, jp_, a, sp, Fhp);
}

template <int MODE, int PI_, bool HET>
__device__ __forceinline__ void closure_work(const DevDomain& D, long long it, const StageArgs& a) {
  int i, j;
  const int b = closure_item(D, it, i, j);
  const DevBlock& B = D.blk[b];
  if (on_interface_side(B, i, j)) return;  // done by the interface item of that node
  closure_node<MODE, PI_, HET>(D, B, i, j, a, -1, nullptr);
}

// Boundary kernel: one thread per interface node (solve + its two edge nodes),
// then one thread per remaining node of the SBP closure strips.  No item
// depends on another, and none depends on the interior kernel of the stage.
template <int MODE, int PI_, bool HET>
__global__ void __launch_bounds__(128) boundary_kernel(const __grid_constant__ DevDomain D, StageArgs a) {
  const long long nif = D.seg_start[D.nseg];
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid < nif) {
    int sg = 0;
    while (tid >= D.seg_start[sg + 1]) ++sg;
    iface_item<MODE, PI_, HET>(D, D.ifc[D.seg_a[sg]], (int)(tid - D.seg_start[sg]), a);
  } else if (tid - nif < D.cstart[4 * D.nblocks]) {
    closure_work<MODE, PI_, HET>(D, tid - nif, a);
  }
}


// ---------------------------------------------------------------------------
// PTX helpers: mbarrier and 1-D bulk copy global -> shared
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 3-D tiled TMA load (no multicast) of one box into shared memory
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Longest a TMA pipeline wait may take before the kernel gives up (a normal
// row-group delivery takes microseconds).
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

// Bounded wait on the phase `parity` of an mbarrier: polls until the phase
// completes or `limit_ns` of %globaltimer time has passed.  On giving up it
// records the event in status[1] (bit 1, read back as FDMAP_ERR_TIMEOUT) and
// returns false; the caller then stops using the slot's data.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, unsigned long long* status,
                                                  unsigned long long limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
#pragma unroll 1
    for (int k = 0; k < 32; ++k)
      if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer_ns() - t0 > limit_ns) break;
  }
  atomicOr(&status[1], 2ull);
  return false;
}


// A row index given at run time or as a compile-time constant
__device__ __forceinline__ int row_value(int r) { return r; }
template <int V>
__device__ __forceinline__ constexpr int row_value(std::integral_constant<int, V>) { return V; }

// Row-group unit u -> (block, strip, first row) for tiles of MW x MR
struct UnitPos {
  int b, sx, j0;
};

template <int MR_>
__device__ __forceinline__ UnitPos unit_pos(const DevDomain& D, long long u) {
  UnitPos p{0, 0, 0};
  int b = 0;
  while (b + 1 < D.nblocks && u >= D.blk[b + 1].march_unit_begin) ++b;
  const DevBlock& B = D.blk[b];
  long long local = u - B.march_unit_begin;
  int groups = (B.ny + MR_ - 1) / MR_;
  p.b = b;
  p.sx = (int)(local / groups);
  p.j0 = (int)(local % groups) * MR_;
  return p;
}

// Register budget of the march kernel: 96 per thread (48K of the SM's 64K for
// a 512-thread CTA) leaves room for one boundary CTA beside it, so the
// edge and closure kernels of the same stage run concurrently with the
// interior march.  The SBP6 mode II variant and the extras variant of a
// 256-thread shape take more to avoid spills.
template <int MODE, int PI_, int EXT, int SH>
constexpr int march_regs() {
  return ((MODE == 2 && PI_ == 3) || (EXT && shape_mw(SH) * shape_mr(SH) <= 256)) ? 128 : 96;
}

template <int MODE, int PI_, bool HET, int EXT, int SH>
__global__ void __maxnreg__((march_regs<MODE, PI_, EXT, SH>()))
    march_kernel(const DevDomain* __restrict__ doms, StageArgs a, MarchPlan plan, const __grid_constant__ TmapSet tm) {
  using L = MarchLayout<MODE, PI_, HET, EXT, SH>;
  using RD = RDef<MODE>;
  constexpr int MW = L::MW, MR = L::MR;
  constexpr int NR = RD::NR;
  constexpr int NF = MODE == 2 ? 6 : 3;
  constexpr int HP = L::HP;
  constexpr int WH = L::WH;
  constexpr int NGS = L::NGS, NCS = L::NCS;
  extern __shared__ unsigned char smem_dyn[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  unsigned long long* nbar = reinterpret_cast<unsigned long long*>(smem + L::BARS_OFF);
  unsigned long long* cbar = nbar + NGS;

  const int tid = threadIdx.x;
  const int cx = tid % MW, ry = tid / MW;
  const unsigned long long t_in = (tid == 0 && doms[0].trace.rec) ? globaltimer_ns() : 0ull;
  const long long ubeg = plan.units * blockIdx.x / gridDim.x;
  const long long uend = plan.units * (blockIdx.x + 1) / gridDim.x;
  const bool load_df = a.scale && a.A != 0.0;  // A = 0 (first stage): A*DF = 0, DF is not read

  const unsigned cbytes = (unsigned)((load_df ? (size_t)NR * MR * MW * 8 : 0) + (MODE == 2 ? (size_t)MR * MW * 8 : 0) +
                                     (size_t)L::NH * MR * MW * 8);

  long long u = ubeg;
  while (u < uend) {
    // instance owning unit u (the last one whose first unit is <= u)
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
    const TmapSet& tmi = plan.tms ? plan.tms[inst] : tm;
    // segment: consecutive row groups of one strip
    const UnitPos p0 = unit_pos<MR>(D, u - base);
    const int b = p0.b;
    const DevBlock& B = D.blk[b];
    const int groups = (B.ny + MR - 1) / MR;
    const long long strip_end = base + B.march_unit_begin + (long long)(p0.sx + 1) * groups;
    const long long seg_end = uend < strip_end ? uend : strip_end;
    const int jr0 = p0.j0;
    const int jr1 = min(B.ny, (int)(jr0 + (seg_end - u) * MR));
    const int i0 = p0.sx * MW;
    const int nx = B.nx, ny = B.ny;
    const long long pitch = B.pitch, plane = B.plane;
    const int ngroups = (jr1 - jr0 + MR - 1) / MR;
    // neighbour groups needed: k = gmin .. gmax (group k holds rows jr0 + k*MR ..)
    const int gmin = jr0 >= MR ? -1 : 0;
    const int gmax = ngroups - 1 + (jr1 < ny ? 1 : 0);
    const CUtensorMap* mF = &tmi.F[b][a.in];
    const CUtensorMap* mF6 = &tmi.F6[b][a.in];
    // artificial dissipation of this block: J with halo columns in the neighbour ring
    const bool diss = EXT == MARCH_DISS && B.Cdiss > 0.0;
    const unsigned nbytes = L::NB_BYTES + (diss ? L::J_BYTES : 0u);

    if (tid == 0) {
      for (int s = 0; s < NGS + NCS; ++s) mbar_init(&nbar[s], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    int nb_next = gmin, c_next = 0;  // next neighbour / centre group to be filled (thread 0)
    auto fill_nb = [&](int k) {  // neighbour group k -> slot (k - gmin) % NGS
      nb_next = k + 1;
      const int sl = (k - gmin) % NGS;
      unsigned char* g = smem + (size_t)sl * L::GSLOT;
      const int row = jr0 + k * MR;
      mbar_arrive_tx(&nbar[sl], nbytes);
      tma_load_3d(g + L::F_OFF, mF, i0 - HP, row, 0, &nbar[sl]);
      tma_load_3d(g + L::MH_OFF, &tmi.MH[b], i0 - HP, row, 0, &nbar[sl]);
      tma_load_3d(g + L::MC_OFF, &tmi.MC[b], i0, row, 2, &nbar[sl]);
      if (diss) tma_load_3d(g + L::J_OFF, &tmi.JH[b], i0 - HP, row, 0, &nbar[sl]);
    };
    auto fill_c = [&](int k) {  // centre group k -> slot k % NCS
      c_next = k + 1;
      const int sl = k % NCS;
      unsigned char* g = smem + (size_t)NGS * L::GSLOT + (size_t)sl * L::CSLOT;
      const int row = jr0 + k * MR;
      mbar_arrive_tx(&cbar[sl], cbytes);
      if (load_df) tma_load_3d(g + L::DF_OFF, &tmi.DF[b], i0, row, 0, &cbar[sl]);
      if (MODE == 2) tma_load_3d(g + L::F6_OFF, mF6, i0, row, 5, &cbar[sl]);
      if (HET) tma_load_3d(g + L::HT_OFF, &tmi.HT[b], i0, row, 0, &cbar[sl]);
    };
    if (tid == 0) {
      fence_proxy_async();
      for (int k = gmin; k <= min(gmax, gmin + NGS - 1); ++k) fill_nb(k);
      for (int k = 0; k < min(ngroups, NCS); ++k) fill_c(k);
    }

    // per-CTA constants for the interior fast path
    double cf[PI_ + 1][3];
#pragma unroll
    for (int s = 1; s <= PI_; ++s)
#pragma unroll
      for (int q = 0; q < 3; ++q) cf[s][q] = B.coef[s][q];
    const double rho_b = B.rho_b, G_b = B.G_b, M_b = B.M_b, gamma_b = B.gamma_b, nu_b = B.nu_b;
    double* __restrict__ DFp = B.DF;
    double* __restrict__ Fout = B.F[a.out];

    const int nbst = D.nbst;
    // body forces of this block (point source / gravity; with EXT also the
    // long-wave forcing and forcing from file), evaluated once per segment
    const bool forces = D.src.use_gravity || (D.src.use_singular && B.src_ok) ||
                        (EXT != MARCH_PLAIN && (D.src.use_singular || B.gforce || B.frc_new));
    const double t_stage = forces ? stage_time(a) : 0.0;
    const int i = i0 + cx;
    PmlSeg pseg{};
    if constexpr (EXT == MARCH_PML && MODE == 2) {
      if (B.pml) pseg = pml_segment<PI_>(D, B);
    }
    int aborted_at = -1;
    // ring slots of neighbour group g-1 and centre group g, advanced with g
    // (a group outside the CTA's range maps to some slot: no node that is
    // computed reads it)
    int gi = ((-1 - gmin) % NGS + NGS) % NGS;
    int ci = 0;
    for (int g = 0; g < ngroups; ++g) {
      // wait for groups g-1, g, g+1 (neighbours; all of them on the first
      // iteration, then the new one) and centre group g; neighbour group k
      // lives in slot (k - gmin) % NGS as that slot's fill (k - gmin) / NGS
      bool ok = true;
      for (int k = (g == 0 ? max(gmin, g - 1) : g + 1); k <= min(gmax, g + 1); ++k)
        ok = mbar_wait_bounded(&nbar[(k - gmin) % NGS], (unsigned)(((k - gmin) / NGS) & 1), D.status) && ok;
      ok = mbar_wait_bounded(&cbar[ci], (unsigned)((g / NCS) & 1), D.status) && ok;
      // a wait that gave up anywhere in the CTA: no compute or store from
      // these slots, no further copies; the CTA drains and leaves
      if (__syncthreads_or(!ok)) {
        aborted_at = g;
        break;
      }
      // every thread has left iteration g-1: neighbour group g-2 and centre
      // group g-1 are no longer needed; their slots take g-2+NGS and g-1+NCS
      if (tid == 0) {
        fence_proxy_async();
        if (g - 2 >= gmin && g - 2 + NGS <= gmax) fill_nb(g - 2 + NGS);
        if (g >= 1 && g - 1 + NCS < ngroups) fill_c(g - 1 + NCS);
      }
      const int j = jr0 + g * MR + ry;
      // this iteration's neighbour slots, groups g-1, g, g+1
      const unsigned char* gq[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) gq[q] = smem + (size_t)(gi + q >= NGS ? gi + q - NGS : gi + q) * L::GSLOT;
      const unsigned char* cslot = smem + (size_t)NGS * L::GSLOT + (size_t)ci * L::CSLOT;
      gi = gi + 1 == NGS ? 0 : gi + 1;
      ci = ci + 1 == NCS ? 0 : ci + 1;
      // the node's work with its row in the group as a compile-time constant
      // (ry is warp-uniform), so that every ring address is a slot pointer
      // plus a constant
      auto node = [&](auto ryc) {
        const int RY = row_value(ryc);  // a compile-time constant, or the thread's row (PML variant)
        const long long c = (long long)j * pitch + i;
        // row j lives in group g, row RY; rows j +- s in group g + (RY +- s) div MR
        auto nrow = [&](int dr, size_t off, int q, int width) -> const double* {
          const int rr = RY + dr;
          const int go = rr >= 0 ? rr / MR : -((MR - 1 - rr) / MR);
          const int r = rr - go * MR;
          return reinterpret_cast<const double*>(gq[1 + go] + off) + ((size_t)q * MR + r) * width;
        };
        const int ry = RY;
        double acc[NF];
        if (load_df) {
          const double* dfc = reinterpret_cast<const double*>(cslot + L::DF_OFF) + (size_t)ry * MW + cx;
#pragma unroll
          for (int l = 0; l < NR; ++l) acc[l] = a.A * dfc[(size_t)l * MR * MW];
        } else {
#pragma unroll
          for (int l = 0; l < NR; ++l) acc[l] = 0.0;
        }
        if (MODE == 2) acc[5] = 0.0;  // DF6 is overwritten by rates_szz below
        double Fc[NF];
#pragma unroll
        for (int l = 0; l < NR; ++l) Fc[l] = nrow(0, L::F_OFF, l, WH)[cx + HP];
        if (MODE == 2) Fc[5] = reinterpret_cast<const double*>(cslot + L::F6_OFF)[(size_t)ry * MW + cx];
        const double Ji = nrow(0, L::MC_OFF, 2, MW)[cx];
        NodeMat m;
        if (HET) {
          const double* ht = reinterpret_cast<const double*>(cslot + L::HT_OFF) + (size_t)ry * MW + cx;
          m.rho = ht[0]; m.G = ht[(size_t)MR * MW];
          if (MODE == 2) { m.M = ht[(size_t)2 * MR * MW]; m.gamma = ht[(size_t)3 * MR * MW]; m.nu = ht[(size_t)4 * MR * MW]; }
          else { m.M = 0.0; m.gamma = 0.0; m.nu = 0.0; }
        } else {
          m.rho = rho_b; m.G = G_b; m.M = M_b; m.gamma = gamma_b; m.nu = nu_b;
        }
        m.rinv = HET ? 1.0 / m.rho : 0.0;
        bool pml = false;
        if constexpr (EXT == MARCH_PML && MODE == 2) {
          if (B.pml) {
            // Cartesian PML rates of the interior region (rates.f90:2089-2126)
            // from the ring; szz at the neighbours through the cache
            const double* Fin = B.F[a.in];
            march_pml_interior<PI_>(pseg, B, c, a, acc, [&](int l, int dq, int dr) -> double {
              if (l == 5) return Fin[5 * plane + c + dq + (long long)dr * pitch];
              return dr == 0 ? nrow(0, L::F_OFF, l, WH)[cx + HP + dq] : nrow(dr, L::F_OFF, l, WH)[cx + HP];
            });
            pml = true;
          }
        }
        if (!pml && !diss) {
          split_rates<MODE, PI_, HET>(
              acc, m, cf, D.DI, Ji,
              [&](int l, int s) { return nrow(0, L::F_OFF, l, WH)[cx + HP + s]; },
              [&](int l, int s) { return nrow(s, L::F_OFF, l, WH)[cx + HP]; },
              [&](int k, int s) { return nrow(0, L::MH_OFF, k, WH)[cx + HP + s]; },
              [&](int k, int s) { return nrow(s, L::MC_OFF, k, MW)[cx]; });
        }
        if (EXT == MARCH_DISS && !pml && diss) {
          // split-form rates and artificial dissipation together
          // (rates_dissipation_interior_mode2/3, rates.f90:939-999,
          // 1397-1482): the neighbour values of every field are read from the
          // ring once per s and serve both; the dissipation sum is
          // 2*AI(0)*F + sum_s AI(s)*Ji*(J F at the four neighbours at distance
          // s), added after the rates, in the tiled kernel's order
          const double Cd = B.Cdiss;
          double dsum[NR];
#pragma unroll
          for (int l = 0; l < NR; ++l) dsum[l] = 2.0 * D.AI[0] * Cd * nrow(0, L::F_OFF, l, WH)[cx + HP];
          const double* hy = nrow(0, L::MH_OFF, 0, WH) + cx + HP;
          const double* hx = nrow(0, L::MH_OFF, 1, WH) + cx + HP;
          const double* jr = nrow(0, L::J_OFF, 0, WH) + cx + HP;
          const double yrc = hy[0], xrc = hx[0];
          const double yqc = nrow(0, L::MC_OFF, 0, MW)[cx], xqc = nrow(0, L::MC_OFF, 1, MW)[cx];
#pragma unroll
          for (int s = 1; s <= PI_; ++s) {
            const double Yrp = 0.5 * (hy[s] + yrc), Xrp = 0.5 * (hx[s] + xrc);
            const double Yrm = 0.5 * (hy[-s] + yrc), Xrm = 0.5 * (hx[-s] + xrc);
            const double Yqp = 0.5 * (nrow(s, L::MC_OFF, 0, MW)[cx] + yqc), Xqp = 0.5 * (nrow(s, L::MC_OFF, 1, MW)[cx] + xqc);
            const double Yqm = 0.5 * (nrow(-s, L::MC_OFF, 0, MW)[cx] + yqc), Xqm = 0.5 * (nrow(-s, L::MC_OFF, 1, MW)[cx] + xqc);
            double fqp[NR], fqm[NR], frp[NR], frm[NR];
#pragma unroll
            for (int l = 0; l < NR; ++l) {
              const double* fr = nrow(0, L::F_OFF, l, WH) + cx + HP;
              fqp[l] = fr[s];
              fqm[l] = fr[-s];
              frp[l] = nrow(s, L::F_OFF, l, WH)[cx + HP];
              frm[l] = nrow(-s, L::F_OFF, l, WH)[cx + HP];
            }
            const double w = HET ? D.DI[s] : 0.0;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
              double sum = 0.0;
              if (RD::fa(r) >= 0) {
                const int f = RD::fa(r);
                double t = Yrp * fqp[f] - Yrm * fqm[f] - Yqp * frp[f] + Yqm * frm[f];
                if (RD::ga(r)) t *= m.gamma;
                sum += t;
              }
              if (RD::fb(r) >= 0) {
                const int f = RD::fb(r);
                double t = -Xrp * fqp[f] + Xrm * fqm[f] + Xqp * frp[f] - Xqm * frm[f];
                if (RD::gb(r)) t *= m.gamma;
                sum += t;
              }
              const double cfr = HET ? mat_coef(m, RD::coef(r), w) : cf[s][RD::coef(r)];
              acc[r] += sum * cfr * Ji;
            }
            const double jqp = jr[s], jqm = jr[-s];
            const double jrp = nrow(s, L::J_OFF, 0, WH)[cx + HP], jrm = nrow(-s, L::J_OFF, 0, WH)[cx + HP];
#pragma unroll
            for (int l = 0; l < NR; ++l)
              dsum[l] += D.AI[s] * Cd * Ji * (jqp * fqp[l] + jqm * fqm[l] + jrp * frp[l] + jrm * frm[l]);
          }
#pragma unroll
          for (int l = 0; l < NR; ++l) acc[l] += dsum[l];
        }
        if (MODE == 2) acc[5] = m.nu * (acc[2] + acc[4]);
        if (forces) body_forces<MODE>(D, B, i, j, t_stage, a, acc);
        if (EXT != MARCH_PLAIN) body_extras<MODE>(B, c, Fc, acc, a);
#pragma unroll
        for (int l = 0; l < NF; ++l) DFp[l * plane + c] = acc[l];
        if (a.update) {
#pragma unroll
          for (int l = 0; l < NF; ++l) Fout[l * plane + c] = Fc[l] + a.Bdt * acc[l];
        }
      };
      if (j < jr1 && i >= nbst && i <= nx - 1 - nbst && j >= nbst && j <= ny - 1 - nbst) {
        if constexpr (EXT == MARCH_PML) {
          node(ry);  // one body: the PML variant is large, and copies per row strain the instruction cache
        } else if constexpr (MR == 2) {
          if (ry == 0) node(std::integral_constant<int, 0>{});
          else node(std::integral_constant<int, 1>{});
        } else {
          static_assert(MR == 4, "row groups of 2 or 4 rows");
          if (ry == 0) node(std::integral_constant<int, 0>{});
          else if (ry == 1) node(std::integral_constant<int, 1>{});
          else if (ry == 2) node(std::integral_constant<int, 2>{});
          else node(std::integral_constant<int, 3>{});
        }
      }
    }
    if (aborted_at >= 0) {
      // wait (bounded again) for every copy this CTA may still have in
      // flight into its shared memory, then end the CTA
      if (tid == 0) {
        const int g = aborted_at;
        for (int k = max(gmin, g - 1); k < nb_next; ++k)
          mbar_wait_bounded(&nbar[(k - gmin) % NGS], (unsigned)(((k - gmin) / NGS) & 1), D.status);
        for (int k = g; k < c_next; ++k) mbar_wait_bounded(&cbar[k % NCS], (unsigned)((k / NCS) & 1), D.status);
      }
      __syncthreads();
      return;
    }
    __syncthreads();
    u = seg_end;
  }
  if (tid == 0) trace_record(doms[0].trace, TRACE_MARCH, t_in);
}

}  // namespace fdmap
