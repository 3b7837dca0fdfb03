// Device-side output (write_output, output.f90:990-1060, and the file layout
// of open_output_file, output.f90:916-987).
//
// Each item samples one field at every step whose index D%n (= loop index
// n - 1, main.f90:189) lies in [nmin, nmax] with (D%n - nmin) % stride == 0,
// at the reference's output point: inside stage 1, after the interface solve
// and rates, before the state update (time_step.f90:129).  Body fields are
// read from the step-start buffer; fault fields from the stage-1 snapshot the
// interface kernel writes when outputs are open.  Values are converted to
// float32 (ps = 4, mpi_routines.f90:12) by one gather launch per step into
// per-item device rings of R output steps.  Whenever an item has R/2 output
// steps not yet copied, the ring is copied to one of two pinned host buffers
// asynchronously, in stream order behind the gathers; the host writes a copy
// out (appending to <prefix>_<name>.dat, the values of each output step with
// i fastest, and <prefix>_<name>.t, D%t of each output step) when it starts
// the next copy, so the steps keep running while files are written.  Flush
// and close wait for everything.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "engine.h"
#include "fdmap_gpu.h"

namespace fdmap {

struct DevOutItem {
  int kind;            // FDMAP_OUT_FAULT, FDMAP_OUT_BODY or FDMAP_OUT_SIDE
  int index;           // interface (fault), body field component, or 4*block + side
  int ffield;          // FDMAP_FAULT_* (fault items)
  int stride;
  long long nmin, nmax;
  int size;            // values per output step
  long long elem0;     // first element in the element arrays
  long long ring0;     // first float of this item's ring
};

__global__ void output_gather_kernel(const __grid_constant__ DevDomain D, const DevOutItem* __restrict__ items, int nitems,
                                     const long long* __restrict__ elem_start, const int* __restrict__ elem_b,
                                     const long long* __restrict__ elem_off, long long nelem, const TimeState* ts,
                                     long long n_explicit, int cur, int R, float* __restrict__ ring) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nelem) return;
  int lo = 0, hi = nitems - 1;  // item holding element e
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (elem_start[mid] <= e) lo = mid;
    else hi = mid - 1;
  }
  const DevOutItem& it = items[lo];
  const long long dn = (ts ? ts->n : n_explicit) - 1;  // D%n during step n
  if (dn < it.nmin || dn > it.nmax || (dn - it.nmin) % it.stride != 0) return;
  const long long rec = (dn - it.nmin) / it.stride;
  double v;
  if (it.kind == FDMAP_OUT_FAULT) {
    const DevIface& I = D.ifc[it.index];
    v = I.fr.st_out[(long long)it.ffield * I.n + elem_off[e]];
  } else if (it.kind == FDMAP_OUT_ENERGY) {
    v = it.ffield == 0 ? D.energy[it.index] : 0.0;
  } else if (it.kind == FDMAP_OUT_SIDE) {
    const DevSide& S = D.blk[it.index >> 2].side[it.index & 3];
    v = it.ffield >= FDMAP_OUT_SIDE_U ? S.Utap[(long long)(it.ffield - FDMAP_OUT_SIDE_U) * S.n + elem_off[e]]
                                      : S.Fhat[(long long)it.ffield * S.n + elem_off[e]];
  } else {
    const DevBlock& B = D.blk[elem_b[e]];
    const int f = it.index;
    if (f < FDMAP_OUT_BODY_U) v = B.F[cur][(long long)f * B.plane + elem_off[e]];
    else if (f < FDMAP_OUT_BODY_PGV) v = B.Utap[(long long)(f - FDMAP_OUT_BODY_U) * B.plane + elem_off[e]];
    else v = (f == FDMAP_OUT_BODY_PGV ? B.pgv : B.pga)[elem_off[e]];
  }
  ring[it.ring0 + (rec % R) * it.size + (e - it.elem0)] = (float)v;
}

struct OutItemHost {
  std::string name;
  DevOutItem d{};
  std::vector<int> eb;
  std::vector<long long> eoff;
  FILE* dat = nullptr;
  FILE* tf = nullptr;
  long long issued = 0;   // output steps whose gathers are enqueued
  long long copied = 0;   // output steps covered by an enqueued ring copy
  long long drained = 0;  // output steps written to the files
  std::vector<float> times;  // D%t of the issued output steps not yet written
};

struct OutputState {
  std::vector<OutItemHost> items;
  std::string prefix;
  int R = 0;
  bool open = false;
  DevOutItem* d_items = nullptr;
  long long* d_elem_start = nullptr;
  int* d_eb = nullptr;
  long long* d_eoff = nullptr;
  float* d_ring = nullptr;
  float* h_ring[2] = {nullptr, nullptr};  // pinned copies of the ring (one in flight, one being written)
  int hbuf = 0;                            // buffer the next copy goes to
  int pbuf = 0;                            // buffer of the copy in flight
  bool pending = false;                    // a copy is in flight
  cudaEvent_t ev = nullptr;                // its completion
  long long nelem = 0, ring_floats = 0;
  std::vector<double*> snapshots;  // st_out per friction interface
  void release() {
    if (ev) cudaEventSynchronize(ev);
    cudaFree(d_items); cudaFree(d_elem_start); cudaFree(d_eb); cudaFree(d_eoff); cudaFree(d_ring);
    for (float*& hr : h_ring) {
      if (hr) cudaFreeHost(hr);
      hr = nullptr;
    }
    if (ev) cudaEventDestroy(ev);
    ev = nullptr;
    pending = false;
    for (double* p : snapshots) cudaFree(p);
    d_items = nullptr; d_elem_start = nullptr; d_eb = nullptr; d_eoff = nullptr; d_ring = nullptr;
    snapshots.clear();
    for (auto& it : items) {
      if (it.dat) fclose(it.dat);
      if (it.tf) fclose(it.tf);
      it.dat = it.tf = nullptr;
    }
  }
};

static bool active(const DevOutItem& d, long long dn) {
  return dn >= d.nmin && dn <= d.nmax && (dn - d.nmin) % d.stride == 0;
}

// append output steps [drained, copied) of every item (all issued ones when
// `all`) from host copy `hr`
static int write_records(OutputState* o, const float* hr, bool all) {
  for (auto& it : o->items) {
    const long long upto = all ? it.issued : it.copied;
    for (long long r = it.drained; r < upto; ++r) {
      const float* src = hr + it.d.ring0 + (r % o->R) * it.d.size;
      if (fwrite(src, sizeof(float), it.d.size, it.dat) != (size_t)it.d.size)
        return set_err(FDMAP_ERR_IO, "cannot write " + o->prefix + "_" + it.name + ".dat");
      const float t = it.times[(size_t)(r - it.drained)];
      if (fwrite(&t, sizeof(float), 1, it.tf) != 1)
        return set_err(FDMAP_ERR_IO, "cannot write " + o->prefix + "_" + it.name + ".t");
    }
    it.times.erase(it.times.begin(), it.times.begin() + (upto - it.drained));
    it.drained = upto;
    if (all) it.copied = upto;
  }
  return FDMAP_OK;
}

// wait for the copy in flight (if any) and write what it holds
static int finish_pending(fdmap_gpu* h) {
  OutputState* o = h->out;
  if (!o->pending) return FDMAP_OK;
  CUDA_TRY(cudaEventSynchronize(o->ev));
  o->pending = false;
  return write_records(o, o->h_ring[o->pbuf], false);
}

// start copying the ring (output steps [copied, issued) of every item) to a
// pinned buffer behind the gathers already enqueued; the previous copy is
// written out first
static int drain_async(fdmap_gpu* h) {
  OutputState* o = h->out;
  int rc = finish_pending(h);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(o->h_ring[o->hbuf], o->d_ring, o->ring_floats * sizeof(float), cudaMemcpyDeviceToHost,
                           h->stream));
  CUDA_TRY(cudaEventRecord(o->ev, h->stream));
  for (auto& it : o->items) it.copied = it.issued;
  o->pending = true;
  o->pbuf = o->hbuf;
  o->hbuf ^= 1;
  return FDMAP_OK;
}

// write every output step issued so far (flush / close)
static int drain(fdmap_gpu* h) {
  OutputState* o = h->out;
  int rc = finish_pending(h);
  if (rc) return rc;
  bool any = false;
  for (auto& it : o->items) any = any || it.issued > it.drained;
  if (any) {
    CUDA_TRY(cudaMemcpyAsync(o->h_ring[o->hbuf], o->d_ring, o->ring_floats * sizeof(float), cudaMemcpyDeviceToHost,
                             h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if ((rc = write_records(o, o->h_ring[o->hbuf], true))) return rc;
  }
  for (auto& it : o->items) {
    fflush(it.dat);
    fflush(it.tf);
  }
  return FDMAP_OK;
}

// before step n (loop index) starting at time t: start a copy once an item
// has R/2 output steps not yet copied, then count the output steps this step
// issues.  A new output step never lands on a ring slot the host has still to
// read: the copy of that slot precedes it in the stream, and the host reads a
// pinned buffer before the next copy into it is enqueued.
int output_before_step(fdmap_gpu* h, long long n, double t) {
  OutputState* o = h->out;
  if (!o || !o->open) return FDMAP_OK;
  const long long dn = n - 1;
  const long long half = std::max(1, o->R / 2);
  bool due = false;
  for (auto& it : o->items)
    if (active(it.d, dn) && it.issued - it.copied >= half) due = true;
  if (due) {
    int rc = drain_async(h);
    if (rc) return rc;
  }
  for (auto& it : o->items)
    if (active(it.d, dn)) {
      it.issued += 1;
      it.times.push_back((float)t);
    }
  return FDMAP_OK;
}

bool output_is_open(const fdmap_gpu* h) { return h->out && h->out->open; }

int output_gather(fdmap_gpu* h, const TimeState* ts, long long n, int cur) {
  OutputState* o = h->out;
  if (!o || !o->open || o->nelem == 0) return FDMAP_OK;
  const int threads = 256;
  const long long blocks = (o->nelem + threads - 1) / threads;
  output_gather_kernel<<<(unsigned)blocks, threads, 0, h->stream>>>(h->hdom, o->d_items, (int)o->items.size(),
                                                                  o->d_elem_start, o->d_eb, o->d_eoff, o->nelem, ts, n,
                                                                  cur, o->R, o->d_ring);
  h->launches++;
  CUDA_TRY(cudaGetLastError());
  return FDMAP_OK;
}

void output_destroy(fdmap_gpu* h) {
  if (!h->out) return;
  h->out->release();
  delete h->out;
  h->out = nullptr;
}

}  // namespace fdmap

using namespace fdmap;

namespace {

int invalidate_graphs(fdmap_gpu* h) {
  for (auto& ge : h->step_graph)
    if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  h->graph_dt = 0.0;
  return FDMAP_OK;
}

// set (or clear) the stage-1 fault snapshot pointers in both domain copies
int set_snapshots(fdmap_gpu* h, bool on) {
  OutputState* o = h->out;
  for (int k = 0; k < h->hdom.nifaces; ++k) {
    DevIface& I = h->hdom.ifc[k];
    if (I.coupling != FDMAP_COUPLING_FRICTION || !I.fr.st) continue;
    if (on) {
      double* p = nullptr;
      CUDA_TRY(cudaMalloc(&p, (size_t)FDMAP_FAULT_NFIELDS * I.n * sizeof(double)));
      CUDA_TRY(cudaMemset(p, 0, (size_t)FDMAP_FAULT_NFIELDS * I.n * sizeof(double)));
      o->snapshots.push_back(p);
      I.fr.st_out = p;
    } else {
      I.fr.st_out = nullptr;
    }
  }
  CUDA_TRY(cudaMemcpy(h->ddom, &h->hdom, sizeof(DevDomain), cudaMemcpyHostToDevice));
  return FDMAP_OK;
}

}  // namespace

extern "C" {

int fdmap_gpu_output_add(fdmap_gpu* h, const char* name, int kind, int index, int field, int mx, int px, int sx,
                         int my, int py, int sy, long long nmin, long long nmax, int stride) {
  if (!h || !name || !*name) return set_err(FDMAP_ERR_INVALID_ARG, "output item needs a handle and a name");
  if (h->out && h->out->open) return set_err(FDMAP_ERR_INVALID_ARG, "outputs are open: add items before opening");
  if (stride < 1 || sx < 1 || sy < 1) return set_err(FDMAP_ERR_INVALID_ARG, "strides must be positive");
  if (nmax < nmin) return set_err(FDMAP_ERR_INVALID_ARG, "empty output window");
  if (!h->out) h->out = new (std::nothrow) OutputState();
  if (!h->out) return set_err(FDMAP_ERR_NOMEM, "out of host memory");
  OutItemHost it;
  it.name = name;
  it.d.kind = kind;
  it.d.nmin = nmin;
  it.d.nmax = nmax;
  it.d.stride = stride;
  if (kind == FDMAP_OUT_FAULT) {
    if (index < 0 || index >= h->hdom.nifaces) return set_err(FDMAP_ERR_INVALID_ARG, "output: interface index out of range");
    const DevIface& I = h->hdom.ifc[index];
    if (I.coupling != FDMAP_COUPLING_FRICTION) return set_err(FDMAP_ERR_INVALID_ARG, "output: interface is not frictional");
    if (field < 0 || field >= FDMAP_FAULT_NFIELDS) return set_err(FDMAP_ERR_INVALID_ARG, "output: bad fault field");
    // mx..px: 1-based node indices along the interface (its m..p range)
    if (mx < 1 || px > I.n || mx > px) return set_err(FDMAP_ERR_INVALID_ARG, "output: fault indices out of range");
    it.d.index = index;
    it.d.ffield = field;
    for (int k = mx; k <= px; k += sx) { it.eb.push_back(0); it.eoff.push_back(k - 1); }
  } else if (kind == FDMAP_OUT_BODY) {
    const int nU = h->mode == 2 ? 2 : 1;
    const bool ok = (field >= 0 && field < h->nF) ||
                    (field >= FDMAP_OUT_BODY_U && field < FDMAP_OUT_BODY_U + nU && h->hdom.blk[0].Utap) ||
                    ((field == FDMAP_OUT_BODY_PGV || field == FDMAP_OUT_BODY_PGA) && h->hdom.blk[0].pgv);
    if (!ok) return set_err(FDMAP_ERR_INVALID_ARG, "output: bad body field (or displacement / peak not tracked)");
    if (mx < 1 || px > h->nx_g || mx > px || my < 1 || py > h->ny_g || my > py)
      return set_err(FDMAP_ERR_INVALID_ARG, "output: body indices out of range");
    it.d.index = field;
    for (int j = my; j <= py; j += sy)
      for (int i = mx; i <= px; i += sx) {
        int b = -1;
        for (int q = 0; q < (int)h->geom.size(); ++q) {
          const BlockGeom& g = h->geom[q];
          if (i >= g.mgx && i < g.mgx + g.nx && j >= g.mgy && j < g.mgy + g.ny) { b = q; break; }
        }
        if (b < 0) return set_err(FDMAP_ERR_INVALID_ARG, "output: node outside every block");
        const BlockGeom& g = h->geom[b];
        it.eb.push_back(b);
        it.eoff.push_back((long long)(j - g.mgy) * g.pitch + (i - g.mgx));
      }
  } else if (kind == FDMAP_OUT_ENERGY) {
    if (!h->d_energy) return set_err(FDMAP_ERR_INVALID_ARG, "output: the domain does not track the energy");
    if (index < -1 || index >= h->hdom.nblocks || field < 0 || field > 1)
      return set_err(FDMAP_ERR_INVALID_ARG, "output: bad energy item");
    it.d.index = index < 0 ? h->hdom.nblocks : index;
    it.d.ffield = field;
    it.eb.push_back(0);
    it.eoff.push_back(0);
  } else if (kind == FDMAP_OUT_SIDE) {
    const int b = index >> 2, s = index & 3;
    if (index < 0 || b >= h->hdom.nblocks) return set_err(FDMAP_ERR_INVALID_ARG, "output: side index out of range");
    const int nU = h->mode == 2 ? 2 : 1;
    if (field < 0 || (field >= h->nF && field < FDMAP_OUT_SIDE_U) || field >= FDMAP_OUT_SIDE_U + nU)
      return set_err(FDMAP_ERR_INVALID_ARG, "output: bad side field");
    const int n = h->hdom.blk[b].side[s].n;
    if (mx < 1 || px > n || mx > px) return set_err(FDMAP_ERR_INVALID_ARG, "output: side indices out of range");
    it.d.index = index;
    it.d.ffield = field;
    for (int k = mx; k <= px; k += sx) { it.eb.push_back(b); it.eoff.push_back(k - 1); }
  } else {
    return set_err(FDMAP_ERR_INVALID_ARG, "output: kind must be FDMAP_OUT_FAULT, FDMAP_OUT_BODY or FDMAP_OUT_SIDE");
  }
  it.d.size = (int)it.eoff.size();
  h->out->items.push_back(std::move(it));
  return FDMAP_OK;
}

int fdmap_gpu_output_open(fdmap_gpu* h, const char* prefix, int ring_steps) {
  if (!h || !prefix) return set_err(FDMAP_ERR_INVALID_ARG, "null argument");
  if (h->partitioned()) return set_err(FDMAP_ERR_UNSUPPORTED, "device-side output is not available on a partition");
  if (!h->out || h->out->items.empty()) return set_err(FDMAP_ERR_INVALID_ARG, "no output items");
  if (h->out->open) return set_err(FDMAP_ERR_INVALID_ARG, "outputs already open");
  if (ring_steps < 1) return set_err(FDMAP_ERR_INVALID_ARG, "ring must hold at least one step");
  CUDA_TRY(cudaSetDevice(h->device));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  OutputState* o = h->out;
  o->prefix = prefix;
  o->R = ring_steps;
  std::vector<DevOutItem> di;
  std::vector<long long> start;
  std::vector<int> eb;
  std::vector<long long> eoff;
  long long ring = 0;
  for (auto& it : o->items) {
    it.d.elem0 = (long long)eoff.size();
    it.d.ring0 = ring;
    start.push_back(it.d.elem0);
    eb.insert(eb.end(), it.eb.begin(), it.eb.end());
    eoff.insert(eoff.end(), it.eoff.begin(), it.eoff.end());
    ring += (long long)o->R * it.d.size;
    di.push_back(it.d);
    it.issued = it.copied = it.drained = 0;
    it.times.clear();
    const std::string base = o->prefix + "_" + it.name;
    it.dat = fopen((base + ".dat").c_str(), "wb");
    it.tf = fopen((base + ".t").c_str(), "wb");
    if (!it.dat || !it.tf) {
      o->release();
      return set_err(FDMAP_ERR_IO, "cannot open " + base + ".dat / .t");
    }
  }
  o->nelem = (long long)eoff.size();
  o->ring_floats = ring;
  auto fail = [&](cudaError_t e) {
    o->release();
    return set_err(FDMAP_ERR_CUDA, std::string("output buffers: ") + cudaGetErrorString(e));
  };
  cudaError_t e;
  if ((e = cudaMalloc(&o->d_items, di.size() * sizeof(DevOutItem))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&o->d_elem_start, start.size() * sizeof(long long))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&o->d_eb, std::max<size_t>(eb.size(), 1) * sizeof(int))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&o->d_eoff, std::max<size_t>(eoff.size(), 1) * sizeof(long long))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&o->d_ring, std::max<long long>(ring, 1) * sizeof(float))) != cudaSuccess) return fail(e);
  for (float*& hr : o->h_ring)
    if ((e = cudaMallocHost(&hr, std::max<long long>(ring, 1) * sizeof(float))) != cudaSuccess) return fail(e);
  if ((e = cudaEventCreateWithFlags(&o->ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  o->hbuf = 0;
  o->pending = false;
  if ((e = cudaMemcpy(o->d_items, di.data(), di.size() * sizeof(DevOutItem), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(o->d_elem_start, start.data(), start.size() * sizeof(long long), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(o->d_eb, eb.data(), eb.size() * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(o->d_eoff, eoff.data(), eoff.size() * sizeof(long long), cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail(e);
  int rc = set_snapshots(h, true);
  if (rc) {
    set_snapshots(h, false);
    o->release();
    return rc;
  }
  o->open = true;
  h->out_next_n = 1;
  return invalidate_graphs(h);
}

int fdmap_gpu_output_flush(fdmap_gpu* h) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  if (!h->out || !h->out->open) return FDMAP_OK;
  CUDA_TRY(cudaSetDevice(h->device));
  return drain(h);
}

int fdmap_gpu_output_close(fdmap_gpu* h) {
  if (!h) return set_err(FDMAP_ERR_INVALID_ARG, "null handle");
  if (!h->out) return FDMAP_OK;
  CUDA_TRY(cudaSetDevice(h->device));
  int rc = h->out->open ? drain(h) : FDMAP_OK;
  int rc2 = h->out->open ? set_snapshots(h, false) : FDMAP_OK;
  invalidate_graphs(h);
  output_destroy(h);
  return rc ? rc : rc2;
}

}  // extern "C"
