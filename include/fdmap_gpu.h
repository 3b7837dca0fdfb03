/*
 * fdmap_gpu.h -- C ABI of the B200 time-stepping engine for FDMAP.
 *
 * Drop-in boundary: a Fortran driver that has run init_domain keeps its time
 * loop (main.f90:168-231) and replaces the body of time_step_LS
 * (time_step.f90:96-165: scale_rates_all, prepare_edges,
 * enforce_edge_conditions, set_rates_all, update_fields_all, exchange_fields)
 * by one call per step.  Plain C types only; fortran/fdmap_gpu_mod.f90 holds
 * the matching bind(C) interfaces.
 *
 * Conventions
 *  - every entry point returns FDMAP_OK (0) or a negative FDMAP_ERR_* code; the
 *    library never aborts or traps (the reference's error() -> MPI_Abort and
 *    Newton double failure -> stop become error codes);
 *  - host arrays are only borrowed for the duration of a call; all state lives
 *    on the device, owned by the handle;
 *  - one handle per host thread; step calls are asynchronous on the handle's
 *    stream, fdmap_gpu_get_* and fdmap_gpu_synchronize block.
 */
#ifndef FDMAP_GPU_H
#define FDMAP_GPU_H

#include "fdmap_desc.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fdmap_gpu fdmap_gpu;

/* Copies the domain to device `device` and, when `init_edges` is non-zero,
 * runs enforce_edge_conditions(D, 0) at d->t0 as init_domain does
 * (domain.f90:346-356): initial hat variables, slip velocity and Nreg.
 * Replaces: the device-resident half of init_domain (domain.f90:45-378). */
int fdmap_gpu_create(const fdmap_desc* d, int device, int init_edges, fdmap_gpu** h);

/* enforce_edge_conditions(D, 0d0) at time t (domain.f90:442-471 with dt = 0). */
int fdmap_gpu_init_edges(fdmap_gpu* h, double t);

/* One low-storage RK step from t0 (time_step_LS, time_step.f90:71-167).
 * final_step != 0 evaluates stage-1 rates and fault solve only, as the
 * reference does on its last loop index (time_step.f90:133). */
int fdmap_gpu_time_step(fdmap_gpu* h, double t0, double dt, int final_step);

/* The main-loop body for n = n_first..n_last: t = t_start + (n-1)*dt, final
 * step when n == nt (main.f90:168-187).  Steps are issued as CUDA graphs. */
int fdmap_gpu_run(fdmap_gpu* h, double t_start, double dt, int n_first, int n_last, int nt);

int fdmap_gpu_synchronize(fdmap_gpu* h);

/* Issue all subsequent work on `stream` (a cudaStream_t of the same device,
 * e.g. the caller's framework stream); NULL restores the handle's own stream. */
int fdmap_gpu_set_stream(fdmap_gpu* h, void* stream);

/* Per-kernel timing: when enabled, CUDA events bracket every launch on the
 * handle's stream.  fdmap_gpu_profile_read fills ms[3] / count[3] with the
 * summed milliseconds and launch counts since enabling: [0] the interior
 * stencil kernel, [1] the boundary-closure kernel, [2] the interface kernel. */
int fdmap_gpu_profile(fdmap_gpu* h, int enable);
int fdmap_gpu_profile_read(fdmap_gpu* h, double* ms, long long* count);
/* The same for up to n (<= 5) kernel kinds: [0..2] as above, [3] the
 * two-stage interior pass, [4] the band kernel of its second stage. */
int fdmap_gpu_profile_read_kinds(fdmap_gpu* h, int n, double* ms, long long* count);

/* Body fields F(nx,ny,nF) and rates DF(nx,ny,nF) in FDMAP's global
 * column-major layout; either pointer may be NULL.  Blocks the host. */
int fdmap_gpu_get_fields(fdmap_gpu* h, double* F, double* DF);
int fdmap_gpu_set_fields(fdmap_gpu* h, const double* F, const double* DF);

/* One FDMAP_FAULT_* field of interface `iface` (0-based), p-m+1 values. */
int fdmap_gpu_get_fault(fdmap_gpu* h, int iface, int field, double* out);
int fdmap_gpu_set_fault(fdmap_gpu* h, int iface, int field, const double* in);

/* Hat variables Fhat(n,nF) of side s (0..3 = L,R,B,T) of block b. */
int fdmap_gpu_get_fhat(fdmap_gpu* h, int b, int s, double* out);

/* Time-loop parameters params[5] = t0, dt, CFL, hmin, hmax and nt.  For a
 * descriptor with fdmap_desc.body these are the engine's own: hmin and hmax
 * reduced over the grid it built on the device, dt, CFL and nt finished from
 * them as set_dt does (domain.f90:1462-1535); hand hmin, hmax to
 * fdmap_host_set_spacing to finish the host domain identically.  Otherwise
 * they are the descriptor's. */
int fdmap_gpu_time_params(fdmap_gpu* h, double* params, int* nt);

/* One metric plane in the global (nx,ny) layout (grid.f90:465-618): the
 * metric terms as the engine holds them, whether uploaded or built on the
 * device.  FDMAP_METRIC_J exists for dissipative blocks only. */
enum { FDMAP_METRIC_XQ = 0, FDMAP_METRIC_XR = 1, FDMAP_METRIC_YQ = 2, FDMAP_METRIC_YR = 3, FDMAP_METRIC_JI = 4,
       FDMAP_METRIC_J = 5 };
int fdmap_gpu_get_metric(fdmap_gpu* h, int which, double* out);

/* Perfectly matched layer fields (F%Wx, F%Wy, fields.f90:35, 203-210):
 * which = 0 Wx, 1 Wy, in the global (nx,ny,nF) layout; zeros in blocks
 * without that layer.  set writes the blocks that have it (resume). */
int fdmap_gpu_get_pml(fdmap_gpu* h, int which, double* out);
int fdmap_gpu_set_pml(fdmap_gpu* h, int which, const double* in);

/* Mechanical energy E[nblocks + 1] of every block and their sum as of the
 * last stage 1 (BF%Etot, F%Etot; domain_list energy_balance = T); 1e40
 * before the first step, as the reference initialises it. */
int fdmap_gpu_get_energy(fdmap_gpu* h, double* E);

/* Body displacement U(nx,ny,nU) and its rate DU (F%U, F%DU; domain_list
 * displacement = T) and peak ground velocity / acceleration pgv, pga (nx,ny;
 * peak = T), global layout; any pointer may be NULL.  FDMAP_ERR_INVALID_ARG
 * when the domain does not track them. */
int fdmap_gpu_get_displacement(fdmap_gpu* h, double* U, double* DU);
int fdmap_gpu_set_displacement(fdmap_gpu* h, const double* U, const double* DU);
int fdmap_gpu_get_peak(fdmap_gpu* h, double* pgv, double* pga);
int fdmap_gpu_set_peak(fdmap_gpu* h, const double* pgv, const double* pga);

/* Boundary displacement U(n,nU) and its rate DU(n,nU) of side s (0..3 =
 * L,R,B,T) of block b (bndF%U, bndF%DU; nU = 2 in mode II, 1 in mode III):
 * integrated from the side's hat velocities every stage as the reference
 * does (scale_rates_boundary / set_rates_boundary / update_fields_boundary,
 * fields.f90:1083-1276).  Either pointer may be NULL. */
int fdmap_gpu_get_side_displacement(fdmap_gpu* h, int b, int s, double* U, double* DU);
int fdmap_gpu_set_side_displacement(fdmap_gpu* h, int b, int s, const double* U, const double* DU);

/* Edge impedances M(n,5) = Zs, Zp, gamma, Ks, Kp of side s (0..3 = L,R,B,T)
 * of block b as the engine holds them (init_edges, domain.f90:1349-1459). */
int fdmap_gpu_get_side_impedance(fdmap_gpu* h, int b, int s, double* out);

/* Device status.  *newton_failures: friction solves whose first Newton
 * attempt failed so far (the reference warns and retries from the failed
 * iterate, friction.f90:789-790, 1012-1036).  Returns FDMAP_ERR_TIMEOUT if a
 * bounded device wait (a TMA pipeline barrier) gave up, else
 * FDMAP_ERR_NEWTON_NOCONV if some retry failed as well (where the reference
 * calls stop, friction.f90:1014), else FDMAP_OK. */
int fdmap_gpu_status(fdmap_gpu* h, long long* newton_failures);

/* counts[0]: first-attempt Newton failures, counts[1]: retries that failed
 * too.  Return value as fdmap_gpu_status. */
int fdmap_gpu_newton_counts(fdmap_gpu* h, long long* counts);

/* Resets the status words (failure counts, timeout flag) to zero. */
int fdmap_gpu_clear_status(fdmap_gpu* h);

/* Tile shape of the interior march kernel: 0 = 128 columns x 4 rows per row
 * group, 1 = 128 x 2 with deep prefetch rings, 2 = 64 x 4, 3 = 128 x 2 with
 * shallow rings and two CTAs per SM.  The engine starts with the first shape
 * whose shared-memory rings fit the domain's variant (a heterogeneous mode II
 * medium or the extras of dissipation, PML, forcing and body displacement
 * need the smaller rings).  set_tile returns FDMAP_ERR_UNSUPPORTED for a
 * shape that cannot serve the domain; get_tile fills any non-NULL pointer
 * with the shape and its width / rows. */
int fdmap_gpu_set_tile(fdmap_gpu* h, int tile);
int fdmap_gpu_get_tile(fdmap_gpu* h, int* tile, int* mw, int* mr);

/* Autotuner of a single domain: times `steps` steps (CUDA graphs, best of two
 * repetitions) with every tile shape the domain can take -- and, where the
 * domain can take two-stage passes (fdmap_gpu_set_pairs), with the passes on
 * and off -- keeps the fastest and returns its tile (best_tile, best_ms per
 * step; either may be NULL; fdmap_gpu_get_pairs tells whether the passes were
 * kept).  The whole device state is copied before and put back after, so
 * tuning does not advance the run.  Call it before opening outputs. */
int fdmap_gpu_tune(fdmap_gpu* h, double dt, int steps, int* best_tile, double* best_ms);

/* Two-stage passes (no routine of the reference: an execution schedule of
 * time_step_LS, time_step.f90:96-165).  Stages (1,2), (3,4), ... of a step
 * run as one interior pass over HBM each, with the boundary work of both
 * stages beside it and the second stage near the block edges after it; the
 * arithmetic of every node is the stage-by-stage arithmetic, so results are
 * bit-identical either way.  Available for homogeneous blocks without
 * dissipation, PML, forcing, displacement, peak motion or energy tracking,
 * SBP2 or SBP4, unpartitioned, and on by default there (FDMAP_PAIRS=0 turns
 * it off at creation).  set_pairs returns FDMAP_ERR_UNSUPPORTED when asked to
 * enable them on a domain that cannot take them; get_pairs returns 1 (in
 * use), 0 (not in use) or a negative error code. */
int fdmap_gpu_set_pairs(fdmap_gpu* h, int enable);
int fdmap_gpu_get_pairs(fdmap_gpu* h);

/* Iteration limit of every Newton solve, 1..99 (the reference's parameter
 * imax = 99, friction.f90:924, is the default).  A driver or test lowers it
 * to provoke solver failures on purpose (fault injection from the host). */
int fdmap_gpu_set_newton_limit(fdmap_gpu* h, int imax);

/* Self-test of the bounded device wait: launches one CTA that waits on an
 * mbarrier nothing will complete, for at most limit_s seconds (0 < limit_s
 * <= 10).  Afterwards fdmap_gpu_status reports FDMAP_ERR_TIMEOUT, exactly as
 * after a TMA pipeline wait that gave up; the context stays usable.  No
 * reference counterpart. */
int fdmap_gpu_test_wait_timeout(fdmap_gpu* h, double limit_s);

/* Counts the non-finite values (NaN, +-Inf) in the current body fields of
 * every block and in the slip rate, shear stress and state of every
 * frictional interface, on the device; FDMAP_ERR_NONFINITE if there are any.
 * count may be NULL. */
int fdmap_gpu_check_finite(fdmap_gpu* h, long long* count);

/* ------------------------------------------------------------------------
 * Device-side output (write_output, output.f90:990-1060).  An item samples
 * one field at each step whose index D%n (= n-1 for loop index n) lies in
 * [nmin, nmax] with (D%n - nmin) % stride == 0, at the reference's output
 * point (stage 1 after the interface solve, before the update,
 * time_step.f90:129).  Values are gathered on the device into float32 rings
 * of `ring_steps` output steps; the host appends them to
 * <prefix>_<name>.dat (i fastest) and D%t to <prefix>_<name>.t, as
 * open_output_file names and lays out its files (output.f90:916-987).
 *   FDMAP_OUT_FAULT: `index` = interface, `field` = FDMAP_FAULT_*,
 *                    nodes mx..px (1-based along the interface) step sx;
 *   FDMAP_OUT_BODY:  `field` = body field component (0..nF-1), or
 *                    FDMAP_OUT_BODY_U + c (displacement component c),
 *                    FDMAP_OUT_BODY_PGV / _PGA (peak motion), global
 *                    nodes mx..px step sx by my..py step sy;
 *   FDMAP_OUT_SIDE:  `index` = 4*block + side (0..3 = L,R,B,T), `field` =
 *                    hat variable component 0..nF-1 or FDMAP_OUT_SIDE_U + c
 *                    for the boundary displacement component c (the bndX
 *                    locations, get_field, domain.f90:763-860), side nodes
 *                    mx..px (1-based along the side) step sx;
 *   FDMAP_OUT_ENERGY: `index` = block (0-based) or -1 for the sum over
 *                    blocks, `field` = 0 for the mechanical energy Etot, 1
 *                    for the dissipated energies and their rates (E, EL..ET,
 *                    DE, DEL..DET), which stay zero because the reference's
 *                    boundary energy flux is a stub (energy.f90:219-236);
 *                    one value per output step (Ebody / Eblock locations).
 * Items are added before fdmap_gpu_output_open; fdmap_gpu_output_flush
 * writes everything recorded so far, fdmap_gpu_output_close flushes and
 * releases the rings. */
enum { FDMAP_OUT_FAULT = 0, FDMAP_OUT_BODY = 1, FDMAP_OUT_SIDE = 2, FDMAP_OUT_ENERGY = 3, FDMAP_OUT_SIDE_U = 8,
       FDMAP_OUT_BODY_U = 16, FDMAP_OUT_BODY_PGV = 24, FDMAP_OUT_BODY_PGA = 25 };
int fdmap_gpu_output_add(fdmap_gpu* h, const char* name, int kind, int index, int field, int mx, int px, int sx,
                         int my, int py, int sy, long long nmin, long long nmax, int stride);
int fdmap_gpu_output_open(fdmap_gpu* h, const char* prefix, int ring_steps);
int fdmap_gpu_output_flush(fdmap_gpu* h);
int fdmap_gpu_output_close(fdmap_gpu* h);

/* max |field| over the nodes of interface `iface` (a friction interface),
 * reduced on the device into *out.  No counterpart in the reference (its
 * drivers scan the Fortran arrays).  Allocates nothing during the call: for
 * drivers that check the fault every step and cannot allocate inside their
 * time loop.  Its scratch is a static device array shared by all handles of a
 * device, so calls on one device must not overlap; faults longer than
 * 1,048,576 nodes are rejected (FDMAP_ERR_UNSUPPORTED).  A NaN anywhere in
 * the field gives NaN.  The first call on a device looks up that scratch and
 * should come before any stream capture. */
int fdmap_gpu_fault_max_noalloc(fdmap_gpu* h, int iface, int field, double* out);

/* ------------------------------------------------------------------------
 * Block-aligned partition over several GPUs.  Replaces the reference's
 * exchange of interface edge rows between processes (exchange_edge,
 * mpi_routines2d.f90:168-208, called from domain.f90:1179-1322): each GPU
 * holds and steps the blocks it owns; an interface whose two sides live on
 * different GPUs is solved on both, redundantly and identically, from the
 * local side's edge values and the peer's, which arrive every stage.  Blocks
 * never share grid nodes, so no halo rows are exchanged.
 *
 * fdmap_gpu_create_part: owned[b] != 0 for the blocks this GPU steps.  The
 * other blocks' body arrays are not allocated.  No initial edge solve is run
 * (it needs the peers' values): call fdmap_gpu_init_edges (callback) or
 * fdmap_gpu_group_init_edges (group) once every partition exists.
 * Outputs, energy balance, forcing files and a body built on the device are
 * refused (FDMAP_ERR_UNSUPPORTED) on a partition.
 * ---------------------------------------------------------------------- */
int fdmap_gpu_create_part(const fdmap_desc* d, int device, const int* owned, fdmap_gpu** h);

/* Interfaces with exactly one side on this GPU (written to ifaces[0..max)); returns their count. */
int fdmap_gpu_part_interfaces(fdmap_gpu* h, int* ifaces, int max);

/* Device buffers of interface `iface` for exchange number `stage`: *send
 * holds this GPU's side's edge values, *recv receives the peer's, both
 * count = nF * (p - m + 1) doubles laid out [l*n + k] (field l, interface
 * node k). */
int fdmap_gpu_part_buffers(fdmap_gpu* h, int iface, long long stage, double** send, double** recv,
                           long long* count);

/* Exchange callback, called by the host once per stage (and by
 * fdmap_gpu_init_edges) after this GPU's edge values have been packed into
 * the send buffers, with the exchange number and the cudaStream_t on which
 * the interface solve of the stage follows.  It queues (on that stream, or
 * otherwise completes before returning) the transfer of every send buffer to
 * the peer and of the peer's values into the receive buffers -- NCCL
 * ncclSend / ncclRecv in a group, MPI, or a device copy -- and returns 0. */
typedef int (*fdmap_exchange_fn)(void* user, long long stage, void* stream);
int fdmap_gpu_set_exchange(fdmap_gpu* h, fdmap_exchange_fn fn, void* user);

/* The partitions of one domain driven by one host thread (one handle per
 * GPU, or several on one GPU): every stage, after all of them have packed
 * their edge values, each copies its peers' values peer to peer on its
 * boundary stream and finishes the stage. */
int fdmap_gpu_group_init_edges(fdmap_gpu* const* hs, int n, double t);
int fdmap_gpu_group_time_step(fdmap_gpu* const* hs, int n, double t0, double dt, int final_step);
int fdmap_gpu_group_run(fdmap_gpu* const* hs, int n, double t_start, double dt, int n_first, int n_last, int nt);

/* Kernel timeline: with capacity > 0 every CTA of the stage kernels
 * (interior march, closure, interface) appends one record of three words --
 * kind (1 march, 2 closure, 3 interface) | SM << 8 | CTA << 16, start and end
 * in ns of the device's global timer -- until `capacity` records are taken;
 * 0 switches it off and keeps the records taken.  Enabling clears them.
 * fdmap_gpu_trace_read
 * copies up to `max` records and returns how many were taken.  No reference
 * counterpart (the reference times whole steps, main.f90:202-253). */
int fdmap_gpu_trace(fdmap_gpu* h, int capacity);
int fdmap_gpu_trace_read(fdmap_gpu* h, unsigned long long* records, int max);

/* Kernel launches issued by the last fdmap_gpu_run / time_step call. */
long long fdmap_gpu_launch_count(fdmap_gpu* h);

/* Device bytes held by the handle. */
long long fdmap_gpu_device_bytes(fdmap_gpu* h);

void fdmap_gpu_destroy(fdmap_gpu* h);

const char* fdmap_gpu_strerror(int code);

/* Last CUDA / validation message on this thread. */
const char* fdmap_gpu_last_error(void);

/* ------------------------------------------------------------------------
 * Batched ensemble: `ninst` independent domains (uneven grid sizes, their own
 * prestress and friction state) advanced together, each stage one launch per
 * kernel kind for all instances, each step a replayed CUDA graph.  The
 * reference runs such an ensemble as separate main.f90 jobs, one per input
 * file; there is no single reference routine this replaces.  Instances must
 * share mode, FD method, RK order and material kind (homogeneous mode II or
 * any mode III) and step with one dt.  Every instance reproduces its plain
 * single-domain run bit for bit.
 * ---------------------------------------------------------------------- */
typedef struct fdmap_ensemble fdmap_ensemble;

/* descs[k]: descriptor of instance k (as for fdmap_gpu_create). */
int fdmap_gpu_ensemble_create(const fdmap_desc* const* descs, int ninst, int device, int init_edges,
                              fdmap_ensemble** e);
int fdmap_gpu_ensemble_size(fdmap_ensemble* e);

/* Handle of instance k for fdmap_gpu_get_* / set_* / status (ordered after
 * the ensemble's work).  Owned by the ensemble; stepping it on its own is an
 * error for the next ensemble step. */
int fdmap_gpu_ensemble_instance(fdmap_ensemble* e, int k, fdmap_gpu** h);

/* As fdmap_gpu_time_step / fdmap_gpu_run, for every instance at once. */
int fdmap_gpu_ensemble_time_step(fdmap_ensemble* e, double t0, double dt, int final_step);
int fdmap_gpu_ensemble_run(fdmap_ensemble* e, double t_start, double dt, int n_first, int n_last, int nt);
int fdmap_gpu_ensemble_synchronize(fdmap_ensemble* e);

/* Launch shape: shape[0] closure-kernel block size (64, 128, 256),
 * shape[1] interface-kernel block size (32, 64, 128), shape[2] 1 = boundary
 * kernels run beside the interior march, 0 = serialised. */
int fdmap_gpu_ensemble_set_shape(fdmap_ensemble* e, const int* shape);
int fdmap_gpu_ensemble_get_shape(fdmap_ensemble* e, int* shape);

/* Autotuner: times `steps` replayed steps of every march tile shape the
 * instances can take, then, on the fastest tile, of every launch shape;
 * applies the fastest and returns it (best_shape[3], best_ms per step;
 * either may be NULL; the tile through fdmap_gpu_ensemble_get_tile).  The
 * ensemble's state is restored afterwards. */
int fdmap_gpu_ensemble_tune(fdmap_ensemble* e, double dt, int steps, int* best_shape, double* best_ms);

/* Two-stage interior passes for every instance (as fdmap_gpu_set_pairs): on
 * by default when every instance can take them; results are bit-identical
 * either way.  get_pairs returns 1, 0 or a negative code. */
int fdmap_gpu_ensemble_set_pairs(fdmap_ensemble* e, int enable);
int fdmap_gpu_ensemble_get_pairs(fdmap_ensemble* e);

/* March tile shape of every instance (as fdmap_gpu_set_tile, 0..3); the
 * autotuner picks it first. */
int fdmap_gpu_ensemble_set_tile(fdmap_ensemble* e, int tile);
int fdmap_gpu_ensemble_get_tile(fdmap_ensemble* e, int* tile);

long long fdmap_gpu_ensemble_launch_count(fdmap_ensemble* e);
void fdmap_gpu_ensemble_destroy(fdmap_ensemble* e);

/* ------------------------------------------------------------------------
 * Forward/backward pair: gradient of the receiver misfit
 *   J = 1/2 sum_{n=1..nt} sum_r (vz(x_r, t_n) - data[n-1][r])^2
 * (vz sampled at every step start, where the reference writes its output,
 * time_step.f90:129) with respect to the density rho(x) and shear modulus
 * G(x) of a heterogeneous mode III domain (absorbing / free / rigid sides,
 * blocks coupled by locked or rate-and-state interfaces) and to the shear
 * prestress S0 of every fault node.  The forward pass is fdmap_gpu_time_step
 * itself; the backward pass is the discrete adjoint of those LS-RK stages
 * (SBP-SAT rates, the edge impedances Zs = rho*cs, Ks = cs*H00i*|grad|/J with
 * cs = sqrt(G/rho), and the interface solve of interfaces.f90:676-1012 /
 * friction.f90:593-828 with its Newton root differentiated implicitly and the
 * state variable's own RK adjoint), with the fields and fault registers
 * checkpointed every `checkpoint_every` steps and each segment recomputed
 * once, or kept resident (fdmap_gpu_adjoint_set_store_budget).  Slip-weakening, forced rupture and regularised normal stress are
 * refused (FDMAP_ERR_UNSUPPORTED).  The reference has no adjoint; there is no
 * routine this replaces.
 * ---------------------------------------------------------------------- */
typedef struct fdmap_adjoint fdmap_adjoint;

/* rec_i, rec_j: 1-based global node indices of the nrec receivers. */
int fdmap_gpu_adjoint_create(const fdmap_desc* d, int device, int nrec, const int* rec_i, const int* rec_j,
                             int checkpoint_every, fdmap_adjoint** a);

/* Replace the material by rho(nx,ny), G(nx,ny) (global layout); the edge
 * impedances follow.  The point source keeps the block density, as in
 * set_source (source.f90:147-252). */
int fdmap_gpu_adjoint_set_material(fdmap_adjoint* a, const double* rho, const double* G);

/* Steps 1..nt-1 from the initial state given at creation.  traces (nt*nrec,
 * sample-major) receives vz at the receivers; with data (nt*nrec) the misfit
 * is returned and the residuals are kept for fdmap_gpu_adjoint_backward.
 * Either pointer may be NULL. */
int fdmap_gpu_adjoint_forward(fdmap_adjoint* a, double t_start, double dt, int nt, const double* data, double* traces,
                              double* misfit);

/* dJ/drho and dJ/dG in the global (nx,ny) layout (either may be NULL). */
int fdmap_gpu_adjoint_backward(fdmap_adjoint* a, double* grad_rho, double* grad_G);

/* Body fields F(nx,ny,3) after the last forward pass. */
int fdmap_gpu_adjoint_fields(fdmap_adjoint* a, double* F);

/* Time parameters of the adjoint's domain, as fdmap_gpu_time_params (with
 * the body built on the device, the spacings the device reduced). */
int fdmap_gpu_adjoint_time_params(fdmap_adjoint* a, double* params, int* nt);

/* Fault nodes of all interfaces, concatenated in interface order: the length
 * of the prestress arrays below (nodes of locked interfaces read as 0). */
int fdmap_gpu_adjoint_fault_size(const fdmap_adjoint* a);

/* Background shear stress of the fault nodes (friction_list stress_file S0,
 * load_stress, friction.f90:1317-1374): set and read back. */
int fdmap_gpu_adjoint_set_prestress(fdmap_adjoint* a, const double* S0);
int fdmap_gpu_adjoint_get_prestress(fdmap_adjoint* a, double* S0);

/* dJ/dS0 per fault node from the last fdmap_gpu_adjoint_backward. */
int fdmap_gpu_adjoint_prestress_gradient(fdmap_adjoint* a, double* grad_S0);

/* Device memory (bytes) a forward pass with data may keep stage inputs in:
 * the stage inputs of its last R segments (checkpoint intervals) stay
 * resident, and the backward pass reverses those without recomputing them.
 * R = the segments that fit in the budget and in the free device memory less
 * 2 GiB, all of them or else one fewer than fit (a further segment store
 * holds the recomputed ones).  0 (the default): every segment is recomputed;
 * a negative budget: all free device memory.  Gradients do not depend on it
 * (the stored inputs are the recomputed ones bit for bit).  The store is
 * sized at the next forward pass with data; changing the material or the
 * prestress drops the resident segments. */
int fdmap_gpu_adjoint_set_store_budget(fdmap_adjoint* a, long long bytes);

/* Bytes of one segment's stage store (checkpoint_every * stages slots). */
long long fdmap_gpu_adjoint_segment_bytes(const fdmap_adjoint* a);

/* Resident segments of the last forward pass with data (0 when none). */
int fdmap_gpu_adjoint_resident_segments(const fdmap_adjoint* a);

void fdmap_gpu_adjoint_destroy(fdmap_adjoint* a);

#ifdef __cplusplus
}
#endif

#endif /* FDMAP_GPU_H */
