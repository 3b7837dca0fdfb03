/*
 * fdmap_oracle.h -- CPU restatement of FDMAP's explicit time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle the GPU engine is
 * checked against, and the timed CPU baseline of bench.py.  Nothing in the
 * product (fdmap_github_b200/) links, imports or calls it.
 *
 * It restates, routine by routine and in the same floating-point evaluation
 * order, FDMAP's time_step_LS (time_step.f90:71-167) and everything it calls
 * for the elastic + interface configurations: scale/update of rates
 * (fields.f90:1061-1242), prepare_edges (domain.f90:420-439, 1325-1346),
 * boundary conditions (boundaries.f90:74-377), locked and frictional
 * interfaces (interfaces.f90:520-1012), friction (friction.f90:555-1506),
 * SAT penalties (time_step.f90:754-851), SBP rates (rates.f90:8-936,
 * rates_heterogeneous.f90:8-917) and point sources (source.f90:147-406).
 *
 * Parity status: the reference (Fortran 90 + MPI) cannot be compiled or run
 * in this environment and ships no golden vectors or test fixtures, so this
 * restatement is "parity unpinned" against reference outputs.  It is pinned
 * instead against known answers that follow from the reference's own
 * definitions: SBP identities of the literal coefficient tables, exactness of
 * the operators on low-order polynomials, manufactured-solution convergence,
 * discrete energy decay, Newton residuals below the reference's atolR, and
 * closed-form characteristic boundary solutions.
 */
#ifndef FDMAP_ORACLE_H
#define FDMAP_ORACLE_H

#include "../include/fdmap_desc.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_domain oracle_domain;

/* Deep-copies the descriptor.  Returns NULL on invalid input. */
oracle_domain* oracle_create(const fdmap_desc* d);
void oracle_destroy(oracle_domain* o);

/* enforce_edge_conditions(D, 0d0) at time t, as init_domain does
 * (domain.f90:346-356): sets Fhat, initial slip velocity, Nreg. */
int oracle_init_edges(oracle_domain* o, double t);

/* One time_step_LS call at time t0 with step dt (time_step.f90:71-167). */
int oracle_time_step(oracle_domain* o, double t0, double dt, int final_step);

/* main.f90 time loop for n = n_first..n_last: t = t_start + (n-1)*dt,
 * final step when n == nt. */
int oracle_run(oracle_domain* o, double t_start, double dt, int n_first, int n_last, int nt);

/* (nx,ny,nF) body fields and rates; either pointer may be NULL. */
int oracle_get_fields(const oracle_domain* o, double* F, double* DF);
int oracle_set_fields(oracle_domain* o, const double* F, const double* DF);

/* Fault field `field` (FDMAP_FAULT_* in fdmap_gpu.h order) of interface iface. */
int oracle_get_fault(const oracle_domain* o, int iface, int field, double* out);

/* Hat variables of side s (0..3) of block b: (n, nF). */
int oracle_get_fhat(const oracle_domain* o, int b, int s, double* out);

/* Body displacement U, DU (nx, ny, nU) and peak motion pgv, pga (nx, ny);
 * any pointer may be NULL; -1 when the domain does not track them. */
int oracle_get_body_extras(const oracle_domain* o, double* U, double* DU, double* pgv, double* pga);

/* Mechanical energy E[nblocks + 1] (every block, then the sum) of the last
 * stage 1 with energy_balance = T; -1 when the domain does not track it. */
int oracle_get_energy(const oracle_domain* o, double* E);

/* Boundary displacement U and rate DU of side s (0..3) of block b: (n, nU) each. */
int oracle_get_side_u(const oracle_domain* o, int b, int s, double* U, double* DU);

/* PML field Wx (which = 0) or Wy (which = 1), (nx, ny, nF); zeros where none. */
int oracle_get_pml(const oracle_domain* o, int which, double* out);

/* Number of Newton failures seen so far (the reference warns and retries
 * from the failed iterate, friction.f90:789-790). */
long long oracle_newton_failures(const oracle_domain* o);

/* Number of solves whose retry failed as well (the reference stops there,
 * friction.f90:1014). */
long long oracle_newton_stops(const oracle_domain* o);

/* Newton residual tolerance as a multiple of the reference's atolR = 1e4*eps
 * (friction.f90:931).  A test runs the oracle at another multiple to measure
 * how far the result moves within the solver's own tolerance. */
int oracle_set_newton_tolerance(oracle_domain* o, double scale);

/* Iteration limit of every Newton solve (the reference's imax = 99,
 * friction.f90:924).  A test lowers it to force failures on the host. */
int oracle_set_newton_limit(oracle_domain* o, int imax);

/* With tap on, every step keeps the 18 fault fields as they stand at the
 * reference's output point (stage 1, after the interface solve and the
 * rates, before the update; time_step.f90:129); read them back per field. */
int oracle_set_tap(oracle_domain* o, int on);
int oracle_get_fault_tap(const oracle_domain* o, int iface, int field, double* out);

/* Setters for resuming from a checkpoint: a fault field, a side's boundary
 * displacement U, DU (n, nU), the body displacement U, DU (nx, ny, nU) and
 * peak motion pgv, pga (nx, ny), the PML field Wx (which = 0) or Wy (1). */
int oracle_set_fault(oracle_domain* o, int iface, int field, const double* in);
int oracle_set_side_u(oracle_domain* o, int b, int s, const double* U, const double* DU);
int oracle_set_body_extras(oracle_domain* o, const double* U, const double* DU, const double* pgv,
                           const double* pga);
int oracle_set_pml(oracle_domain* o, int which, const double* in);

/* Block-aligned partition (the reference's exchange_edge between processes,
 * mpi_routines2d.f90:168-208): owned[b] != 0 for the blocks this rank steps;
 * the others are filled with NaN.  Every stage (and the initial edge solve),
 * after the edge values are gathered, `fn(user, exchange_number)` runs; it
 * reads this rank's side of every interface cut by the partition
 * (oracle_get_iface_edge, side 0 = minus, 1 = plus; [l*n + k]) and writes
 * the peer's side (oracle_set_iface_edge), and returns 0. */
int oracle_set_owned(oracle_domain* o, const int* owned);
int oracle_set_exchange(oracle_domain* o, int (*fn)(void*, long long), void* user);
int oracle_get_iface_edge(oracle_domain* o, int iface, int side, double* out);
int oracle_set_iface_edge(oracle_domain* o, int iface, int side, const double* in);

/* Number of OpenMP threads the oracle uses (1 when built without OpenMP),
 * and a cap on it (n > 0). */
int oracle_num_threads(void);
void oracle_set_num_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
