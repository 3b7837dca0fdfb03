/*
 * fdmap_host.h -- host-side domain initialisation.
 *
 * In a production FDMAP run the Fortran driver performs init_domain
 * (domain.f90:45-378) itself and passes the resulting arrays to the GPU engine
 * through fdmap_desc.  This library ships a C++ restatement of that
 * initialisation so that FDMAP's own namelist input files (the `.in` format read
 * by main.f90:29-78 and the per-block/per-interface lists) can drive the GPU
 * engine without the Fortran toolchain.  It reads:
 *   problem_list, domain_list, and per '!---BLOCKn---' grid_list,
 *   boundaries_list, material_list, fields_list, operator_list; per
 *   '!---IFACEn---' interface_list, friction_list, thermpres_list; source_list;
 * plus the binary side files FDMAP reads (curve files, heterogeneous medium,
 * friction / stress / state files), all real*8 in native byte order.
 */
#ifndef FDMAP_HOST_H
#define FDMAP_HOST_H

#include "fdmap_desc.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fdmap_domain fdmap_domain; /* owns every array the descriptor points to */

/* Parse `input_text` (contents of an FDMAP .in file) and initialise the domain.
 * Relative file names inside the input are resolved against `base_dir`
 * (may be NULL = current directory).  Replaces init_domain + the time-loop
 * setup of main.f90:57-116.  Returns FDMAP_OK or a negative FDMAP_ERR_*;
 * fdmap_host_last_error() then describes the failure. */
int fdmap_host_init(const char* input_text, const char* base_dir, fdmap_domain** out);

/* Flags of fdmap_host_init_ex. */
enum { FDMAP_INIT_BODY_ON_DEVICE = 1 };

/* As fdmap_host_init.  With FDMAP_INIT_BODY_ON_DEVICE the host does only the
 * O(nx + ny) part of init_domain (input, edge curves, side initial fields and
 * normals, interfaces and friction, the source search) and leaves the
 * O(nx * ny) body -- transfinite grid and metrics (grid.f90:391-618), initial
 * fields (fields.f90:774-897), side impedances (domain.f90:1349-1459) -- to
 * the engine, which builds it on the device from fdmap_desc.body.  dt, CFL,
 * hmin and hmax stay NaN (nt 0) until fdmap_host_set_spacing. */
int fdmap_host_init_ex(const char* input_text, const char* base_dir, int flags, fdmap_domain** out);

/* Finish set_dt (domain.f90:1462-1535) of a domain initialised with
 * FDMAP_INIT_BODY_ON_DEVICE from the grid spacings the engine reduced
 * (fdmap_gpu_time_params): dt, CFL, nt, hmin, hmax and the CFL/dt-scaled Cdiss
 * of every block, with the arithmetic of fdmap_host_init. */
int fdmap_host_set_spacing(fdmap_domain* dom, double hmin, double hmax);

/* The descriptor of an initialised domain (owned by the domain). */
const fdmap_desc* fdmap_host_desc(const fdmap_domain* dom);

/* Mutable access for callers that seed states before handing the domain over. */
fdmap_desc* fdmap_host_desc_mut(fdmap_domain* dom);

void fdmap_host_free(fdmap_domain* dom);

/* Scalar summary for bindings without struct support:
 * ints[10] = mode, nF, nx, ny, nblocks, nifaces, nt, rk_order, fd_method, heterogeneous
 * dbls[5]  = t0, dt, CFL, hmin, hmax */
int fdmap_host_info(const fdmap_domain* dom, int* ints, double* dbls);

/* Optional body fields: flags[3] = displacement, peak, energy_balance (domain_list). */
int fdmap_host_body_flags(const fdmap_domain* dom, int* flags);

/* Number of nodes p-m+1 of interface `iface` (0-based), or a negative code. */
int fdmap_host_iface_n(const fdmap_domain* dom, int iface);

/* Interface layout: info[4] = direction (0 'x', 1 'y'), m, p (1-based global
 * indices along the interface), coupling. */
int fdmap_host_iface_info(const fdmap_domain* dom, int iface, int* info);

/* Blocks on the minus and plus side of interface `iface`: blocks[2], 0-based
 * (interface_list iblockm / iblockp, interfaces.f90:26-135). */
int fdmap_host_iface_blocks(const fdmap_domain* dom, int iface, int* blocks);

/* Interface geometry: x[n], y[n] of interface `iface` (NULL if absent). */
const double* fdmap_host_iface_xy(const fdmap_domain* dom, int iface, int which);

/* Side arrays of block `block`, side `side` (0..3 = L, R, B, T): "F0" (n, nF),
 * "M" (n, 5), "normal" (n, 2), "x" or "y" (n); *count receives the length.
 * NULL if absent. */
const double* fdmap_host_side_array(const fdmap_domain* dom, int block, int side, const char* name, long long* count);

/* Scaled artificial dissipation coefficient of block `block` (Cdiss*CFL/dt,
 * domain.f90:317-320), or a negative code for a bad index. */
double fdmap_host_block_cdiss(const fdmap_domain* dom, int block);

/* Perfectly matched layer of block `block` (pml_list, material.f90:152-222):
 * flags[2] = pmlx, pmly; params[7] = n, sigma, kappa, mx, px, my, py. */
int fdmap_host_block_pml(const fdmap_domain* dom, int block, int* flags, double* params);

/* Block index limits: lim[4] = mgx, pgx, mgy, pgy (1-based). */
int fdmap_host_block_limits(const fdmap_domain* dom, int block, int* lim);

/* Pointer to a body array owned by the domain ("F", "DF", "x", "y", "xq", "xr",
 * "yq", "yr", "J", "Ji", "rho", "cs", "cp", "G", "M", "gamma", "nu"); *count
 * receives its length.  NULL if the name is unknown or the array is absent. */
double* fdmap_host_array(fdmap_domain* dom, const char* name, long long* count);

/* Human-readable description of the last error on this thread. */
const char* fdmap_host_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* FDMAP_HOST_H */
