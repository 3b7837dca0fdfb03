/*
 * fdmap_desc.h -- plain-C description of an FDMAP domain as it stands after
 * FDMAP's host-side initialisation (init_domain, domain.f90:45-378).
 *
 * This is the data a Fortran driver already holds when it enters the time loop
 * (main.f90:168-231).  It is handed, by pointer, to the time-stepping engines
 * (fdmap_gpu_* in fdmap_gpu.h, and the CPU oracle used by the tests).  Every
 * struct is ISO_C_BINDING compatible: ints, doubles and pointers only.
 *
 * Layout conventions (the reference's own, see fields.f90:5-43, grid.f90:26-29):
 *   - global body arrays are Fortran column-major over the single-process index
 *     space 1..nx, 1..ny (no ghost layers): A(i,j) lives at A[(i-1) + nx*(j-1)],
 *     multi-field arrays F(i,j,l) at F[(i-1) + nx*(j-1) + nx*ny*(l-1)];
 *   - side arrays of a block are indexed along the side: for L/R sides by
 *     j = mgy..pgy, for B/T sides by i = mgx..pgx; a side array M(k,c) with
 *     n = number of side nodes lives at M[k + n*c] (k = 0..n-1, c = 0..);
 *   - interface arrays are indexed by the global index m..p along the interface
 *     (n = p-m+1), same column-major convention.
 * Units are FDMAP's: km, s, m/s, MPa, g/cm^3, km/s.
 */
#ifndef FDMAP_DESC_H
#define FDMAP_DESC_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes returned by every entry point (no abort or trap inside) */
enum {
  FDMAP_OK = 0,
  FDMAP_ERR_INVALID_ARG = -1,
  FDMAP_ERR_CUDA = -2,
  FDMAP_ERR_NONFINITE = -3,
  FDMAP_ERR_NEWTON_NOCONV = -4,
  FDMAP_ERR_TIMEOUT = -5,
  FDMAP_ERR_UNSUPPORTED = -6,
  FDMAP_ERR_IO = -7,
  FDMAP_ERR_NOMEM = -8
};

/* summation-by-parts operators (fd_coeff.f90:51-71) */
enum { FDMAP_SBP2 = 2, FDMAP_SBP4 = 4, FDMAP_SBP6 = 6 };

/* outer boundary conditions (boundaries.f90:155-377) */
enum {
  FDMAP_BC_NONE = 0,
  FDMAP_BC_ABSORBING = 1,
  FDMAP_BC_FREE = 2,
  FDMAP_BC_RIGID = 3,
  FDMAP_BC_ABSORBING_0 = 4, /* '-0' variants: initial fields not subtracted */
  FDMAP_BC_FREE_0 = 5,
  FDMAP_BC_RIGID_0 = 6,
  FDMAP_BC_ABSORBING_VELOCITY = 7,
  FDMAP_BC_FREE_VELOCITY = 8
};

/* interface coupling (interfaces.f90:541-647) */
enum { FDMAP_COUPLING_LOCKED = 0, FDMAP_COUPLING_FRICTION = 1 };

/* friction laws (friction.f90:700-826, 1147-1264) */
enum {
  FDMAP_FR_FRICTIONLESS = 0,
  FDMAP_FR_LOCKED = 1,
  FDMAP_FR_SW = 2,
  FDMAP_FR_SL = 3,
  FDMAP_FR_FL = 4,
  FDMAP_FR_RSL = 5,
  FDMAP_FR_RFL = 6,
  FDMAP_FR_RSF = 7,
  FDMAP_FR_RAL = 8
};

/* load shapes for the fault nucleation load (friction.f90:1348-1369) */
enum {
  FDMAP_LD_NONE = 0, /* '' */
  FDMAP_LD_UNIFORM = 1,
  FDMAP_LD_LINEAR = 2,
  FDMAP_LD_BOXCAR = 3,
  FDMAP_LD_SMOOTH_BOXCAR = 4,
  FDMAP_LD_TRIANGLE = 5,
  FDMAP_LD_SMOOTH = 6,
  FDMAP_LD_GAUSSIAN = 7
};

/* source time functions (source.f90:208-223) */
enum { FDMAP_STF_RAMP = 0, FDMAP_STF_SINUSOID = 1, FDMAP_STF_GAUSSIAN = 2, FDMAP_STF_RICKER = 3 };

/* per-fault-node fields of fr_type (friction.f90:48), in checkpoint order
 * (checkpoint_friction, friction.f90:528-546) */
enum {
  FDMAP_FAULT_D = 0,
  FDMAP_FAULT_PSI = 1,
  FDMAP_FAULT_DPSI = 2,
  FDMAP_FAULT_TRUP = 3,
  FDMAP_FAULT_V = 4,
  FDMAP_FAULT_O = 5,
  FDMAP_FAULT_S = 6,
  FDMAP_FAULT_N = 7,
  FDMAP_FAULT_S0 = 8,
  FDMAP_FAULT_N0 = 9,
  FDMAP_FAULT_DS = 10,
  FDMAP_FAULT_DN = 11,
  FDMAP_FAULT_DDS = 12,
  FDMAP_FAULT_DDN = 13,
  FDMAP_FAULT_W = 14,
  FDMAP_FAULT_DW = 15,
  FDMAP_FAULT_NREG = 16,
  FDMAP_FAULT_DNREG = 17,
  FDMAP_FAULT_NFIELDS = 18
};

/* one side of a block (bnd_fields, fields.f90:5-20; curve normal, geometry.f90:9-12) */
typedef struct fdmap_side {
  int bc;          /* FDMAP_BC_* */
  int n;           /* number of nodes along the side */
  double* M;       /* (n,5): Zs, Zp, gamma, Ks, Kp        (init_edges, domain.f90:1349) */
  double* F0;      /* (n,nF): initial fields on the side  (init_fields_side, fields.f90:826) */
  double* normal;  /* (n,2): outward unit normal          (interp_block, grid.f90:420-454) */
  double* x;       /* (n): coordinates of side nodes */
  double* y;
} fdmap_side;

/* one block (block_grid + block_material, grid.f90:12-24, material.f90:17-23) */
typedef struct fdmap_block {
  int mgx, pgx, mgy, pgy; /* global 1-based index limits */
  double rho, cs, cp, G, M, gamma, nu; /* block (homogeneous) material */
  double F0[9];           /* block prestress vx0,vy0,vz0,sxx0,sxy0,sxz0,syy0,syz0,szz0
                             (BF%F0, fields.f90:156); mode III faults resolve the
                             in-plane components onto the fault (interfaces.f90:863) */
  fdmap_side side[4];     /* 0=L, 1=R, 2=B, 3=T */
  /* point source for this block (set_source, source.f90:181-204): host-evaluated
   * search results; src_ok=0 when the source point lies outside this block */
  int src_ok, src_i0, src_j0;
  double src_hx, src_hy, src_ax, src_ay;
  /* artificial dissipation coefficient of the block, already scaled by CFL/dt
   * (operator_list Cdiss, domain.f90:172-180, 319); 0 = no dissipation */
  double Cdiss;
  /* perfectly matched layer (pml_list, material.f90:152-222): auxiliary fields
   * Wx (pmlx) / Wy (pmly) with damping sigma*|distance past [mx,px] / [my,py]|^n
   * (sigma itself when n <= 0) and frequency shift kappa.  Its rates
   * (rates_*_mode2_pml, rates.f90:2024-2619) replace the block's ordinary ones
   * in mode II when Cdiss = 0 (time_step.f90:354); mode III ignores it. */
  int pmlx, pmly;
  double pml_n, pml_sigma, pml_kappa, pml_mx, pml_px, pml_my, pml_py;
} fdmap_block;

/* friction state and parameters of one interface (fr_type, friction.f90:38-49) */
typedef struct fdmap_friction {
  int law;          /* FDMAP_FR_* */
  int reg;          /* regularised normal stress */
  int rup_field;    /* 0 = 'V', 1 = 'D' */
  double rup_threshold;
  double angle, xlockm, xlockp, flock, skempton;
  int force;        /* kinematic forcing (FR%force) */
  double kn_c0, kn_fd, kn_dfdx, kn_vL, kn_vR, kn_xL, kn_xR, kn_tmax;
  int ld_shape;     /* FDMAP_LD_* */
  double ld_S, ld_N, ld_T, ld_R, ld_x0, ld_y0;
  int tp_use;       /* thermal pressurisation present: N0 -= p0 (thermpres.f90:477-487) */
  double tp_p0;
  /* per-node parameters (n); rate-and-state and slip-weakening sets */
  double *a, *b, *V0, *f0, *L, *fw, *Vw;
  double *c0, *fs, *fd, *Dc;
  double *bsS0, *bsN0;  /* background stress from stress_file, NULL if absent */
  /* per-node state (n): in at create, out through get_fault */
  double *V, *O, *S, *N, *S0, *N0, *Ds, *Dn, *DDs, *DDn;
  double *Psi, *DPsi, *D, *trup, *W, *DW, *Nreg, *DNreg;
} fdmap_friction;

/* interface between two blocks (iface_type, interfaces.f90:9-20) */
typedef struct fdmap_iface {
  int direction;        /* 0 = 'x' (normal along x), 1 = 'y' */
  int iblockm, iblockp; /* 0-based block indices of the minus and plus sides */
  int m, p;             /* global index range along the interface */
  int coupling;         /* FDMAP_COUPLING_* */
  double* nhat;         /* (n,2) unit normal pointing from minus to plus block */
  double* x;            /* (n) coordinates of interface nodes */
  double* y;
  fdmap_friction fr;
} fdmap_iface;

/* point source (source_type, source.f90:7-17) */
typedef struct fdmap_source {
  int use_singular;     /* point force / moment tensor active */
  int use_gravity;
  int stf;              /* FDMAP_STF_* */
  double x0, y0, t_center, t_duration;
  double Fx, Fy, Fz, Mxx, Mxy, Myy, Mzx, Mzy;
  double gx, gy, gz;
  /* source_list problem = 'Forcing' (source.f90:299-312), mode III only:
   * DF(vz) += amp*exp(-(x/sigma)^2/2 - (y/sigma)^2/2)
   *           * exp(-((t - 4 sigmat)/sigmat)^2/2) / (sigmat*sqrt(2 pi)) */
  int gauss_forcing;
  double gauss_amp, gauss_sigma, gauss_sigmat;
  /* forcing_from_file (source.f90:315-322, 409-502): the file holds one
   * (nx,ny,nF) real*8 frame per time step, frame 0 at the initial time; each
   * step reads the next frame and the stage rates add the two frames
   * interpolated linearly in time.  NULL = no forcing file. */
  const char* forcing_filename;
} fdmap_source;

/* shapes of a fields_perturb item (perturb_fields, fields.f90:900-934) */
enum {
  FDMAP_PERTURB_NONE = 0, /* '' */
  FDMAP_PERTURB_LINEAR = 1,
  FDMAP_PERTURB_BOXCAR = 2,
  FDMAP_PERTURB_TRIANGLE = 3,
  FDMAP_PERTURB_SMOOTH = 4,
  FDMAP_PERTURB_GAUSSIAN = 5
};

/* one fields_perturb item (fields.f90:61-67) */
typedef struct fdmap_perturb {
  int shape;       /* FDMAP_PERTURB_* */
  double x0, y0, Lx, Ly;
  double v[6];     /* perturbation field vector in the mode's field order */
} fdmap_perturb;

/* What the device needs to build one block's body itself (on-device
 * initialisation): the grid follows from the side curves (fdmap_side x, y)
 * and these corners, the initial fields from F0 and the perturbations. */
typedef struct fdmap_block_body {
  double LB[2], LT[2], RB[2], RT[2]; /* block corners (block_list, grid.f90:120-150) */
  double F0[6];                      /* initial fields in the mode's field order */
  fdmap_perturb p[5];                /* fields_list p1..p5 */
  double Cdiss;                      /* operator_list Cdiss before the CFL/dt scaling */
  double* side_mat[4];               /* heterogeneous blocks: (n,3) rho, cs, cp at the
                                        side nodes; NULL for homogeneous blocks */
} fdmap_block_body;

/* On-device initialisation: when fdmap_desc.body is set, the body arrays
 * (F, DF, x, y, metrics, J, Ji) and the side impedances fdmap_side.M are left
 * NULL by the host and the engine builds them on the device (grid.f90:391-618,
 * fields.f90:774-897, domain.f90:1349-1459), reducing hmin and hmax there; the
 * time step is then finished from these set_dt inputs (domain.f90:1462-1535). */
typedef struct fdmap_body {
  fdmap_block_body* blocks; /* nblocks */
  double dt_in, CFL_in, refine, tend;
  int nt_in;
  double c;                 /* sqrt(cs_max^2 + cp_max^2) */
} fdmap_body;

/* the whole domain (domain_type, domain.f90:24-39) */
typedef struct fdmap_desc {
  int mode;             /* 2 = plane strain (nF=6), 3 = antiplane (nF=3) */
  int nF;
  int fd_method;        /* FDMAP_SBP* */
  int rk_order;         /* low-storage RK order 1..4 (time_step.f90:14-68) */
  int nx, ny;           /* global index space */
  int nblocks, nifaces;
  fdmap_block* blocks;
  fdmap_iface* ifaces;
  int heterogeneous;    /* allocated(E%rho): per-node material arrays in use */
  double *F, *DF;       /* (nx,ny,nF) */
  double *x, *y;        /* (nx,ny) node coordinates */
  double *xq, *xr, *yq, *yr, *J, *Ji; /* (nx,ny) metric terms (grid.f90:465-618) */
  double *rho, *cs, *cp, *G, *M, *gamma, *nu; /* (nx,ny) heterogeneous material or NULL */
  fdmap_source src;
  /* time-loop parameters produced by the driver (main.f90:57-116, set_dt) */
  double t0, dt, CFL;
  int nt;
  double hmin, hmax;
  /* non-NULL: body built on the device (t0 is final; dt, CFL, nt, hmin, hmax
   * are finished by the engine, fdmap_gpu_time_params) */
  const fdmap_body* body;
  /* domain_list displacement: body displacement U (nx,ny,nU) integrated from
   * the velocities (set_rates_displacement, fields.f90:1245-1258); peak: peak
   * ground velocity and acceleration pgv, pga (nx,ny) updated in stage 1
   * (update_fields_peak, fields.f90:1136-1164) */
  int displacement, peak;
  /* domain_list energy_balance: the mechanical energy of every block in stage
   * 1 (energy_block, energy.f90:35-96); the boundary energy flux of the
   * reference is a stub (energy_rates_boundary, energy.f90:219-236), so the
   * dissipated energies stay zero */
  int energy_balance;
} fdmap_desc;

#ifdef __cplusplus
}
#endif

#endif /* FDMAP_DESC_H */
